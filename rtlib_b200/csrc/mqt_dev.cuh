// Device-side Morton quadtree routines (MortonQuadTreeT, OPX7UtilsMorton.h:253-449).
#pragma once
#include "common.cuh"
#include "canonical.cuh"

namespace rtpg {

// Deepest supported level: a cell's pyramid of (4^(L+1)-1)/3 int64 sums must fit in shared
// memory during the build (level 7: 175 KB).  RTLib's configured maximum is 6
// (OPX7/CMakeLists.txt:103).
constexpr uint32_t kMqtMaxLevel = 7;
constexpr double kInvPiD = 0.318309886183790691216444201927515678107738494873046875;

struct MqtDev {
    uint32_t ncells, level;
    float fraction;
    FixedPoint fx;
    unsigned long long* leaves;  // ncells * 4^L, building
    float* pyramid;              // ncells * (4^(L+1)-1)/3, sampling
    unsigned* status;
};

__host__ __device__ __forceinline__ uint32_t mqt_level_offset(uint32_t l) { return ((1u << (2 * l)) - 1u) / 3u; }

// MortonUtils::Part1By1_16 / Comp1By1_16 (OPX7UtilsMorton.h:41-89)
__device__ __forceinline__ uint32_t part1by1(uint32_t x) {
    x &= 0x0000FFFF;
    x = (x ^ (x << 8)) & 0x00FF00FF;
    x = (x ^ (x << 4)) & 0x0F0F0F0F;
    x = (x ^ (x << 2)) & 0x33333333;
    x = (x ^ (x << 1)) & 0x55555555;
    return x;
}
__device__ __forceinline__ uint32_t compact1by1(uint32_t x) {
    x &= 0x55555555;
    x = (x ^ (x >> 1)) & 0x33333333;
    x = (x ^ (x >> 2)) & 0x0F0F0F0F;
    x = (x ^ (x >> 4)) & 0x00FF00FF;
    x = (x ^ (x >> 8)) & 0x0000FFFF;
    return x;
}

// leaf Morton code of MortonQuadTreeT::Record (:267-270): uint(uv * 2^L) per axis, clamped
// to 2^L - 1 (uv == 1 would otherwise address past the level)
__device__ __forceinline__ uint32_t mqt_leaf_code(uint32_t level, float u, float v) {
    const float nn = (float)(1u << level);
    const uint32_t maxi = (1u << level) - 1u;
    uint32_t px = __float2uint_rz(__fmul_rn(u, nn)), py = __float2uint_rz(__fmul_rn(v, nn));
    px = px > maxi ? maxi : px;
    py = py > maxi ? maxi : py;
    return (part1by1(py) << 1) + part1by1(px);
}

__device__ __forceinline__ float2 dir_to_canonical_mqt(float x, float y, float z) { return dir_to_canonical(x, y, z); }
__device__ __forceinline__ float3 canonical_to_dir_mqt(float u, float v) { return canonical_to_dir(u, v); }

// MortonQuadTreeT::SampleAndPdf (:286-344), float order as written
// A cell outside [0, ncells) (UINT32_MAX marks a hash-grid miss) samples like an empty
// tree: uniform with pdf 1 (RTLib reads out of bounds there).
__device__ __forceinline__ float2 mqt_sample_and_pdf(const MqtDev& t, uint32_t cell, uint32_t& rng, float& pdf) {
    const float* w = t.pyramid + (size_t)(cell < t.ncells ? cell : 0u) * mqt_level_offset(t.level + 1);
    float total = cell < t.ncells ? w[0] : 0.0f;
    if (total <= 0.0f) {
        const float a = rnd1(rng);
        const float b = rnd1(rng);
        pdf = 1.0f;
        return make_float2(a, b);
    }
    uint32_t size = 4, offset = 1, code = 0;
    for (uint32_t l = 0; l < t.level; ++l) {
        // level offsets (4^l-1)/3 are odd, so the four children are read one by one
        const float* qp = w + offset + (code << 2);
        const float4 q = make_float4(qp[0], qp[1], qp[2], qp[3]);
        // both sides of the first choice as selects of their operands (the same divisions of
        // the same values, without the two divergent branches)
        const float partial_l = __fadd_rn(q.x, q.z);
        const float boundary = __fdiv_rn(partial_l, total);
        const float draw = rnd1(rng);
        const bool right = !(draw < boundary);
        const float partial = right ? __fadd_rn(q.y, q.w) : partial_l;
        const float sample = __fdiv_rn(right ? __fsub_rn(draw, boundary) : draw,
                                       right ? __fsub_rn(1.0f, boundary) : boundary);
        const uint32_t cl = (right ? 1u : 0u) | (sample >= __fdiv_rn(right ? q.y : q.x, partial) ? 2u : 0u);
        total = cl == 0 ? q.x : (cl == 1 ? q.y : (cl == 2 ? q.z : q.w));
        code = (code << 2) + cl;
        offset += size;
        size *= 4;
    }
    const float nn = (float)(1u << t.level);
    const uint32_t xi = compact1by1(code), yi = compact1by1(code >> 1);
    const float rx = rnd1(rng);
    const float px = __fdiv_rn(__fadd_rn((float)xi, rx), nn);
    const float ry = rnd1(rng);
    const float py = __fdiv_rn(__fadd_rn((float)yi, ry), nn);
    pdf = __fmul_rn(__fdiv_rn(total, w[0]), (float)(1u << (2 * t.level)));
    return make_float2(px, py);
}

// MortonQuadTreeT::Pdf (:401-414)
__device__ __forceinline__ float mqt_pdf(const MqtDev& t, uint32_t cell, float u, float v) {
    if (cell >= t.ncells) return 1.0f;
    const float* w = t.pyramid + (size_t)cell * mqt_level_offset(t.level + 1);
    if (w[0] <= 0.0f) return 1.0f;
    const float nn = (float)(1u << t.level);
    const uint32_t idx = mqt_level_offset(t.level) + mqt_leaf_code(t.level, u, v);
    return __fmul_rn(__fmul_rn(__fdiv_rn(w[idx], w[0]), nn), nn);
}

}  // namespace rtpg
