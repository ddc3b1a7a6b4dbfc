// Device-side SD-tree layout and per-query routines (record descent, guided sample, pdf).
//
// Layout in HBM (all capacities fixed at creation, counts live in device memory):
//   STree   snode[i] (u32): leaf -> kLeafBit | dtree index, interior -> index of child 0
//           (child 1 = child 0 + 1).  The split axis of a node is its depth mod 3, as
//           RTLib's SubDivide assigns it (OPX7UtilsPathGuiding.h:1240).
//   DTrees  per tree d: building range b_off/b_cnt, sampling range s_off/s_cnt, building
//           stat-weight (int64 fixed point), sampling sum / area / stat-weight (float),
//           level starts of the breadth-first building tree.
//   pools   building nodes: 4 x u64 fixed-point sums (32 B) + ushort4 local children;
//           sampling nodes: SNode, 32 B = one DRAM sector: float4 sums + ushort4 children.
#pragma once
#include "common.cuh"
#include "limits.cuh"
#include "canonical.cuh"

namespace rtpg {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kMaxLevels = kMaxDTreeDepth + 1;  // level-start entries per tree

struct __align__(32) SNode {
    float4 sums;
    ushort4 child;  // local index of the child quadtree node, 0 = leaf quadrant
    uint32_t pad0, pad1;
};

struct SDTreeDev {
    float3 mn, mx;  // cubified AABB
    FixedPoint fx;
    unsigned* status;
    uint32_t* counts;  // [0] STree nodes, [1] DTrees, [2] building nodes in use
    uint32_t* snode;
    uint32_t* b_off;
    uint32_t* b_cnt;
    uint32_t* s_off;
    uint32_t* s_cnt;
    unsigned long long* b_statw;
    float* s_sum;
    float* s_area;
    float* s_statw;
    uint8_t* s_guided;  // DTreeT::GetMean() > 0 of each sampling tree, set where its sum and stat-weight are
    uint16_t* b_lvl;  // kMaxLevels + 1 per tree
    uint8_t* b_nlvl;
    unsigned long long* b_sums;  // 4 per building node
    ushort4* b_child;
    float* b_area;  // per building node, scratch of the build
    SNode* s_nodes;
    uint32_t cap_snodes, cap_dtrees, cap_nodes;
    uint32_t max_depth;
    float fraction;
};

// STreeT::GetDTreeWrapper (PG.h:639-648) with STreeNodeT::GetChildIdx (PG.h:546-552):
// p = (pos - min) / (max - min); at each interior node p[axis] *= 2, idx = int(p[axis]),
// p[axis] -= idx, the axis cycling x, y, z with depth.  idx is clamped to [0,1] so that
// p == 1 or points outside the box stay in bounds.  The voxel variant also halves the voxel
// size along the split axis per level, as GetDTreeWrapper(p, size) does.
__device__ __forceinline__ bool stree_step(const uint32_t* __restrict__ snode, uint32_t& code, float& p) {
    const float v = __fmul_rn(p, 2.0f);
    int idx = __float2int_rz(v);
    idx = idx < 0 ? 0 : (idx > 1 ? 1 : idx);
    p = __fsub_rn(v, (float)idx);
    code = snode[code + (uint32_t)idx];
    return (code & kLeafBit) != 0;
}
__device__ __forceinline__ uint32_t stree_lookup(const uint32_t* __restrict__ snode, float3 mn, float3 mx, float px,
                                                 float py, float pz) {
    float x = __fdiv_rn(__fsub_rn(px, mn.x), __fsub_rn(mx.x, mn.x));
    float y = __fdiv_rn(__fsub_rn(py, mn.y), __fsub_rn(mx.y, mn.y));
    float z = __fdiv_rn(__fsub_rn(pz, mn.z), __fsub_rn(mx.z, mn.z));
    uint32_t code = snode[0];
    if (!(code & kLeafBit)) {
        for (;;) {
            if (stree_step(snode, code, x)) break;
            if (stree_step(snode, code, y)) break;
            if (stree_step(snode, code, z)) break;
        }
    }
    return code & ~kLeafBit;
}
__device__ __forceinline__ uint32_t stree_lookup_voxel(const uint32_t* __restrict__ snode, float3 mn, float3 mx,
                                                       float px, float py, float pz, float3& voxel) {
    float sx = __fsub_rn(mx.x, mn.x), sy = __fsub_rn(mx.y, mn.y), sz = __fsub_rn(mx.z, mn.z);
    float x = __fdiv_rn(__fsub_rn(px, mn.x), sx);
    float y = __fdiv_rn(__fsub_rn(py, mn.y), sy);
    float z = __fdiv_rn(__fsub_rn(pz, mn.z), sz);
    uint32_t code = snode[0];
    if (!(code & kLeafBit)) {
        for (;;) {
            sx *= 0.5f;
            if (stree_step(snode, code, x)) break;
            sy *= 0.5f;
            if (stree_step(snode, code, y)) break;
            sz *= 0.5f;
            if (stree_step(snode, code, z)) break;
        }
    }
    voxel = make_float3(sx, sy, sz);
    return code & ~kLeafBit;
}

// DTreeNodeT::GetChildIdx (PG.h:69-82)
__device__ __forceinline__ int quad_child(float& u, float& v) {
    int r = 0;
    if (u < 0.5f) u = __fmul_rn(u, 2.0f);
    else { u = __fsub_rn(__fmul_rn(2.0f, u), 1.0f); r |= 1; }
    if (v < 0.5f) v = __fmul_rn(v, 2.0f);
    else { v = __fsub_rn(__fmul_rn(2.0f, v), 1.0f); r |= 2; }
    return r;
}

// Building-tree descent of DTreeNodeT::Record (PG.h:113-125): returns the global index of the
// quadrant sum (node * 4 + quadrant) the record lands in.
__device__ __forceinline__ uint32_t dtree_record_slot(const ushort4* __restrict__ b_child, uint32_t off, float u,
                                                      float v) {
    uint32_t cur = 0;
    int idx = quad_child(u, v);
    for (;;) {
        const ushort4 c = b_child[off + cur];
        const uint32_t nxt = idx == 0 ? c.x : (idx == 1 ? c.y : (idx == 2 ? c.z : c.w));
        if (!nxt) break;
        cur = nxt;
        idx = quad_child(u, v);
    }
    return (off + cur) * 4u + (uint32_t)idx;
}

__device__ __forceinline__ float sel4(const float4& s, int i) { return i == 0 ? s.x : (i == 1 ? s.y : (i == 2 ? s.z : s.w)); }
__device__ __forceinline__ uint32_t sel4(const ushort4& s, int i) { return i == 0 ? s.x : (i == 1 ? s.y : (i == 2 ? s.z : s.w)); }

// DTreeT::GetMean (PG.h:447-451)
__device__ __forceinline__ float dtree_mean(float statw, float sum) {
    if (statw <= 0.0f) return 0.0f;
    const float factor = __fdiv_rn(kInv2Pi, __fmul_rn(2.0f, statw));
    return __fmul_rn(factor, sum);
}

// DTreeT::Pdf (PG.h:485-490) -> DTreeNodeT::Pdf (PG.h:279-320)
__device__ __forceinline__ float dtree_pdf_g(const SNode* __restrict__ nodes, uint32_t off, bool guided, float u,
                                             float v) {
    if (!guided) return __fdiv_rn(__fmul_rn(1.0f, kInv2Pi), 2.0f);
    float result = 1.0f;
    uint32_t cur = 0;
    int idx = quad_child(u, v);
    for (;;) {
        const SNode nd = nodes[off + cur];
        const float4 s = nd.sums;
        const float total = __fadd_rn(__fadd_rn(__fadd_rn(s.x, s.y), s.z), s.w);
        const float si = sel4(s, idx);
        if (si <= 0.0f) {
            result = 0.0f;
            break;
        }
        result = __fmul_rn(result, __fdiv_rn(__fmul_rn(4.0f, si), total));
        const uint32_t c = sel4(nd.child, idx);
        if (!c) break;
        cur = c;
        idx = quad_child(u, v);
    }
    return __fdiv_rn(__fmul_rn(result, kInv2Pi), 2.0f);
}

// The square [x, x + w) x [y, y + w) of the node where a sampling descent stopped, and the
// pdf DTreeNodeT::Pdf gives every point inside it.
struct DSquare {
    float x, y, w, pdf;
    __device__ __forceinline__ bool holds(float u, float v) const { return u >= x && u < x + w && v >= y && v < y + w; }
};

// dtree_pdf_g at (u, v) when the point lies in the square sampling stopped in, else the full
// descent: equal to dtree_pdf_g(nodes, off, guided, u, v) bit for bit either way.
__device__ __forceinline__ float dtree_pdf_in(const SNode* __restrict__ nodes, uint32_t off, bool guided,
                                              const DSquare& sq, float u, float v) {
    return sq.holds(u, v) ? sq.pdf : dtree_pdf_g(nodes, off, guided, u, v);
}

// DTreeT::Sample (PG.h:478-484) -> DTreeNodeT::Sample (PG.h:229-277), float order as written;
// `guided` is DTreeT::GetMean() > 0 (uniform sampling of the square otherwise).  The pdf of
// the sampled point comes out of the same descent: DTreeNodeT::Pdf walks the binary digits of
// (u, v) (quad_child doubles exactly), so for any point inside the square of the node where
// sampling stopped it visits exactly the nodes sampling visited, with the same quadrant sums;
// the factors 4 s_i / total are formed in the same order here.  `sq` returns that square and
// pdf (uniform sampling: the unit square, whose pdf is constant).
__device__ __forceinline__ float2 dtree_sample_sq(const SNode* __restrict__ nodes, uint32_t off, bool guided,
                                                  uint32_t& rng, DSquare& sq) {
    if (!guided) {
        const float a = rnd1(rng);
        const float b = rnd1(rng);
        sq = DSquare{0.0f, 0.0f, 1.0f, __fdiv_rn(__fmul_rn(1.0f, kInv2Pi), 2.0f)};
        return make_float2(a, b);
    }
    uint32_t cur = 0;
    float rx = 0.0f, ry = 0.0f, size = 1.0f, result = 1.0f;
    float bx = 0.0f, by = 0.0f;  // corner of the square where the descent stopped
    for (;;) {
        const SNode nd = nodes[off + cur];
        const float4 s = nd.sums;
        int idx = 0;
        const float topLeft = s.x, topRight = s.y;
        float partial = __fadd_rn(s.x, s.z);
        const float total = __fadd_rn(__fadd_rn(__fadd_rn(s.x, s.y), s.z), s.w);
        float boundary = __fdiv_rn(partial, total);
        float ox = 0.0f, oy = 0.0f;
        float sample = rnd1(rng);
        if (sample < boundary) {
            sample = __fdiv_rn(sample, boundary);
            boundary = __fdiv_rn(topLeft, partial);
        } else {
            partial = __fsub_rn(total, partial);
            ox = 0.5f;
            sample = __fdiv_rn(__fsub_rn(sample, boundary), __fsub_rn(1.0f, boundary));
            boundary = __fdiv_rn(topRight, partial);
            idx |= 1;
        }
        if (sample >= boundary) {
            oy = 0.5f;
            idx |= 2;
        }
        rx = __fadd_rn(rx, __fmul_rn(size, ox));
        ry = __fadd_rn(ry, __fmul_rn(size, oy));
        size = __fmul_rn(size, 0.5f);
        const float si = sel4(s, idx);
        // the pdf descent's step at this node (DTreeNodeT::Pdf, PG.h:295-300)
        if (si <= 0.0f) result = 0.0f;
        else result = __fmul_rn(result, __fdiv_rn(__fmul_rn(4.0f, si), total));
        const uint32_t c = sel4(nd.child, idx);
        if (c == 0 || si <= 0.0f) {
            bx = rx;
            by = ry;
            const float a = rnd1(rng);
            const float b = rnd1(rng);
            rx = __fadd_rn(rx, __fmul_rn(size, a));
            ry = __fadd_rn(ry, __fmul_rn(size, b));
            break;
        }
        cur = c;
    }
    // bx, by and bx + size are dyadic with few bits: the comparisons of holds() are exact
    sq = DSquare{bx, by, size, __fdiv_rn(__fmul_rn(result, kInv2Pi), 2.0f)};
    return make_float2(fminf(fmaxf(rx, 0.0f), 1.0f), fminf(fmaxf(ry, 0.0f), 1.0f));
}

}  // namespace rtpg
