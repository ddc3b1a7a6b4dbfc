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
//           sampling nodes: SNode, 32 B = one DRAM sector: float4 sums + ushort4 children,
//           and beside it SQNode, the 32 B a sampling or pdf descent reads (see there).
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

// What a sampling or pdf descent reads of a sampling node: the quotients of
// the quadrant sums that DTreeNodeT::Sample and ::Pdf (PG.h:229-320) divide out at every visit,
// formed once when the node is written, with the same IEEE operations on the same operands, so
// that a descent reads them instead of dividing (bit-identical results).  A draw of rnd1 is
// s = k 2^-23 for the integer k = (next state) >> 9 < 2^23, and both choices of Sample are
// non-decreasing in s where they can be reached, so each is k >= K for the smallest K that
// makes it (kNever when none does), found by bisecting the 2^23 draws with the divisions
// themselves; the descent compares integers and decides exactly as the divisions would:
//   kb:       s >= bnd, bnd = partial / total, partial = s0 + s2, total = ((s0 + s1) + s2) + s3
//             (quadrant 1 or 3);
//   ktl, ktr: left of bnd, s / bnd >= topLeft / partial; right of it,
//             (s - bnd) / (1 - bnd) >= topRight / (total - partial) (quadrant 2 or 3);
//   fac_i = 4 s_i / total (the pdf factor of quadrant i), 0 where s_i <= 0: there
//         DTreeNodeT::Sample / Pdf stop with pdf 0 (PG.h:268-300), which the product by 0 gives.
//         The factors sit in an array of their own (one float4 per node): the dependent chain
//         of a descent (node -> choice -> child) reads only the 16-byte SQNode, half the
//         footprint in L1, and the factor it multiplies is a load off that chain;
//   meta: bits 0-15 the first child; bits 16 + 4 i .. 19 + 4 i quadrant i's nibble: bit 0 set
//         where the descent stops in quadrant i (no child, or s_i <= 0), bits 1-2 the number of
//         children before quadrant i.
// The children of a node are consecutive in quadrant order (the reset numbers them so, and
// so does the import), so child i = first + the number of children before i.
struct __align__(16) SQNode {
    uint32_t kb, ktl, ktr;
    uint32_t meta;
};
__host__ __device__ inline float sq_div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
__host__ __device__ inline float sq_sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
constexpr uint32_t kDrawSteps = 1u << 23;  // rnd1 draws k 2^-23, k < 2^23
constexpr uint32_t kNever = kDrawSteps;      // a threshold no draw reaches
__host__ __device__ inline float draw_value(uint32_t k) { return (float)k * 0x1p-23f; }
// Sample's choices for draw s: side 0 the first (s >= bnd), side 1 (2) the second left (right)
// of bnd against b = topLeft / partial (topRight / (total - partial))
__host__ __device__ inline bool sq_choice(int side, float s, float bnd, float b) {
    if (side == 0) return !(s < bnd);
    const float q = side == 1 ? sq_div(s, bnd) : sq_div(sq_sub(s, bnd), sq_sub(1.0f, bnd));
    return q >= b;
}
// the smallest k for which sq_choice holds at draw k 2^-23, kNever when none does (bisection
// over the draws; sq_choice is non-decreasing in s where that side is reachable)
__host__ __device__ inline uint32_t sq_threshold(int side, float bnd, float b) {
    uint32_t lo = 0, hi = kDrawSteps - 1;
    if (!sq_choice(side, draw_value(hi), bnd, b)) return kNever;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sq_choice(side, draw_value(mid), bnd, b)) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}
__host__ __device__ inline SQNode make_sqnode(float4 s, ushort4 child, float4& fac) {
    SQNode n;
    const float partial = s.x + s.z;
    const float total = ((s.x + s.y) + s.z) + s.w;
    const float bnd = sq_div(partial, total);
    n.kb = sq_threshold(0, bnd, 0.0f);
    n.ktl = sq_threshold(1, bnd, sq_div(s.x, partial));
    n.ktr = sq_threshold(2, bnd, sq_div(s.y, total - partial));
    const float sq[4] = {s.x, s.y, s.z, s.w};
    const uint32_t c[4] = {child.x, child.y, child.z, child.w};
    uint32_t first = 0, before = 0, nib = 0;
    for (int q = 0; q < 4; ++q) {
        (&fac.x)[q] = sq[q] <= 0.0f ? 0.0f : sq_div(4.0f * sq[q], total);
        if (c[q] && !first) first = c[q];
        nib |= ((!c[q] || sq[q] <= 0.0f ? 1u : 0u) | (before << 1)) << (4 * q);
        if (c[q]) ++before;
    }
    n.meta = (first & 0xffffu) | (nib << 16);
    return n;
}
// quadrant idx's nibble of a meta word (in its low 4 bits; the bits above are not cleared)
__device__ __forceinline__ uint32_t sq_nibble(uint32_t meta, uint32_t idx) { return meta >> (16 + 4 * idx); }
__device__ __forceinline__ bool sq_stops(uint32_t nib) { return (nib & 1u) != 0; }
__device__ __forceinline__ uint32_t sq_child(uint32_t meta, uint32_t nib) { return (meta & 0xffffu) + ((nib >> 1) & 3u); }

struct SDTreeDev {
    float3 mn, mx;  // cubified AABB
    FixedPoint fx;
    unsigned* status;
    uint32_t* counts;  // [0] STree nodes, [1] DTrees, [2] building nodes in use, [3] sampling nodes
    float3 inv_size;   // 1 / (mx - mn) per axis where that size is a power of two, else 0
    uint32_t* snode;
    // the node reached after the first kTopLevels levels (or the leaf above them) for every
    // combination of the first three binary digits of x, y and z; rebuilt whenever the STree changes
    uint32_t* stop;
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
    SQNode* s_q;    // per sampling node, what the descents read
    float4* s_fac;  // per sampling node, the pdf factors of its quadrants
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
// (p - mn) / (mx - mn); inv: the reciprocal of that size where it is a power of two (0 else),
// whose product is the quotient bit for bit
__device__ __forceinline__ float stree_norm(float p, float mn, float mx, float inv) {
    const float d = __fsub_rn(p, mn);
    return inv != 0.0f ? __fmul_rn(d, inv) : __fdiv_rn(d, __fsub_rn(mx, mn));
}
// The child indices stree_step produces along one axis are the binary digits of p: doubling
// and subtracting 1 are exact in float, so for p in [0, 1) level k of that axis yields bit k of
// the fraction, floor(p 2^31) holds the first 31 of them, and frac(p 2^31) (exact) is the p the
// steps would carry on with.  p >= 1 yields 1 at every level and p < 0 or NaN yields 0, with p
// itself carried on.
struct AxisDigits {
    uint32_t bits;
    float s;  // p 2^31 inside [0, 1), p outside
    bool in;
    // the p the steps carry on with after the 31 digits (only walks deeper than 93 levels)
    __device__ __forceinline__ float rest() const { return in ? __fsub_rn(s, __uint2float_rz(bits)) : s; }
};
__device__ __forceinline__ AxisDigits axis_digits(float p) {
    if (p >= 0.0f && p < 1.0f) {
        const float s = __fmul_rn(p, 2147483648.0f);
        return AxisDigits{__float2uint_rz(s), s, true};
    }
    return AxisDigits{p >= 1.0f ? 0x7fffffffu : 0u, p, false};
}
constexpr int kTopLevels = 9;  // 3 digits per axis
constexpr uint32_t kTopCells = 1u << kTopLevels;
// top-table index of the first three digits of each axis (bits 30..28)
__device__ __forceinline__ uint32_t top_cell(uint32_t bx, uint32_t by, uint32_t bz) {
    return (((bx >> 28) & 7u) << 6) | (((by >> 28) & 7u) << 3) | ((bz >> 28) & 7u);
}
// `top` (optional): the table of the first kTopLevels levels (SDTreeDev::stop); the walk then
// starts from the entry and continues with the fourth digit of each axis
__device__ __forceinline__ uint32_t stree_lookup(const uint32_t* __restrict__ snode, float3 mn, float3 mx, float px,
                                                 float py, float pz, float3 inv = float3{0.0f, 0.0f, 0.0f},
                                                 const uint32_t* __restrict__ top = nullptr) {
    uint32_t code = snode[0];
    if (code & kLeafBit) return code & ~kLeafBit;
    const AxisDigits ax = axis_digits(stree_norm(px, mn.x, mx.x, inv.x));
    const AxisDigits ay = axis_digits(stree_norm(py, mn.y, mx.y, inv.y));
    const AxisDigits az = axis_digits(stree_norm(pz, mn.z, mx.z, inv.z));
    int sh0 = 30;
    if (top) {
        code = top[top_cell(ax.bits, ay.bits, az.bits)];
        if (code & kLeafBit) return code & ~kLeafBit;
        sh0 = 30 - kTopLevels / 3;
    }
    // levels 3k, 3k+1, 3k+2 take bit 30-k of x, y, z
    for (int sh = sh0; sh >= 0; --sh) {
        code = snode[code + ((ax.bits >> sh) & 1u)];
        if (code & kLeafBit) return code & ~kLeafBit;
        code = snode[code + ((ay.bits >> sh) & 1u)];
        if (code & kLeafBit) return code & ~kLeafBit;
        code = snode[code + ((az.bits >> sh) & 1u)];
        if (code & kLeafBit) return code & ~kLeafBit;
    }
    // deeper than 93 levels: the per-level steps from where the digits end
    float x = ax.rest(), y = ay.rest(), z = az.rest();
    for (;;) {
        if (stree_step(snode, code, x)) break;
        if (stree_step(snode, code, y)) break;
        if (stree_step(snode, code, z)) break;
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

// DTreeT::Pdf (PG.h:485-490) -> DTreeNodeT::Pdf (PG.h:279-320), with the factors 4 s_i / total
// precomputed per node; the last division by 2 is the exact product by 0.5
__device__ __forceinline__ float dtree_pdf_g(const SQNode* __restrict__ nodes, const float4* __restrict__ facs,
                                             uint32_t off, bool guided, float u, float v) {
    if (!guided) return __fmul_rn(__fmul_rn(1.0f, kInv2Pi), 0.5f);
    float result = 1.0f;
    uint32_t cur = 0;
    int idx = quad_child(u, v);
    for (;;) {
        const uint32_t meta = nodes[off + cur].meta;
        result = __fmul_rn(result, (&facs[off + cur].x)[idx]);  // 0 where s_idx <= 0
        const uint32_t nib = sq_nibble(meta, (uint32_t)idx);
        if (sq_stops(nib)) break;
        cur = sq_child(meta, nib);
        idx = quad_child(u, v);
    }
    return __fmul_rn(__fmul_rn(result, kInv2Pi), 0.5f);
}

// The square [x, x + w) x [y, y + w) of the node where a sampling descent stopped, and the
// pdf DTreeNodeT::Pdf gives every point inside it.
struct DSquare {
    float x, y, w, pdf;
    __device__ __forceinline__ bool holds(float u, float v) const { return u >= x && u < x + w && v >= y && v < y + w; }
};

// dtree_pdf_g at (u, v) when the point lies in the square sampling stopped in, else the full
// descent: equal to dtree_pdf_g(nodes, off, guided, u, v) bit for bit either way.
__device__ __forceinline__ float dtree_pdf_in(const SQNode* __restrict__ nodes, const float4* __restrict__ facs,
                                              uint32_t off, bool guided, const DSquare& sq, float u, float v) {
    return sq.holds(u, v) ? sq.pdf : dtree_pdf_g(nodes, facs, off, guided, u, v);
}

// DTreeT::Sample (PG.h:478-484) -> DTreeNodeT::Sample (PG.h:229-277), float order as written;
// `guided` is DTreeT::GetMean() > 0 (uniform sampling of the square otherwise).  The pdf of
// the sampled point comes out of the same descent: DTreeNodeT::Pdf walks the binary digits of
// (u, v) (quad_child doubles exactly), so for any point inside the square of the node where
// sampling stopped it visits exactly the nodes sampling visited, with the same quadrant sums
// and so the same precomputed factors 4 s_i / total.  `sq` returns that square and
// pdf (uniform sampling: the unit square, whose pdf is constant).
__device__ __forceinline__ float2 dtree_sample_sq(const SQNode* __restrict__ nodes, const float4* __restrict__ facs,
                                                  uint32_t off, bool guided, uint32_t& rng, DSquare& sq) {
    if (!guided) {
        const float a = rnd1(rng);
        const float b = rnd1(rng);
        sq = DSquare{0.0f, 0.0f, 1.0f, __fmul_rn(__fmul_rn(1.0f, kInv2Pi), 0.5f)};
        return make_float2(a, b);
    }
    uint32_t cur = 0;
    float rx = 0.0f, ry = 0.0f, size = 1.0f, result = 1.0f;
    float bx = 0.0f, by = 0.0f;  // corner of the square where the descent stopped
    for (;;) {
        // thresholds and meta word in one 16-byte load; the factors load beside it, off the chain
        const uint4 w = *reinterpret_cast<const uint4*>(nodes + off + cur);
        const float4 f = facs[off + cur];
        const uint32_t meta = w.w;
        const uint32_t k = xs32_next(rng) >> 9;     // rnd1's draw, k 2^-23
        const bool right = k >= w.x;                // quadrant 1 or 3 (kb)
        const bool low = k >= (right ? w.z : w.y);  // quadrant 2 or 3 (ktr, ktl)
        // rx + size * ox with ox in {0, 0.5}: size * 0.5 is exact and adding size * 0 keeps rx
        const float hs = __fmul_rn(size, 0.5f);
        if (right) rx = __fadd_rn(rx, hs);
        if (low) ry = __fadd_rn(ry, hs);
        size = hs;
        // the pdf descent's step at this node (DTreeNodeT::Pdf, PG.h:295-300): 0 where s <= 0
        result = __fmul_rn(result, low ? (right ? f.w : f.z) : (right ? f.y : f.x));
        const uint32_t nib = sq_nibble(meta, (right ? 1u : 0u) | (low ? 2u : 0u));
        if (sq_stops(nib)) {
            bx = rx;
            by = ry;
            const float a = rnd1(rng);
            const float b = rnd1(rng);
            rx = __fadd_rn(rx, __fmul_rn(size, a));
            ry = __fadd_rn(ry, __fmul_rn(size, b));
            break;
        }
        cur = sq_child(meta, nib);
    }
    // bx, by and bx + size are dyadic with few bits: the comparisons of holds() are exact
    sq = DSquare{bx, by, size, __fmul_rn(__fmul_rn(result, kInv2Pi), 0.5f)};
    return make_float2(fminf(fmaxf(rx, 0.0f), 1.0f), fminf(fmaxf(ry, 0.0f), 1.0f));
}

}  // namespace rtpg
