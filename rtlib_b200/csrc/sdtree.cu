// SD-tree on the GPU: record, build, spatial refine + quadtree reset, guided sample / pdf,
// plus the C ABI (rtpg_sdtree_*) and the pass controller (rtpg_controller_*).
//
// RTLib keeps the tree on the host and round-trips it through PCIe every pass
// (RTSTreeWrapperT::Download / Build / Reset / Upload, OPX7UtilsPathGuiding.h:1353-1728,
// driven by RTSTreeControllerT::BegTrace/EndTrace :1808-1887).  Here every step is a kernel
// on device-resident arrays; counts stay in device memory so a whole pass can be captured
// in a CUDA graph.
#include <math.h>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <new>

#include "common.cuh"
#include "sdtree_dev.cuh"

namespace rtpg {

constexpr int kRecordBlock = 256;
constexpr int kTreeBlock = 256;
constexpr uint32_t kVirtual = 0xffffffffu;

// ------------------------------------------------------------------ clear
__global__ void k_clear(SDTreeDev t) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        t.counts[0] = 1;
        t.counts[1] = 1;
        t.counts[2] = 1;
        t.counts[3] = 1;
        t.snode[0] = kLeafBit | 0u;
        t.b_off[0] = 0; t.b_cnt[0] = 1; t.s_off[0] = 0; t.s_cnt[0] = 1;
        t.b_statw[0] = 0ull;
        t.s_sum[0] = 0.0f; t.s_area[0] = 0.0f; t.s_statw[0] = 0.0f; t.s_guided[0] = 0;
        t.b_lvl[0] = 0; t.b_lvl[1] = 1; t.b_nlvl[0] = 1;
        for (int q = 0; q < 4; ++q) t.b_sums[q] = 0ull;
        t.b_child[0] = make_ushort4(0, 0, 0, 0);
        SNode z;
        z.sums = make_float4(0.f, 0.f, 0.f, 0.f);
        z.child = make_ushort4(0, 0, 0, 0);
        z.pad0 = z.pad1 = 0;
        t.s_nodes[0] = z;
        t.s_q[0] = make_sqnode(z.sums, z.child, t.s_fac[0]);
    }
}

// The STree's top table (SDTreeDev::stop): entry c holds the node the first kTopLevels steps
// reach for digits x = c >> 6, y = (c >> 3) & 7, z = c & 7 (three per axis, most significant
// first), or the leaf where the walk stops earlier -- exactly what stree_lookup's per-level
// steps give for those digits.
__global__ void k_stree_top(SDTreeDev t) {
    grid_dependency_wait();
    for (uint32_t c = threadIdx.x; c < kTopCells; c += blockDim.x) {
        const uint32_t d[3] = {c >> 6, (c >> 3) & 7u, c & 7u};
        uint32_t code = t.snode[0];
        for (int l = 0; l < kTopLevels && !(code & kLeafBit); ++l)
            code = t.snode[code + ((d[l % 3] >> (2 - l / 3)) & 1u)];
        t.stop[c] = code;
    }
}

// ------------------------------------------------------------------ record
// One thread per record (grid-stride, warp-uniform trip count so that the warp-aggregated
// atomics run converged).  Two 64-bit fixed-point atomics per record: the DTree's stat-weight
// and the leaf quadrant sum (RecordIrradiance, PG.h:417-428).  When the whole tree is small
// (at most kPrivQuads quadrants and kPrivTrees DTrees) every CTA accumulates in shared memory
// and flushes once, which removes the same-address contention of a freshly cleared tree.
constexpr uint32_t kPrivQuads = 2048;
constexpr uint32_t kPrivTrees = 512;
constexpr uint32_t kStageSTreeRecord = 4096;  // 16 KB + 16 KB + 4 KB of static shared memory
template <bool CANON>
__global__ void __launch_bounds__(kRecordBlock) k_record(SDTreeDev t, int64_t n, const float* __restrict__ pos,
                                                         const float* __restrict__ dir, const float* __restrict__ radiance,
                                                         const float* __restrict__ wo_pdf,
                                                         const float* __restrict__ stat_w,
                                                         const uint8_t* __restrict__ is_delta) {
    __shared__ uint32_t s_st[kStageSTreeRecord];
    __shared__ unsigned long long s_q[kPrivQuads];
    __shared__ unsigned long long s_w[kPrivTrees];
    const uint32_t nst = t.counts[0];
    const uint32_t nq = t.counts[2] * 4u, ndt = t.counts[1];
    const bool staged = nst <= kStageSTreeRecord;
    const bool priv = nq <= kPrivQuads && ndt <= kPrivTrees;
    if (staged)
        for (uint32_t i = threadIdx.x; i < nst; i += blockDim.x) s_st[i] = t.snode[i];
    if (priv) {
        for (uint32_t i = threadIdx.x; i < nq; i += blockDim.x) s_q[i] = 0ull;
        for (uint32_t i = threadIdx.x; i < ndt; i += blockDim.x) s_w[i] = 0ull;
    }
    __syncthreads();
    const uint32_t* st = staged ? s_st : t.snode;
    unsigned long long* acc_w = priv ? s_w : t.b_statw;
    unsigned long long* acc_q = priv ? s_q : t.b_sums;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        unsigned long long k_w = ~0ull, k_s = ~0ull, v_w = 0, v_s = 0;
        if (i < n && !(is_delta && is_delta[i])) {
            const float wo = wo_pdf ? wo_pdf[i] : 1.0f;
            const float sw = stat_w ? stat_w[i] : 1.0f;
            const float irr = __fdiv_rn(radiance[i], wo);
            if (isfinite(sw) && sw > 0.0f) {
                const uint32_t d = stree_lookup(st, t.mn, t.mx, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], t.inv_size,
                                                staged ? nullptr : t.stop);
                k_w = d;
                v_w = to_fx(sw, t.fx, t.status);
                if (isfinite(irr) && irr > 0.0f) {
                    float u, v;
                    if (CANON) {
                        const float2 c = reinterpret_cast<const float2*>(dir)[i];
                        u = c.x; v = c.y;
                    } else {
                        const float2 c = dir_to_canonical(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
                        u = c.x; v = c.y;
                    }
                    k_s = dtree_record_slot(t.b_child, t.b_off[d], u, v);
                    v_s = to_fx(__fmul_rn(irr, sw), t.fx, t.status);
                }
            }
        }
        if (priv) {
            // shared-memory sums: a warp's records spread over many quadrants, so plain
            // 64-bit shared atomics beat aggregating them first
            if (k_w != ~0ull) atomicAdd(acc_w + k_w, v_w);
            if (k_s != ~0ull) atomicAdd(acc_q + k_s, v_s);
        } else {
            warp_add_u64(k_w, v_w, acc_w);
            warp_add_u64(k_s, v_s, acc_q);
        }
    }
    if (priv) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nq; i += blockDim.x)
            if (s_q[i]) atomicAdd(t.b_sums + i, s_q[i]);
        for (uint32_t i = threadIdx.x; i < ndt; i += blockDim.x)
            if (s_w[i]) atomicAdd(t.b_statw + i, s_w[i]);
    }
}

// zeroes n 64-bit counters (a kernel rather than a memset so the refine chain stays a chain of
// dependent launches)
__global__ void k_zero_u64(unsigned long long* p, int n) {
    grid_dependency_wait();
    if (threadIdx.x < n) p[threadIdx.x] = 0ull;
}

// ------------------------------------------------------------------ build
// One CTA per DTree (grid-stride over trees).  Levels of the breadth-first building tree are
// processed deepest first: an interior quadrant's fixed-point sum is the exact sum of its
// child's four quadrants (DTreeNodeT::Build, PG.h:356-369).  Then the float sums, the area
// (DTreeNodeT::GetArea, PG.h:342-355, same float order), the root sum (RTDTreeT::Build,
// PG.h:948-957) and the sampling copy (RTDTreeWrapperT::Build, PG.h:1086-1090).
__global__ void __launch_bounds__(kTreeBlock) k_build(SDTreeDev t) {
    grid_dependency_wait();
    const uint32_t ndt = t.counts[1];
    for (uint32_t d = blockIdx.x; d < ndt; d += gridDim.x) {
        const uint32_t off = t.b_off[d];
        const uint32_t cnt = t.b_cnt[d];
        const int nl = t.b_nlvl[d];
        const uint16_t* lv = t.b_lvl + size_t(d) * (kMaxLevels + 1);
        for (int l = nl - 2; l >= 0; --l) {
            const uint32_t a = lv[l], b = lv[l + 1];
            for (uint32_t j = a + threadIdx.x; j < b; j += blockDim.x) {
                const ushort4 c = t.b_child[off + j];
                const uint32_t cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (cc[q]) {
                        const unsigned long long* s = t.b_sums + size_t(off + cc[q]) * 4;
                        t.b_sums[size_t(off + j) * 4 + q] = s[0] + s[1] + s[2] + s[3];
                    }
                }
            }
            __syncthreads();
        }
        // area bottom-up, writes sampling nodes
        for (int l = nl - 1; l >= 0; --l) {
            const uint32_t a = lv[l], b = lv[l + 1];
            for (uint32_t j = a + threadIdx.x; j < b; j += blockDim.x) {
                const ushort4 c = t.b_child[off + j];
                const uint32_t cc[4] = {c.x, c.y, c.z, c.w};
                const unsigned long long* s = t.b_sums + size_t(off + j) * 4;
                float f[4];
                float area = 0.0f;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    f[q] = fx_to_float(s[q], t.fx);
                    if (f[q] > 0.0f) {
                        if (!cc[q]) area = __fadd_rn(area, 0.25f);
                        else area = __fadd_rn(area, __fdiv_rn(t.b_area[off + cc[q]], 4.0f));
                    }
                }
                t.b_area[off + j] = area;
                SNode nd;
                nd.sums = make_float4(f[0], f[1], f[2], f[3]);
                nd.child = c;
                nd.pad0 = nd.pad1 = 0;
                t.s_nodes[off + j] = nd;
                t.s_q[off + j] = make_sqnode(nd.sums, c, t.s_fac[off + j]);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const float4 r = t.s_nodes[off].sums;
            const float sum = __fadd_rn(__fadd_rn(__fadd_rn(r.x, r.y), r.z), r.w);
            const float statw = fx_to_float(t.b_statw[d], t.fx);
            t.s_sum[d] = sum;
            t.s_area[d] = t.b_area[off];
            t.s_statw[d] = statw;
            t.s_guided[d] = dtree_mean(statw, sum) > 0.0f ? 1 : 0;  // read per query instead of recomputed
            t.s_off[d] = off;
            t.s_cnt[d] = cnt;
        }
        __syncthreads();
    }
    // every building node is now a sampling node, at the same index
    if (blockIdx.x == 0 && threadIdx.x == 0) t.counts[3] = t.counts[2];
}

// ------------------------------------------------------------------ spatial refine
// Footprint guard of RTSTreeT::Refine (PG.h:1276-1285): 24-byte nodes and 24-byte headers
// of the building and sampling tree of every STree node; interior nodes hold default
// one-node trees (SubDivide resets the parent's wrapper, PG.h:1246).
__global__ void k_footprint(SDTreeDev t, unsigned long long* fp) {
    grid_dependency_wait();
    const uint32_t n = t.counts[0];
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = t.snode[i];
        if (c & kLeafBit) {
            const uint32_t d = c & ~kLeafBit;
            s += 24ull * (t.b_cnt[d] + t.s_cnt[d]) + 48ull;
        } else {
            s += 96ull;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(fp, s);
}

// Per STree node: how many halvings of the building stat-weight stay above the threshold
// (ShallSplit, PG.h:1270-1274, cascading through SubDivide's w/2, PG.h:1243).  A leaf that
// splits k times becomes a complete subtree with 2^(k+1)-2 new nodes and 2^k leaves.
// tot64[1] / tot64[2] receive the 64-bit totals of new STree nodes / DTrees, which the apply
// step checks against the capacities (the 32-bit scan totals could wrap).
__global__ void k_refine_count(SDTreeDev t, float thf, int32_t max_mb, uint32_t kmax, unsigned long long* tot64,
                               uint32_t* cnt_s, uint32_t* cnt_d, uint32_t* ksplit) {
    grid_dependency_wait();
    const uint32_t n = t.counts[0];
    const bool allowed = max_mb < 0 || (tot64[0] / 1000000ull) < (unsigned long long)max_mb;
    unsigned long long ss = 0, sd = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = t.snode[i];
        uint32_t k = 0;
        if (allowed && (c & kLeafBit)) {
            float w = fx_to_float(t.b_statw[c & ~kLeafBit], t.fx);
            while (w > thf && k < kmax) {
                w = __fdiv_rn(w, 2.0f);
                ++k;
            }
            if (w > thf) atomicOr(t.status, RTPG_STATUS_STREE_CAPACITY);  // depth capped by capacity
        }
        ksplit[i] = k;
        cnt_s[i] = k ? (2u << k) - 2u : 0u;
        cnt_d[i] = k ? (1u << k) - 1u : 0u;
        ss += cnt_s[i];
        sd += cnt_d[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ss += __shfl_down_sync(0xffffffffu, ss, o);
        sd += __shfl_down_sync(0xffffffffu, sd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (ss) atomicAdd(tot64 + 1, ss);
        if (sd) atomicAdd(tot64 + 2, sd);
    }
}

// Writes the complete subtrees, one thread per new STree node and one per new DTree (the
// owning leaf is found by binary search in the scanned offsets).  New nodes are numbered level
// by level inside each leaf's block; leaf j of a subtree gets the old DTree (j == 0) or a new
// one that shares the parent's sampling quadtree (read-only until the next build) --
// SubDivide copies the whole wrapper into both children (PG.h:1236-1244).
__device__ __forceinline__ uint32_t owner_of(const uint32_t* off, const uint32_t* cnt, uint32_t n, uint32_t q) {
    uint32_t lo = 0, hi = n;  // last i with off[i] <= q and cnt[i] > 0
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (off[m] <= q) lo = m;
        else hi = m;
    }
    while (cnt[lo] == 0 || off[lo] > q) --lo;  // skip empty entries sharing the same offset
    return lo;
}
__global__ void k_refine_apply(SDTreeDev t, const uint32_t* ksplit, const uint32_t* off_s, const uint32_t* cnt_s,
                               const uint32_t* off_d, const uint32_t* cnt_d, const unsigned long long* tot64) {
    grid_dependency_wait();
    const uint32_t n = t.counts[0], ndt = t.counts[1];
    if (n + tot64[1] > t.cap_snodes || ndt + tot64[2] > t.cap_dtrees) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(t.status, RTPG_STATUS_STREE_CAPACITY);
        return;
    }
    const uint32_t tot_s = (uint32_t)tot64[1], tot_d = (uint32_t)tot64[2];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < tot_s; q += stride) {
        const uint32_t i = owner_of(off_s, cnt_s, n, q);
        const uint32_t k = ksplit[i];
        const uint32_t B = n + off_s[i];
        const uint32_t r = q - off_s[i];  // position in the block: level l holds [2^l - 2, 2^(l+1) - 2)
        const uint32_t l = 31 - __clz(r + 2);
        const uint32_t j = r + 2 - (1u << l);
        if (l < k) {
            t.snode[B + r] = B + (2u << l) - 2 + 2 * j;
        } else {
            const uint32_t dold = t.snode[i] & ~kLeafBit;
            t.snode[B + r] = kLeafBit | (j == 0 ? dold : ndt + off_d[i] + j - 1);
        }
    }
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < tot_d; q += stride) {
        const uint32_t i = owner_of(off_d, cnt_d, n, q);
        const uint32_t dold = t.snode[i] & ~kLeafBit;
        const uint32_t d = ndt + q;
        // building fields alias the parent's tree until the quadtree reset writes the new one;
        // they only remain if the reset hits a capacity limit (RTPG_STATUS_DNODE_CAPACITY),
        // which keeps later records in bounds
        t.b_off[d] = t.b_off[dold];
        t.b_cnt[d] = t.b_cnt[dold];
        t.b_nlvl[d] = t.b_nlvl[dold];
        t.b_statw[d] = 0ull;
        for (uint32_t x = 0; x <= kMaxLevels; ++x)
            t.b_lvl[size_t(d) * (kMaxLevels + 1) + x] = t.b_lvl[size_t(dold) * (kMaxLevels + 1) + x];
        t.s_off[d] = t.s_off[dold];
        t.s_cnt[d] = t.s_cnt[dold];
        t.s_sum[d] = t.s_sum[dold];
        t.s_area[d] = t.s_area[dold];
        t.s_statw[d] = t.s_statw[dold];
        t.s_guided[d] = t.s_guided[dold];
    }
}
// the split leaves become interior nodes; runs after k_refine_apply read snode[i]
__global__ void k_refine_link(SDTreeDev t, const uint32_t* ksplit, const uint32_t* off_s,
                              const unsigned long long* tot64) {
    grid_dependency_wait();
    const uint32_t n = t.counts[0], ndt = t.counts[1];
    if (n + tot64[1] > t.cap_snodes || ndt + tot64[2] > t.cap_dtrees) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (ksplit[i]) t.snode[i] = n + off_s[i];
}
__global__ void k_refine_commit(SDTreeDev t, const unsigned long long* tot64) {
    grid_dependency_wait();
    const uint32_t n = t.counts[0], ndt = t.counts[1];
    if (n + tot64[1] > t.cap_snodes || ndt + tot64[2] > t.cap_dtrees) return;
    t.counts[0] = n + (uint32_t)tot64[1];
    t.counts[1] = ndt + (uint32_t)tot64[2];
}

// ------------------------------------------------------------------ quadtree reset
// RTDTreeT::Reset (PG.h:888-947) breadth first, one CTA per tree.  New node j either mirrors
// node src[j] of the tree's sampling quadtree or -- under a sampling leaf quadrant -- is a
// "copy of itself" whose four sums are vsum[j] = parent quadrant / 4 (PG.h:926-933).
// Quadrant i of a node at depth `depth` gets a child iff depth < maxDepth and
// sum_i / total > th (total = sampling root sum; 0.25^depth when total <= 0).  Children are
// numbered in (node, quadrant) order via a block scan, level by level; the same pass runs
// twice, first to count, then to write at the scanned offset.
template <bool WRITE>
__global__ void __launch_bounds__(kTreeBlock) k_reset(SDTreeDev t, float th, uint32_t* node_count,
                                                      const uint32_t* node_off, unsigned long long* node_total) {
    grid_dependency_wait();
    extern __shared__ uint32_t sm[];
    uint32_t* src = sm;                                              // kDTreeNodeCap
    float* vsum = reinterpret_cast<float*>(sm + kDTreeNodeCap);      // kDTreeNodeCap
    __shared__ uint32_t warp_tot[kTreeBlock / 32];
    __shared__ uint32_t s_ntotal;
    if (WRITE && *node_total > t.cap_nodes) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(t.status, RTPG_STATUS_DNODE_CAPACITY);
        return;
    }
    const uint32_t ndt = t.counts[1];
    for (uint32_t d = blockIdx.x; d < ndt; d += gridDim.x) {
        const float total = t.s_sum[d];
        const uint32_t soff = t.s_off[d];
        const uint32_t boff = WRITE ? node_off[d] : 0;
        uint16_t* lv = t.b_lvl + size_t(d) * (kMaxLevels + 1);
        if (threadIdx.x == 0) {
            src[0] = 0;
            vsum[0] = 0.0f;
            s_ntotal = 1;
            if (WRITE) lv[0] = 0;
        }
        __syncthreads();
        uint32_t lvl_start = 0, lvl_end = 1, nlev = 0;
        int depth = 1;
        while (lvl_start < lvl_end) {
            const float frac_empty = ldexpf(1.0f, -2 * depth);
            for (uint32_t chunk = lvl_start; chunk < lvl_end; chunk += blockDim.x) {
                const uint32_t j = chunk + threadIdx.x;
                uint32_t mask = 0;
                float si[4] = {0.f, 0.f, 0.f, 0.f};
                ushort4 sc = make_ushort4(0, 0, 0, 0);
                uint32_t s = kVirtual;
                if (j < lvl_end) {
                    s = src[j];
                    if (s != kVirtual) {
                        const SNode nd = t.s_nodes[soff + s];
                        si[0] = nd.sums.x; si[1] = nd.sums.y; si[2] = nd.sums.z; si[3] = nd.sums.w;
                        sc = nd.child;
                    } else {
                        si[0] = si[1] = si[2] = si[3] = vsum[j];
                    }
                    if (depth < (int)t.max_depth) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float f = total > 0.0f ? __fdiv_rn(si[q], total) : frac_empty;
                            if (f > th) mask |= 1u << q;
                        }
                    }
                }
                const uint32_t base = s_ntotal;
                uint32_t tot;
                uint32_t next = base + block_exclusive_scan<kTreeBlock>(__popc(mask), warp_tot, tot);
                ushort4 out = make_ushort4(0, 0, 0, 0);
                if (j < lvl_end) {
                    const uint32_t scc[4] = {sc.x, sc.y, sc.z, sc.w};
                    uint32_t oc[4] = {0, 0, 0, 0};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (mask & (1u << q)) {
                            const uint32_t idx = next++;
                            if (idx < kDTreeNodeCap) {
                                if (s != kVirtual && scc[q]) { src[idx] = scc[q]; vsum[idx] = 0.0f; }
                                else { src[idx] = kVirtual; vsum[idx] = __fdiv_rn(si[q], 4.0f); }
                                oc[q] = idx;
                            }
                        }
                    }
                    out = make_ushort4(oc[0], oc[1], oc[2], oc[3]);
                    if (WRITE) t.b_child[boff + j] = out;
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    uint32_t nt = base + tot;
                    if (nt > kDTreeNodeCap) {
                        nt = kDTreeNodeCap;
                        atomicOr(t.status, RTPG_STATUS_DTREE_NODE_CAP);
                    }
                    s_ntotal = nt;
                }
                __syncthreads();
            }
            lvl_start = lvl_end;
            lvl_end = s_ntotal;
            ++nlev;
            ++depth;
            if (WRITE && threadIdx.x == 0) lv[nlev] = (uint16_t)lvl_start;
        }
        const uint32_t cnt = s_ntotal;
        if (!WRITE) {
            if (threadIdx.x == 0) {
                node_count[d] = cnt;
                atomicAdd(node_total, (unsigned long long)cnt);
            }
        } else {
            for (uint32_t j = threadIdx.x; j < 4 * cnt; j += blockDim.x) t.b_sums[size_t(boff) * 4 + j] = 0ull;
            if (threadIdx.x == 0) {
                t.b_off[d] = boff;
                t.b_cnt[d] = cnt;
                t.b_statw[d] = 0ull;
                t.b_nlvl[d] = (uint8_t)nlev;
            }
        }
        __syncthreads();
    }
}
__global__ void k_reset_commit(SDTreeDev t, const unsigned long long* node_total) {
    grid_dependency_wait();
    if (*node_total <= t.cap_nodes) t.counts[2] = (uint32_t)*node_total;
}

// ------------------------------------------------------------------ sample / pdf
// One query per thread: STree descent (tree staged in shared memory when it fits), the
// DTree's GetMean test once, the guided sample, the pdf of the sampled canonical point
// (DTreeT::Pdf) and optionally the direction and the pdf of that direction after the
// dir -> canonical round trip the closest-hit program performs (SimpleGuide.cu:361-368).
// The descents read the 32-byte SQNode of each visited node and the STree through L1.  Staging
// them in shared memory measured slower on B200 (config 1 / its 2-pass variant: 64.8 / 23.7 G
// queries/s with the STree and the whole pool staged, 63.4 / 28.4 with every tree's root
// level staged, 65.5 / 31.1 with no staging): the shared memory comes out of the same 256 KB
// per SM as L1, which then no longer holds the deeper levels.
constexpr uint32_t kSampleBlock = 256;
// largest query count whose 3 n element offsets (plus a grid stride) stay inside int32
constexpr int64_t kMaxIndex32 = (int64_t(1) << 31) / 4;
// I: the query index type (32-bit while 3 n fits, which saves the 64-bit address arithmetic)
template <class I>
__global__ void __launch_bounds__(kSampleBlock, 8) k_sample_pdf(SDTreeDev t, I n, const float* __restrict__ pos,
                                                               const uint32_t* __restrict__ seeds, uint32_t seed_base,
                                                               float* __restrict__ out_uv, float* __restrict__ out_pdf_uv,
                                                               float* __restrict__ out_dir, float* __restrict__ out_pdf_dir) {
    const I stride = I(gridDim.x) * I(blockDim.x);
    for (I i = I(blockIdx.x) * I(blockDim.x) + I(threadIdx.x); i < n; i += stride) {
        const uint32_t d = stree_lookup(t.snode, t.mn, t.mx, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], t.inv_size, t.stop);
        uint32_t rng = seeds ? seeds[i] : (pcg1d(seed_base + (uint32_t)i) | 1u);
        const uint32_t off = t.s_off[d];
        const bool guided = t.s_guided[d] != 0;
        DSquare sq;
        const float2 uv = dtree_sample_sq(t.s_q, t.s_fac, off, guided, rng, sq);
        if (out_uv) reinterpret_cast<float2*>(out_uv)[i] = uv;
        if (out_pdf_uv) out_pdf_uv[i] = dtree_pdf_in(t.s_q, t.s_fac, off, guided, sq, uv.x, uv.y);
        if (out_dir || out_pdf_dir) {
            const float3 dv = normalize3(canonical_to_dir(uv.x, uv.y));
            if (out_dir) {
                out_dir[3 * i] = dv.x;
                out_dir[3 * i + 1] = dv.y;
                out_dir[3 * i + 2] = dv.z;
            }
            if (out_pdf_dir) {
                const float2 c = dir_to_canonical(dv.x, dv.y, dv.z);
                out_pdf_dir[i] = dtree_pdf_in(t.s_q, t.s_fac, off, guided, sq, c.x, c.y);
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_pdf(SDTreeDev t, int64_t n, const float* __restrict__ pos,
                                             const float* __restrict__ dir, int canonical, float* __restrict__ out) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t d = stree_lookup(t.snode, t.mn, t.mx, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], t.inv_size, t.stop);
        float2 c;
        if (canonical) c = reinterpret_cast<const float2*>(dir)[i];
        else c = dir_to_canonical(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        out[i] = dtree_pdf_g(t.s_q, t.s_fac, t.s_off[d], t.s_guided[d] != 0, c.x, c.y);
    }
}

}  // namespace rtpg

using namespace rtpg;

// ================================================================== host object
struct rtpg_sdtree {
    SDTreeDev dev{};
    float mn[3], mx[3];
    uint32_t max_depth = 20;
    float fraction = 0.3f;
    int bits = 24;
    std::vector<void*> allocs;
    // refine scratch
    uint32_t *cnt_s = nullptr, *off_s = nullptr, *cnt_d = nullptr, *off_d = nullptr, *ksplit = nullptr;
    uint32_t *partials = nullptr, *totals = nullptr, *node_cnt = nullptr, *node_off = nullptr;
    unsigned long long* fp = nullptr;
    size_t bytes = 0;

    template <class T>
    int alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, count * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(RTPG_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        allocs.push_back(q);
        bytes += count * sizeof(T);
        *p = static_cast<T*>(q);
        return RTPG_OK;
    }
    ~rtpg_sdtree() {
        for (void* p : allocs) cudaFree(p);
    }
};

namespace rtpg {
SDTreeDev sdtree_device_view(const rtpg_sdtree* t) { return t->dev; }
}

static int sdtree_clear(rtpg_sdtree* h, cudaStream_t st) {
    RTPG_CUDA(cudaMemsetAsync(h->dev.status, 0, sizeof(unsigned), st));
    k_clear<<<1, 32, 0, st>>>(h->dev);
    k_stree_top<<<1, kTopCells, 0, st>>>(h->dev);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

static int reset_smem() { return int(kDTreeNodeCap * 8); }

extern "C" {

int rtpg_sdtree_create(const float* aabb_min, const float* aabb_max, uint32_t max_dtree_depth, float fraction,
                       const rtpg_sdtree_caps* caps, rtpg_sdtree** out) {
    if (!aabb_min || !aabb_max || !out) return fail(RTPG_EINVAL, "rtpg_sdtree_create: null argument");
    if (max_dtree_depth < 1 || max_dtree_depth > kMaxDTreeDepth)
        return fail(RTPG_EINVAL, "rtpg_sdtree_create: max_dtree_depth must be in [1, %u]", kMaxDTreeDepth);
    rtpg_sdtree_caps c{1u << 20, 1u << 19, 1u << 23, 24};
    if (caps) {
        if (caps->max_stree_nodes) c.max_stree_nodes = caps->max_stree_nodes;
        if (caps->max_dtrees) c.max_dtrees = caps->max_dtrees;
        if (caps->max_dtree_nodes_total) c.max_dtree_nodes_total = caps->max_dtree_nodes_total;
        if (caps->fixed_point_bits) c.fixed_point_bits = caps->fixed_point_bits;
    }
    if (c.fixed_point_bits < 0 || c.fixed_point_bits > 40)
        return fail(RTPG_EINVAL, "rtpg_sdtree_create: fixed_point_bits must be in [0, 40]");
    if (c.max_stree_nodes >= kLeafBit || c.max_dtrees >= kLeafBit || c.max_dtree_nodes_total >= (1u << 31))
        return fail(RTPG_EINVAL, "rtpg_sdtree_create: capacities must be below 2^31");
    for (int k = 0; k < 3; ++k)
        if (!(aabb_max[k] >= aabb_min[k]) || !isfinite(aabb_min[k]) || !isfinite(aabb_max[k]))
            return fail(RTPG_EINVAL, "rtpg_sdtree_create: invalid AABB");
    auto* h = new (std::nothrow) rtpg_sdtree();
    if (!h) return fail(RTPG_ENOMEM, "rtpg_sdtree_create: out of host memory");
    // RTSTreeT ctor (PG.h:1211-1217): cubify to the largest extent
    const float sx = aabb_max[0] - aabb_min[0], sy = aabb_max[1] - aabb_min[1], sz = aabb_max[2] - aabb_min[2];
    const float m = std::max(std::max(sx, sy), sz);
    for (int k = 0; k < 3; ++k) {
        h->mn[k] = aabb_min[k];
        h->mx[k] = aabb_min[k] + m;
    }
    h->max_depth = max_dtree_depth;
    h->fraction = fraction;
    h->bits = c.fixed_point_bits;
    SDTreeDev& t = h->dev;
    t.mn = make_float3(h->mn[0], h->mn[1], h->mn[2]);
    t.mx = make_float3(h->mx[0], h->mx[1], h->mx[2]);
    {
        // a division by a power of two equals the product with its reciprocal, bit for bit
        float inv[3];
        for (int k = 0; k < 3; ++k) {
            const float d = h->mx[k] - h->mn[k];
            int e = 0;
            inv[k] = (d > 0.0f && std::isfinite(d) && std::frexp(d, &e) == 0.5f && e > -120 && e < 120)
                         ? std::ldexp(1.0f, 1 - e) : 0.0f;
        }
        t.inv_size = make_float3(inv[0], inv[1], inv[2]);
    }
    t.fx.scale = ldexpf(1.0f, c.fixed_point_bits);
    t.fx.inv_scale = ldexpf(1.0f, -c.fixed_point_bits);
    t.cap_snodes = c.max_stree_nodes;
    t.cap_dtrees = c.max_dtrees;
    t.cap_nodes = c.max_dtree_nodes_total;
    t.max_depth = max_dtree_depth;
    t.fraction = fraction;
    int r = RTPG_OK;
    const size_t nd = c.max_dtrees, nn = c.max_dtree_nodes_total, ns = c.max_stree_nodes;
    if ((r = h->alloc(&t.status, 1)) || (r = h->alloc(&t.counts, 4)) || (r = h->alloc(&t.snode, ns)) ||
        (r = h->alloc(&t.stop, kTopCells)) ||
        (r = h->alloc(&t.b_off, nd)) || (r = h->alloc(&t.b_cnt, nd)) || (r = h->alloc(&t.s_off, nd)) ||
        (r = h->alloc(&t.s_cnt, nd)) || (r = h->alloc(&t.b_statw, nd)) || (r = h->alloc(&t.s_sum, nd)) ||
        (r = h->alloc(&t.s_area, nd)) || (r = h->alloc(&t.s_statw, nd)) || (r = h->alloc(&t.s_guided, nd)) ||
        (r = h->alloc(&t.b_lvl, nd * (kMaxLevels + 1))) || (r = h->alloc(&t.b_nlvl, nd)) ||
        (r = h->alloc(&t.b_sums, nn * 4)) || (r = h->alloc(&t.b_child, nn)) || (r = h->alloc(&t.b_area, nn)) ||
        (r = h->alloc(&t.s_nodes, nn)) || (r = h->alloc(&t.s_q, nn)) || (r = h->alloc(&t.s_fac, nn)) || (r = h->alloc(&h->cnt_s, ns)) || (r = h->alloc(&h->off_s, ns)) ||
        (r = h->alloc(&h->cnt_d, ns)) || (r = h->alloc(&h->off_d, ns)) || (r = h->alloc(&h->ksplit, ns)) ||
        (r = h->alloc(&h->node_cnt, nd)) || (r = h->alloc(&h->node_off, nd)) ||
        (r = h->alloc(&h->partials, 2 * scan_partials_words(std::max(c.max_stree_nodes, c.max_dtrees)))) ||
        (r = h->alloc(&h->totals, 4)) || (r = h->alloc(&h->fp, 4))) {
        delete h;
        return r;
    }
    cudaError_t e = cudaFuncSetAttribute(k_reset<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, reset_smem());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_reset<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, reset_smem());
    if (e != cudaSuccess) {
        delete h;
        return fail(RTPG_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    }
    if ((r = sdtree_clear(h, 0))) {
        delete h;
        return r;
    }
    e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        delete h;
        return fail(RTPG_ECUDA, "rtpg_sdtree_create: %s", cudaGetErrorString(e));
    }
    *out = h;
    return RTPG_OK;
}

int rtpg_sdtree_destroy(rtpg_sdtree* h) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_destroy: null handle");
    delete h;
    return RTPG_OK;
}

int rtpg_sdtree_clear(rtpg_sdtree* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_clear: null handle");
    return sdtree_clear(h, as_stream(stream));
}

int rtpg_sdtree_record(rtpg_sdtree* h, int64_t n, const float* pos, const float* dir, int dir_is_canonical,
                       const float* radiance, const float* wo_pdf, const float* stat_weight, const uint8_t* is_delta,
                       void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_record: null handle");
    if (n < 0) return fail(RTPG_EINVAL, "rtpg_sdtree_record: n < 0");
    if (n == 0) return RTPG_OK;
    if (!pos || !dir || !radiance) return fail(RTPG_EINVAL, "rtpg_sdtree_record: pos, dir and radiance are required");
    if ((dir_is_canonical && !aligned8(dir)) || !aligned4(pos) || !aligned4(radiance))
        return fail(RTPG_EINVAL, "rtpg_sdtree_record: misaligned array (float2 arrays need 8-byte alignment)");
    // one resident wave: 6 CTAs of 256 per SM (36 KB of static shared memory each)
    const int g = grid_for(n, kRecordBlock, 6);
    if (dir_is_canonical)
        k_record<true><<<g, kRecordBlock, 0, as_stream(stream)>>>(h->dev, n, pos, dir, radiance, wo_pdf, stat_weight, is_delta);
    else
        k_record<false><<<g, kRecordBlock, 0, as_stream(stream)>>>(h->dev, n, pos, dir, radiance, wo_pdf, stat_weight, is_delta);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_sdtree_build(rtpg_sdtree* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_build: null handle");
    RTPG_CUDA(launch_dependent(k_build, kSMs * 4, kTreeBlock, 0, as_stream(stream), h->dev));
    return RTPG_OK;
}

int rtpg_sdtree_refine(rtpg_sdtree* h, uint64_t spatial_threshold, int32_t max_mb, float dtree_subdiv_th, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_refine: null handle");
    cudaStream_t st = as_stream(stream);
    SDTreeDev& t = h->dev;
    // spatial part; fp[0] footprint, fp[1..2] new STree nodes / DTrees, fp[3] quadtree nodes
    // every kernel of the refine is a dependent launch (it waits for its predecessor in-kernel)
    RTPG_CUDA(launch_dependent(k_zero_u64, 1, 32, 0, st, h->fp, 4));
    if (max_mb >= 0) RTPG_CUDA(launch_dependent(k_footprint, kSMs * 2, 256, 0, st, t, h->fp));
    const float thf = (float)spatial_threshold;  // the size_t threshold as the float compare sees it
    uint32_t kmax = 0;
    while (kmax < 24 && (2ull << (kmax + 1)) <= t.cap_snodes) ++kmax;
    RTPG_CUDA(launch_dependent(k_refine_count, grid_for(t.cap_snodes, 256, 8), 256, 0, st, t, thf, max_mb, kmax, h->fp,
                               h->cnt_s, h->cnt_d, h->ksplit));
    int r;
    // new STree nodes and new DTrees per leaf: one pass over both count arrays
    if ((r = scan_exclusive_u32x2(h->cnt_s, h->off_s, h->totals + 0, h->cnt_d, h->off_d, h->totals + 1, t.counts + 0,
                                  t.cap_snodes, h->partials, st)))
        return r;
    RTPG_CUDA(launch_dependent(k_refine_apply, kSMs * 4, 256, 0, st, t, h->ksplit, h->off_s, h->cnt_s, h->off_d,
                               h->cnt_d, h->fp));
    RTPG_CUDA(launch_dependent(k_refine_link, grid_for(t.cap_snodes, 256, 4), 256, 0, st, t, h->ksplit, h->off_s, h->fp));
    RTPG_CUDA(launch_dependent(k_refine_commit, 1, 1, 0, st, t, h->fp));
    RTPG_CUDA(launch_dependent(k_stree_top, 1, kTopCells, 0, st, t));
    // quadtree reset of every leaf
    RTPG_CUDA(launch_dependent(k_reset<false>, kSMs, kTreeBlock, reset_smem(), st, t, dtree_subdiv_th, h->node_cnt,
                               (const uint32_t*)nullptr, h->fp + 3));
    if ((r = scan_exclusive_u32(h->node_cnt, h->node_off, t.counts + 1, t.cap_dtrees, h->partials, h->totals + 2, st)))
        return r;
    RTPG_CUDA(launch_dependent(k_reset<true>, kSMs, kTreeBlock, reset_smem(), st, t, dtree_subdiv_th, (uint32_t*)nullptr,
                               (const uint32_t*)h->node_off, h->fp + 3));
    RTPG_CUDA(launch_dependent(k_reset_commit, 1, 1, 0, st, t, (const unsigned long long*)(h->fp + 3)));
    return RTPG_OK;
}

int rtpg_sdtree_reset(rtpg_sdtree* h, int32_t iteration, int32_t samples_per_pass, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_reset: null handle");
    if (iteration <= 0) return RTPG_OK;
    // size_t sTreeTh = std::sqrt(std::pow(2.0, iter) * samplePerPasses / 4.0f) * 4000 (PG.h:1649)
    const uint64_t th = (uint64_t)(std::sqrt(std::pow(2.0, iteration) * samples_per_pass / 4.0f) * 4000);
    return rtpg_sdtree_refine(h, th, 2000, 0.01f, stream);
}

int rtpg_sdtree_sample_pdf(rtpg_sdtree* h, int64_t n, const float* pos, const uint32_t* seeds, uint32_t seed_base,
                           float* out_uv, float* out_pdf_uv, float* out_dir, float* out_pdf_dir, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_sample_pdf: null handle");
    if (n < 0 || (n > 0 && !pos)) return fail(RTPG_EINVAL, "rtpg_sdtree_sample_pdf: bad arguments");
    if (!aligned8(out_uv) || !aligned4(pos)) return fail(RTPG_EINVAL, "rtpg_sdtree_sample_pdf: misaligned array");
    if (n == 0) return RTPG_OK;
    // one resident wave: 8 CTAs of 256 per SM (32 registers a thread)
    if (n <= kMaxIndex32)
        k_sample_pdf<int32_t><<<grid_for(n, kSampleBlock, 8), kSampleBlock, 0, as_stream(stream)>>>(
            h->dev, (int32_t)n, pos, seeds, seed_base, out_uv, out_pdf_uv, out_dir, out_pdf_dir);
    else
        k_sample_pdf<int64_t><<<grid_for(n, kSampleBlock, 8), kSampleBlock, 0, as_stream(stream)>>>(
            h->dev, n, pos, seeds, seed_base, out_uv, out_pdf_uv, out_dir, out_pdf_dir);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_sdtree_pdf(rtpg_sdtree* h, int64_t n, const float* pos, const float* dir, int dir_is_canonical,
                    float* out_pdf, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_pdf: null handle");
    if (n < 0 || (n > 0 && (!pos || !dir || !out_pdf))) return fail(RTPG_EINVAL, "rtpg_sdtree_pdf: bad arguments");
    if ((dir_is_canonical && !aligned8(dir)) || !aligned4(pos)) return fail(RTPG_EINVAL, "rtpg_sdtree_pdf: misaligned array");
    if (n == 0) return RTPG_OK;
    k_pdf<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(h->dev, n, pos, dir, dir_is_canonical, out_pdf);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_sdtree_stats(rtpg_sdtree* h, uint32_t* stree_nodes, uint32_t* dtrees, uint32_t* dtree_nodes, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_sdtree_stats: null handle");
    uint32_t c[4];
    RTPG_CUDA(cudaMemcpyAsync(c, h->dev.counts, sizeof(c), cudaMemcpyDeviceToHost, as_stream(stream)));
    RTPG_CUDA(cudaStreamSynchronize(as_stream(stream)));
    if (stree_nodes) *stree_nodes = c[0];
    if (dtrees) *dtrees = c[1];
    if (dtree_nodes) *dtree_nodes = c[2];
    return RTPG_OK;
}

int rtpg_sdtree_memory_footprint(rtpg_sdtree* h, uint64_t* bytes) {
    if (!h || !bytes) return fail(RTPG_EINVAL, "rtpg_sdtree_memory_footprint: null argument");
    *bytes = h->bytes;
    return RTPG_OK;
}

int rtpg_sdtree_status(rtpg_sdtree* h, uint32_t* status, int clear, void* stream) {
    if (!h || !status) return fail(RTPG_EINVAL, "rtpg_sdtree_status: null argument");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemcpyAsync(status, h->dev.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    if (clear) RTPG_CUDA(cudaMemsetAsync(h->dev.status, 0, sizeof(uint32_t), st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ export (host side)
namespace {
struct HostTree {
    std::vector<uint32_t> snode, b_off, b_cnt, s_off, s_cnt;
    std::vector<unsigned long long> b_statw, b_sums;
    std::vector<float> s_sum, s_area, s_statw;
    std::vector<ushort4> b_child;
    std::vector<SNode> s_nodes;
    float inv_scale;
};
struct ExportOut {
    std::vector<uint8_t> smask, dmask;
    std::vector<float> scalars, dsums;
    std::vector<int64_t> counts;
};
void exp_dtree(const HostTree& h, bool sampling, uint32_t off, uint32_t n, ExportOut& e) {
    uint32_t c[4];
    float s[4];
    if (sampling) {
        const SNode& nd = h.s_nodes[off + n];
        c[0] = nd.child.x; c[1] = nd.child.y; c[2] = nd.child.z; c[3] = nd.child.w;
        s[0] = nd.sums.x; s[1] = nd.sums.y; s[2] = nd.sums.z; s[3] = nd.sums.w;
    } else {
        const ushort4 ch = h.b_child[off + n];
        c[0] = ch.x; c[1] = ch.y; c[2] = ch.z; c[3] = ch.w;
        for (int q = 0; q < 4; ++q) s[q] = (float)(long long)h.b_sums[size_t(off + n) * 4 + q] * h.inv_scale;
    }
    uint8_t m = 0;
    for (int q = 0; q < 4; ++q)
        if (c[q]) m |= uint8_t(1u << q);
    e.dmask.push_back(m);
    for (int q = 0; q < 4; ++q) e.dsums.push_back(s[q]);
    for (int q = 0; q < 4; ++q)
        if (c[q]) exp_dtree(h, sampling, off, c[q], e);
}
void exp_stree(const HostTree& h, bool sampling, uint32_t i, ExportOut& e) {
    const uint32_t code = h.snode[i];
    const bool leaf = (code & kLeafBit) != 0;
    e.smask.push_back(leaf ? 0 : 1);
    if (leaf) {
        const uint32_t d = code & ~kLeafBit;
        e.scalars.push_back((float)(long long)h.b_statw[d] * h.inv_scale);
        e.scalars.push_back(h.s_sum[d]);
        e.scalars.push_back(h.s_area[d]);
        e.scalars.push_back(h.s_statw[d]);
        const size_t before = e.dmask.size();
        exp_dtree(h, sampling, sampling ? h.s_off[d] : h.b_off[d], 0, e);
        e.counts.push_back(int64_t(e.dmask.size() - before));
        return;
    }
    exp_stree(h, sampling, code, e);
    exp_stree(h, sampling, code + 1, e);
}
template <class T>
cudaError_t dl(std::vector<T>& v, const T* p, size_t n, cudaStream_t st) {
    v.resize(n);
    if (!n) return cudaSuccess;
    return cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, st);
}
}  // namespace

extern "C" int rtpg_sdtree_export(rtpg_sdtree* h, int sampling, int64_t* sizes, uint8_t* smask, float* scalars,
                                  int64_t* counts, uint8_t* dmask, float* dsums, void* stream) {
    if (!h || !sizes) return fail(RTPG_EINVAL, "rtpg_sdtree_export: null argument");
    cudaStream_t st = as_stream(stream);
    uint32_t c[4];
    RTPG_CUDA(cudaMemcpyAsync(c, h->dev.counts, sizeof(c), cudaMemcpyDeviceToHost, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    HostTree ht;
    const SDTreeDev& t = h->dev;
    ht.inv_scale = t.fx.inv_scale;
    const uint32_t ns = c[0], nd = c[1];
    RTPG_CUDA(dl(ht.snode, t.snode, ns, st));
    RTPG_CUDA(dl(ht.b_off, t.b_off, nd, st));
    RTPG_CUDA(dl(ht.b_cnt, t.b_cnt, nd, st));
    RTPG_CUDA(dl(ht.s_off, t.s_off, nd, st));
    RTPG_CUDA(dl(ht.s_cnt, t.s_cnt, nd, st));
    RTPG_CUDA(dl(ht.b_statw, t.b_statw, nd, st));
    RTPG_CUDA(dl(ht.s_sum, t.s_sum, nd, st));
    RTPG_CUDA(dl(ht.s_area, t.s_area, nd, st));
    RTPG_CUDA(dl(ht.s_statw, t.s_statw, nd, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    uint32_t bmax = 0, smax = 0;
    for (uint32_t d = 0; d < nd; ++d) {
        bmax = std::max(bmax, ht.b_off[d] + ht.b_cnt[d]);
        smax = std::max(smax, ht.s_off[d] + ht.s_cnt[d]);
    }
    RTPG_CUDA(dl(ht.b_child, t.b_child, bmax, st));
    RTPG_CUDA(dl(ht.b_sums, t.b_sums, size_t(bmax) * 4, st));
    RTPG_CUDA(dl(ht.s_nodes, t.s_nodes, smax, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    ExportOut e;
    exp_stree(ht, sampling != 0, 0, e);
    sizes[0] = (int64_t)e.smask.size();
    sizes[1] = (int64_t)e.counts.size();
    sizes[2] = (int64_t)e.dmask.size();
    if (smask) memcpy(smask, e.smask.data(), e.smask.size());
    if (scalars) memcpy(scalars, e.scalars.data(), e.scalars.size() * sizeof(float));
    if (counts) memcpy(counts, e.counts.data(), e.counts.size() * sizeof(int64_t));
    if (dmask) memcpy(dmask, e.dmask.data(), e.dmask.size());
    if (dsums) memcpy(dsums, e.dsums.data(), e.dsums.size() * sizeof(float));
    return RTPG_OK;
}

// ------------------------------------------------------------------ import (host side)
// The inverse of the export: the pre-order streams of the STree and of every leaf's building
// and sampling quadtree are laid out as the kernels expect them -- STree children adjacent
// (child 1 = child 0 + 1), quadtrees breadth first with their level starts, building sums in
// fixed point, sampling nodes as float.  RTLib's counterpart is RTSTreeWrapperT::Upload
// (OPX7UtilsPathGuiding.h:1353-1564), which flattens the host trees into device buffers.
namespace {
struct QNode {
    uint8_t mask;
    float sums[4];
    uint32_t child[4];  // index into the parsed node list (valid where mask has the bit)
};
// Parses one quadtree of `count` pre-order nodes starting at stream position `pos`.
bool parse_dtree(const uint8_t* mask, const float* sums, int64_t total, int64_t pos, int64_t count,
                 std::vector<QNode>& out, std::string& err) {
    out.clear();
    if (count < 1 || pos < 0 || pos + count > total) {
        err = "quadtree node range outside the stream";
        return false;
    }
    // explicit stack of (node, next quadrant to visit)
    std::vector<std::pair<uint32_t, int>> stack;
    int64_t k = pos;
    auto take = [&](uint32_t& idx) -> bool {
        if (k >= pos + count) return false;
        QNode n{};
        n.mask = mask[k];
        if (n.mask & ~0xFu) return false;
        for (int q = 0; q < 4; ++q) n.sums[q] = sums[4 * k + q];
        idx = (uint32_t)out.size();
        out.push_back(n);
        ++k;
        return true;
    };
    uint32_t root;
    if (!take(root)) {
        err = "empty quadtree";
        return false;
    }
    stack.push_back({root, 0});
    while (!stack.empty()) {
        auto& top = stack.back();
        if (top.second >= 4) {
            stack.pop_back();
            continue;
        }
        const int q = top.second++;
        if (!(out[top.first].mask & (1u << q))) continue;
        uint32_t c;
        if (!take(c)) {
            err = "quadtree stream ends inside a tree";
            return false;
        }
        out[stack.back().first].child[q] = c;
        if (stack.size() > kMaxDTreeDepth + 1) {
            err = "quadtree deeper than the supported maximum";
            return false;
        }
        stack.push_back({c, 0});
    }
    if (k != pos + count) {
        err = "quadtree node count does not match its stream";
        return false;
    }
    return true;
}
// Breadth-first numbering of a parsed quadtree: order[j] = parsed index of node j, level
// starts (one entry per level plus the end).
void bfs_dtree(const std::vector<QNode>& t, std::vector<uint32_t>& order, std::vector<uint32_t>& lvl) {
    order.assign(1, 0u);
    lvl.assign(1, 0u);
    size_t a = 0;
    while (a < order.size()) {
        const size_t b = order.size();
        lvl.push_back((uint32_t)b);
        for (size_t j = a; j < b; ++j)
            for (int q = 0; q < 4; ++q)
                if (t[order[j]].mask & (1u << q)) order.push_back(t[order[j]].child[q]);
        a = b;
    }
    // lvl holds the start of every level and, last, the node count (its final level is empty)
    if (lvl.size() >= 2 && lvl[lvl.size() - 1] == lvl[lvl.size() - 2]) lvl.pop_back();
}
template <class T>
cudaError_t ul(T* dst, const std::vector<T>& v, cudaStream_t st) {
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}
}  // namespace

extern "C" int rtpg_sdtree_import(rtpg_sdtree* h, int64_t stree_nodes, int64_t leaves, const uint8_t* stree_mask,
                                  const float* leaf_scalars, int64_t building_nodes, const int64_t* building_counts,
                                  const uint8_t* building_mask, const float* building_sums, int64_t sampling_nodes,
                                  const int64_t* sampling_counts, const uint8_t* sampling_mask,
                                  const float* sampling_sums, void* stream) {
    if (!h || !stree_mask || !leaf_scalars || !building_counts || !building_mask || !building_sums ||
        !sampling_counts || !sampling_mask || !sampling_sums)
        return fail(RTPG_EINVAL, "rtpg_sdtree_import: null argument");
    SDTreeDev& t = h->dev;
    if (stree_nodes < 1 || leaves < 1 || stree_nodes != 2 * leaves - 1)
        return fail(RTPG_EINVAL, "rtpg_sdtree_import: %lld STree nodes cannot hold %lld leaves", (long long)stree_nodes,
                    (long long)leaves);
    if (stree_nodes > (int64_t)t.cap_snodes || leaves > (int64_t)t.cap_dtrees)
        return fail(RTPG_ECAPACITY, "rtpg_sdtree_import: %lld STree nodes / %lld leaves exceed the capacities %u / %u",
                    (long long)stree_nodes, (long long)leaves, t.cap_snodes, t.cap_dtrees);
    if (building_nodes > (int64_t)t.cap_nodes || sampling_nodes > (int64_t)t.cap_nodes)
        return fail(RTPG_ECAPACITY, "rtpg_sdtree_import: quadtree nodes exceed the pool capacity %u", t.cap_nodes);
    // STree: pre-order mask -> adjacent-children layout, breadth first; leaves keep their
    // pre-order rank as DTree index (the order of the scalars and counts)
    struct SN { int64_t c0 = -1, c1 = -1; int64_t leaf = -1; };
    std::vector<SN> sn;
    sn.reserve((size_t)stree_nodes);
    {
        std::vector<std::pair<int64_t, int>> stack;  // (node, children attached)
        int64_t k = 0, leaf = 0;
        auto take = [&]() -> int64_t {
            const uint8_t m = stree_mask[k++];
            SN n;
            if (m == 0) n.leaf = leaf++;
            else if (m != 1) return -2;
            sn.push_back(n);
            return (int64_t)sn.size() - 1;
        };
        const int64_t root = take();
        if (root < 0) return fail(RTPG_EINVAL, "rtpg_sdtree_import: STree mask values must be 0 or 1");
        if (sn[root].leaf < 0) stack.push_back({root, 0});
        while (!stack.empty()) {
            auto& top = stack.back();
            if (top.second == 2) {
                stack.pop_back();
                continue;
            }
            if (k >= stree_nodes) return fail(RTPG_EINVAL, "rtpg_sdtree_import: STree stream ends inside the tree");
            const int which = top.second++;
            const int64_t parent = top.first;
            const int64_t c = take();
            if (c < 0) return fail(RTPG_EINVAL, "rtpg_sdtree_import: STree mask values must be 0 or 1");
            (which == 0 ? sn[parent].c0 : sn[parent].c1) = c;
            if (sn[c].leaf < 0) stack.push_back({c, 0});
        }
        if (k != stree_nodes || leaf != leaves)
            return fail(RTPG_EINVAL, "rtpg_sdtree_import: STree stream does not match its sizes");
    }
    std::vector<uint32_t> snode((size_t)stree_nodes);
    {
        std::vector<int64_t> order(1, 0);  // breadth-first: order[i] = parsed node of device node i
        for (size_t i = 0; i < order.size(); ++i) {
            const SN& n = sn[order[i]];
            if (n.leaf >= 0) {
                snode[i] = kLeafBit | (uint32_t)n.leaf;
            } else {
                snode[i] = (uint32_t)order.size();
                order.push_back(n.c0);
                order.push_back(n.c1);
            }
        }
    }
    // quadtrees
    const size_t L = (size_t)leaves;
    std::vector<uint32_t> b_off(L), b_cnt(L), s_off(L), s_cnt(L);
    std::vector<unsigned long long> b_statw(L);
    std::vector<float> s_sum(L), s_area(L), s_statw(L);
    std::vector<uint8_t> s_guided(L), b_nlvl(L);
    std::vector<uint16_t> b_lvl(L * (kMaxLevels + 1), 0);
    std::vector<unsigned long long> b_sums;
    std::vector<ushort4> b_child;
    std::vector<SNode> s_nodes;
    std::vector<SQNode> s_q;
    std::vector<float4> s_fac;
    const float scale = t.fx.scale;
    auto fx = [&](float v, unsigned long long& out) -> bool {
        const float s = v * scale;
        if (!std::isfinite(s) || std::fabs(s) >= 9.2233720368547758e18f) return false;
        out = (unsigned long long)std::llrint(s);
        return true;
    };
    std::vector<QNode> q;
    std::vector<uint32_t> order, lvl;
    std::string err;
    int64_t bpos = 0, spos = 0;
    for (size_t d = 0; d < L; ++d) {
        const float* sc = leaf_scalars + 4 * d;
        if (!fx(sc[0], b_statw[d])) return fail(RTPG_EINVAL, "rtpg_sdtree_import: leaf %zu stat-weight not representable", d);
        s_sum[d] = sc[1];
        s_area[d] = sc[2];
        s_statw[d] = sc[3];
        // DTreeT::GetMean() > 0 (PG.h:447-451), as the build sets it
        s_guided[d] = (sc[3] > 0.0f && (float)(kInv2Pi / (2.0f * sc[3])) * sc[1] > 0.0f) ? 1 : 0;
        // building tree
        if (!parse_dtree(building_mask, building_sums, building_nodes, bpos, building_counts[d], q, err))
            return fail(RTPG_EINVAL, "rtpg_sdtree_import: building tree of leaf %zu: %s", d, err.c_str());
        bpos += building_counts[d];
        bfs_dtree(q, order, lvl);
        if (order.size() > kDTreeNodeCap || lvl.size() - 1 > kMaxLevels)
            return fail(RTPG_ECAPACITY, "rtpg_sdtree_import: building tree of leaf %zu exceeds %u nodes or %u levels", d,
                        kDTreeNodeCap, kMaxLevels);
        std::vector<uint32_t> rank(q.size());
        for (size_t j = 0; j < order.size(); ++j) rank[order[j]] = (uint32_t)j;
        b_off[d] = (uint32_t)b_child.size();
        b_cnt[d] = (uint32_t)order.size();
        b_nlvl[d] = (uint8_t)(lvl.size() - 1);
        for (size_t l = 0; l < lvl.size(); ++l) b_lvl[d * (kMaxLevels + 1) + l] = (uint16_t)lvl[l];
        for (uint32_t j : order) {
            const QNode& n = q[j];
            uint16_t c[4];
            for (int k = 0; k < 4; ++k) {
                c[k] = (n.mask & (1u << k)) ? (uint16_t)rank[n.child[k]] : (uint16_t)0;
                unsigned long long v;
                if (!fx(n.sums[k], v))
                    return fail(RTPG_EINVAL, "rtpg_sdtree_import: building sum of leaf %zu not representable", d);
                b_sums.push_back(v);
            }
            b_child.push_back(make_ushort4(c[0], c[1], c[2], c[3]));
        }
        // sampling tree
        if (!parse_dtree(sampling_mask, sampling_sums, sampling_nodes, spos, sampling_counts[d], q, err))
            return fail(RTPG_EINVAL, "rtpg_sdtree_import: sampling tree of leaf %zu: %s", d, err.c_str());
        spos += sampling_counts[d];
        bfs_dtree(q, order, lvl);
        if (order.size() > kDTreeNodeCap)
            return fail(RTPG_ECAPACITY, "rtpg_sdtree_import: sampling tree of leaf %zu exceeds %u nodes", d, kDTreeNodeCap);
        rank.assign(q.size(), 0);
        for (size_t j = 0; j < order.size(); ++j) rank[order[j]] = (uint32_t)j;
        s_off[d] = (uint32_t)s_nodes.size();
        s_cnt[d] = (uint32_t)order.size();
        for (uint32_t j : order) {
            const QNode& n = q[j];
            SNode nd;
            nd.sums = make_float4(n.sums[0], n.sums[1], n.sums[2], n.sums[3]);
            uint16_t c[4];
            for (int k = 0; k < 4; ++k) c[k] = (n.mask & (1u << k)) ? (uint16_t)rank[n.child[k]] : (uint16_t)0;
            nd.child = make_ushort4(c[0], c[1], c[2], c[3]);
            nd.pad0 = nd.pad1 = 0;
            s_nodes.push_back(nd);
            float4 fac;
            s_q.push_back(make_sqnode(nd.sums, nd.child, fac));
            s_fac.push_back(fac);
        }
    }
    if (bpos != building_nodes || spos != sampling_nodes)
        return fail(RTPG_EINVAL, "rtpg_sdtree_import: quadtree streams hold nodes beyond the leaves' counts");
    if (b_child.size() > t.cap_nodes || s_nodes.size() > t.cap_nodes)
        return fail(RTPG_ECAPACITY, "rtpg_sdtree_import: quadtree nodes exceed the pool capacity %u", t.cap_nodes);
    cudaStream_t st = as_stream(stream);
    const uint32_t counts[4] = {(uint32_t)stree_nodes, (uint32_t)leaves, (uint32_t)b_child.size(),
                                (uint32_t)s_nodes.size()};
    RTPG_CUDA(cudaMemcpyAsync(t.counts, counts, sizeof(counts), cudaMemcpyHostToDevice, st));
    RTPG_CUDA(ul(t.snode, snode, st));
    RTPG_CUDA(ul(t.b_off, b_off, st));
    RTPG_CUDA(ul(t.b_cnt, b_cnt, st));
    RTPG_CUDA(ul(t.s_off, s_off, st));
    RTPG_CUDA(ul(t.s_cnt, s_cnt, st));
    RTPG_CUDA(ul(t.b_statw, b_statw, st));
    RTPG_CUDA(ul(t.s_sum, s_sum, st));
    RTPG_CUDA(ul(t.s_area, s_area, st));
    RTPG_CUDA(ul(t.s_statw, s_statw, st));
    RTPG_CUDA(ul(t.s_guided, s_guided, st));
    RTPG_CUDA(ul(t.b_lvl, b_lvl, st));
    RTPG_CUDA(ul(t.b_nlvl, b_nlvl, st));
    RTPG_CUDA(ul(t.b_sums, b_sums, st));
    RTPG_CUDA(ul(t.b_child, b_child, st));
    RTPG_CUDA(ul(t.s_nodes, s_nodes, st));
    RTPG_CUDA(ul(t.s_q, s_q, st));
    RTPG_CUDA(ul(t.s_fac, s_fac, st));
    k_stree_top<<<1, kTopCells, 0, st>>>(t);
    RTPG_LAUNCH_CHECK();
    // the host vectors must outlive the copies
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

// ================================================================== pass controller
// RTSTreeControllerT (PG.h:1769-1920), host logic unchanged; the Download/Upload pairs
// around Reset and Build disappear because the tree never leaves the GPU.
struct rtpg_controller {
    rtpg_sdtree* tree;
    uint32_t sample_for_budget, samples_per_launch, iteration_for_built;
    float ratio_for_budget;
    bool start = false, executing = false;
    uint32_t per_all = 0, per_tmp = 0, remain = 0, pass = 0, iteration = 0;
    int32_t state = RTPG_TRACE_RECORD;
};

extern "C" {

int rtpg_controller_create(rtpg_sdtree* tree, uint32_t sample_for_budget, uint32_t iteration_for_built,
                           float ratio_for_budget, uint32_t samples_per_launch, rtpg_controller** out) {
    if (!tree || !out || samples_per_launch == 0) return fail(RTPG_EINVAL, "rtpg_controller_create: bad arguments");
    auto* c = new (std::nothrow) rtpg_controller();
    if (!c) return fail(RTPG_ENOMEM, "rtpg_controller_create: out of host memory");
    c->tree = tree;
    c->sample_for_budget = sample_for_budget;
    c->samples_per_launch = samples_per_launch;
    c->iteration_for_built = iteration_for_built;
    c->ratio_for_budget = ratio_for_budget;
    *out = c;
    return RTPG_OK;
}
int rtpg_controller_destroy(rtpg_controller* c) {
    delete c;
    return RTPG_OK;
}
int rtpg_controller_start(rtpg_controller* c) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_controller_start: null handle");
    c->start = true;  // RTSTreeControllerT::Start, PG.h:1804-1806
    return RTPG_OK;
}
// RTSTreeControllerT::BegTrace (PG.h:1808-1865)
int rtpg_controller_begin(rtpg_controller* c, void* stream) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_controller_begin: null handle");
    int r;
    if (c->start) {
        c->per_all = 0;
        c->per_tmp = 0;
        c->iteration = 0;
        c->start = false;
        c->executing = true;
        c->remain = ((c->sample_for_budget - 1 + c->samples_per_launch) / c->samples_per_launch) * c->samples_per_launch;
        c->pass = 0;
        c->state = RTPG_TRACE_RECORD;
        if ((r = rtpg_sdtree_clear(c->tree, stream))) return r;
    }
    if (!c->executing) return RTPG_OK;
    if (c->per_tmp == 0) {
        c->remain -= c->pass;
        c->pass = std::min<uint32_t>(c->remain, (1u << c->iteration) * c->samples_per_launch);
        if ((c->remain - c->pass < 2 * c->pass) ||
            (c->per_all >= c->ratio_for_budget * static_cast<float>(c->sample_for_budget)))
            c->pass = c->remain;
        if (c->remain > c->pass)
            if ((r = rtpg_sdtree_reset(c->tree, (int32_t)c->iteration, (int32_t)c->pass, stream))) return r;
    }
    if (c->iteration > c->iteration_for_built)
        c->state = c->remain > c->pass ? RTPG_TRACE_RECORD_AND_SAMPLE : RTPG_TRACE_SAMPLE;
    else
        c->state = RTPG_TRACE_RECORD;
    return RTPG_OK;
}
// RTSTreeControllerT::EndTrace (PG.h:1867-1887)
int rtpg_controller_end(rtpg_controller* c, void* stream) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_controller_end: null handle");
    if (!c->executing) return RTPG_OK;
    c->per_all += c->samples_per_launch;
    c->per_tmp += c->samples_per_launch;
    if (c->per_tmp >= c->pass) {
        int r = rtpg_sdtree_build(c->tree, stream);
        if (r) return r;
        c->iteration++;
        c->per_tmp = 0;
    }
    if (c->per_all > c->sample_for_budget) {
        c->executing = false;
        c->per_all = 0;
    }
    return RTPG_OK;
}
int rtpg_controller_get(rtpg_controller* c, int32_t* state, uint32_t* iteration, uint32_t* samples_in_pass,
                        int32_t* executing) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_controller_get: null handle");
    if (state) *state = c->state;
    if (iteration) *iteration = c->iteration;
    if (samples_in_pass) *samples_in_pass = c->per_tmp;
    if (executing) *executing = c->executing ? 1 : 0;
    return RTPG_OK;
}

}  // extern "C"
