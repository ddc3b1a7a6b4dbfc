// Morton-indexed directional quadtrees, one complete tree per hash-grid cell (RTLib's "HashTree"
// guide: MortonQuadTreeT / MortonQuadTreeWrapperT, OPX7UtilsMorton.h:253-531, host wrapper
// RTMortonQuadTreeWrapperT :590-764, pyramid build mortonBuildKernel,
// OPX7UtilsMortonBuild.cu:2-16).
//
// Layout in HBM: building leaves, int64 fixed point, cell-major: leaves[cell * 4^L + code]
// (the reference records only the leaf level too, OPX7UtilsMorton.h:282-283); sampling
// pyramid, float, per cell (4^(L+1)-1)/3 entries, level l at offset (4^l-1)/3, Morton order
// inside a level (code = part1by1(y) << 1 | part1by1(x)).
//
// Update (RTMortonQuadTreeWrapperT::Update + LaunchBuildKernel, :640-651, :916-941) is one
// kernel: a warp (levels up to 5) or a CTA (levels 6, 7) per cell reads the cell's leaves,
// reduces the pyramid in shared memory with exact integer sums, writes it as float to the
// sampling buffer and zeroes the leaves (RTLib launches 1024x more blocks than cells and loops
// serially per cell).
#include <algorithm>
#include <new>
#include <vector>

#include "common.cuh"
#include "limits.cuh"
#include "mqt_dev.cuh"

namespace rtpg {

constexpr int kMqtBuildBlock = 256;

__global__ void __launch_bounds__(256) k_mqt_record(MqtDev t, int64_t n, const uint32_t* __restrict__ cell,
                                                    const float* __restrict__ dir, int canonical,
                                                    const float* __restrict__ value) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        unsigned long long key = ~0ull, v = 0;
        if (i < n) {
            const uint32_t c = cell[i];
            const float x = value[i];
            if (c != 0xffffffffu && c < t.ncells && isfinite(x) && x > 0.0f) {
                float2 uv;
                if (canonical) uv = reinterpret_cast<const float2*>(dir)[i];
                else uv = dir_to_canonical_mqt(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
                key = ((unsigned long long)c << (2 * t.level)) + mqt_leaf_code(t.level, uv.x, uv.y);
                v = to_fx(x, t.fx, t.status);
            }
        }
        warp_add_u64(key, v, t.leaves);
    }
}

// One CTA per cell: leaves -> exact pyramid in shared memory -> float sampling pyramid.
__global__ void __launch_bounds__(kMqtBuildBlock) k_mqt_build(MqtDev t) {
    extern __shared__ unsigned long long sp[];  // (4^(L+1)-1)/3 entries
    const uint32_t L = t.level;
    const uint32_t nleaf = 1u << (2 * L);
    const uint32_t off_leaf = mqt_level_offset(L);
    const uint32_t per = mqt_level_offset(L + 1);
    for (uint32_t c = blockIdx.x; c < t.ncells; c += gridDim.x) {
        unsigned long long* lf = t.leaves + (size_t)c * nleaf;
        for (uint32_t k = threadIdx.x; k < nleaf; k += blockDim.x) {
            sp[off_leaf + k] = lf[k];
            lf[k] = 0ull;
        }
        __syncthreads();
        for (int l = (int)L - 1; l >= 0; --l) {
            const uint32_t o = mqt_level_offset(l), oc = mqt_level_offset(l + 1), cnt = 1u << (2 * l);
            for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x)
                sp[o + k] = sp[oc + 4 * k] + sp[oc + 4 * k + 1] + sp[oc + 4 * k + 2] + sp[oc + 4 * k + 3];
            __syncthreads();
        }
        float* w = t.pyramid + (size_t)c * per;
        for (uint32_t k = threadIdx.x; k < per; k += blockDim.x) w[k] = fx_to_float(sp[k], t.fx);
        __syncthreads();
    }
}

// Levels 1 and 2 (up to kMqtWarpLevel): one warp per cell, kMqtWarps cells per CTA.  The warp reads the
// cell's leaves with 16-byte loads (and zeroes them with 16-byte stores), reduces the pyramid
// in its own shared memory with exact integer sums and writes it out with consecutive lanes on
// consecutive floats; no block-wide barrier, so every warp of the SM keeps a cell's loads in
// flight.  Same results as k_mqt_build (integer sums do not depend on their order).
constexpr uint32_t kMqtWarpLevel = 2;  // levels 3 to 5 use k_mqt_build_reg
constexpr int kMqtWarps = 8;
__global__ void __launch_bounds__(32 * kMqtWarps) k_mqt_build_warp(MqtDev t) {
    extern __shared__ unsigned long long swarp[];  // kMqtWarps x (4^(L+1)-1)/3 entries
    const uint32_t L = t.level;
    const uint32_t nleaf = 1u << (2 * L);  // >= 4: 16-byte aligned rows of leaves
    const uint32_t off_leaf = mqt_level_offset(L);
    const uint32_t per = mqt_level_offset(L + 1);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned long long* sp = swarp + (size_t)warp * per;
    const uint32_t nw = gridDim.x * kMqtWarps;
    for (uint32_t c = blockIdx.x * kMqtWarps + warp; c < t.ncells; c += nw) {
        ulonglong2* lf = reinterpret_cast<ulonglong2*>(t.leaves + (size_t)c * nleaf);
        for (uint32_t k = lane; k < nleaf / 2; k += 32) {
            const ulonglong2 v = lf[k];
            lf[k] = make_ulonglong2(0ull, 0ull);
            sp[off_leaf + 2 * k] = v.x;
            sp[off_leaf + 2 * k + 1] = v.y;
        }
        __syncwarp();
        for (int l = (int)L - 1; l >= 0; --l) {
            const uint32_t o = mqt_level_offset(l), oc = mqt_level_offset(l + 1), cnt = 1u << (2 * l);
            for (uint32_t k = lane; k < cnt; k += 32)
                sp[o + k] = sp[oc + 4 * k] + sp[oc + 4 * k + 1] + sp[oc + 4 * k + 2] + sp[oc + 4 * k + 3];
            __syncwarp();
        }
        float* w = t.pyramid + (size_t)c * per;
        for (uint32_t k = lane; k < per; k += 32) w[k] = fx_to_float(sp[k], t.fx);
        __syncwarp();
    }
}

// Levels 3 to 5: the reduction in registers.  Lane l owns leaves [l P, (l + 1) P) with
// P = 4^L / 32 (2, 8 or 32), loaded and zeroed as 16-byte vectors; the levels whose nodes span
// at most P leaves are summed inside the lane, the three levels above them span 2, 8 and 32
// lanes and come from butterfly shuffles.  The float pyramid is assembled in a per-warp
// shared buffer and stored with consecutive lanes on consecutive floats.
template <int L>
__global__ void __launch_bounds__(32 * kMqtWarps) k_mqt_build_reg(MqtDev t) {
    constexpr int NLEAF = 1 << (2 * L), P = NLEAF / 32, PER = ((1 << (2 * (L + 1))) - 1) / 3;
    static_assert(L >= 3 && L <= 5, "levels 3..5");
    __shared__ float sbuf[kMqtWarps][PER];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    float* fb = sbuf[warp];
    const uint32_t nw = gridDim.x * kMqtWarps;
    for (uint32_t c = blockIdx.x * kMqtWarps + warp; c < t.ncells; c += nw) {
        ulonglong2* lf = reinterpret_cast<ulonglong2*>(t.leaves + (size_t)c * NLEAF) + lane * (P / 2);
        unsigned long long v[P];
#pragma unroll
        for (int j = 0; j < P / 2; ++j) {
            const ulonglong2 x = lf[j];
            v[2 * j] = x.x;
            v[2 * j + 1] = x.y;
        }
#pragma unroll
        for (int j = 0; j < P / 2; ++j) lf[j] = make_ulonglong2(0ull, 0ull);
        // the leaf level, then the lane-local levels (each a quarter of the one below)
#pragma unroll
        for (int j = 0; j < P; ++j) fb[mqt_level_offset(L) + lane * P + j] = fx_to_float(v[j], t.fx);
        int lvl = L - 1;
        int n = P;  // values of the current level held by this lane
#pragma unroll
        for (int step = 0; step < 3 && n >= 4; ++step) {
#pragma unroll
            for (int j = 0; j < n / 4; ++j) v[j] = v[4 * j] + v[4 * j + 1] + v[4 * j + 2] + v[4 * j + 3];
            n /= 4;
#pragma unroll
            for (int j = 0; j < n; ++j) fb[mqt_level_offset(lvl) + lane * n + j] = fx_to_float(v[j], t.fx);
            --lvl;
        }
        // two values are left in every lane: their sum is the lane's run
        unsigned long long s = 0;
#pragma unroll
        for (int j = 0; j < n; ++j) s += v[j];
        // nodes spanning 2, 8 and 32 lanes
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        if ((lane & 1u) == 0) fb[mqt_level_offset(lvl) + (lane >> 1)] = fx_to_float(s, t.fx);
        --lvl;
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        if ((lane & 7u) == 0) fb[mqt_level_offset(lvl) + (lane >> 3)] = fx_to_float(s, t.fx);
        --lvl;
        s += __shfl_xor_sync(0xffffffffu, s, 8);
        s += __shfl_xor_sync(0xffffffffu, s, 16);
        if (lane == 0) fb[0] = fx_to_float(s, t.fx);
        __syncwarp();
        float* w = t.pyramid + (size_t)c * PER;
        for (uint32_t k = lane; k < (uint32_t)PER; k += 32) w[k] = fb[k];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(256) k_mqt_sample(MqtDev t, int64_t n, const uint32_t* __restrict__ cell,
                                                    const uint32_t* __restrict__ seeds, uint32_t seed_base,
                                                    float* __restrict__ out_uv, float* __restrict__ out_pdf,
                                                    float* __restrict__ out_dir, float* __restrict__ out_pdf_tree) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t c = cell[i];
        uint32_t rng = seeds ? seeds[i] : (pcg1d(seed_base + (uint32_t)i) | 1u);
        float pdf;
        const float2 uv = mqt_sample_and_pdf(t, c, rng, pdf);
        if (out_uv) reinterpret_cast<float2*>(out_uv)[i] = uv;
        if (out_pdf_tree) out_pdf_tree[i] = pdf;
        // MortonQuadTreeWrapperT::SampleAndPdf (OPX7UtilsMorton.h:486-500):
        // pdf *= (0.25f * RTLIB_M_INV_PI), evaluated in double as written
        if (out_pdf) out_pdf[i] = (float)((double)pdf * (0.25 * kInvPiD));
        if (out_dir) {
            const float3 d = canonical_to_dir_mqt(uv.x, uv.y);
            out_dir[3 * i] = d.x;
            out_dir[3 * i + 1] = d.y;
            out_dir[3 * i + 2] = d.z;
        }
    }
}

__global__ void __launch_bounds__(256) k_mqt_pdf(MqtDev t, int64_t n, const uint32_t* __restrict__ cell,
                                                 const float* __restrict__ dir, int canonical, float* __restrict__ out,
                                                 int tree_level) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        float2 uv;
        if (canonical) uv = reinterpret_cast<const float2*>(dir)[i];
        else uv = dir_to_canonical_mqt(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        const float p = mqt_pdf(t, cell[i], uv.x, uv.y);
        // MortonQuadTreeWrapperT::Pdf (:515-524): tree.Pdf(dir2) * 0.25f * RTLIB_M_INV_PI
        out[i] = tree_level ? p : (float)((double)(p * 0.25f) * kInvPiD);
    }
}

}  // namespace rtpg

using namespace rtpg;

struct rtpg_mqt {
    MqtDev dev{};
    std::vector<void*> allocs;
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
    ~rtpg_mqt() {
        for (void* p : allocs) cudaFree(p);
    }
};

static int mqt_smem(uint32_t level) { return int(mqt_level_offset(level + 1) * sizeof(unsigned long long)); }
static int mqt_smem_warp(uint32_t level) { return kMqtWarps * mqt_smem(level); }

extern "C" {

// RTMortonQuadTreeWrapperT(ctx, maxHashSize, maxTreeLevel, fraction) + Allocate (MO.h:597-638)
int rtpg_mqt_create(uint32_t num_cells, uint32_t level, float fraction, int32_t fixed_point_bits, rtpg_mqt** out) {
    if (!out || num_cells == 0) return fail(RTPG_EINVAL, "rtpg_mqt_create: bad arguments");
    if (level < 1 || level > kMqtMaxLevel) return fail(RTPG_EINVAL, "rtpg_mqt_create: level must be in [1, %u]", kMqtMaxLevel);
    if (fixed_point_bits == 0) fixed_point_bits = 24;
    if (fixed_point_bits < 0 || fixed_point_bits > 40) return fail(RTPG_EINVAL, "rtpg_mqt_create: fixed_point_bits in [0,40]");
    auto* h = new (std::nothrow) rtpg_mqt();
    if (!h) return fail(RTPG_ENOMEM, "rtpg_mqt_create: out of host memory");
    MqtDev& t = h->dev;
    t.ncells = num_cells;
    t.level = level;
    t.fraction = fraction;
    t.fx.scale = ldexpf(1.0f, fixed_point_bits);
    t.fx.inv_scale = ldexpf(1.0f, -fixed_point_bits);
    const size_t nleaf = (size_t)num_cells << (2 * level), npyr = (size_t)num_cells * mqt_level_offset(level + 1);
    int r;
    if ((r = h->alloc(&t.leaves, nleaf)) || (r = h->alloc(&t.pyramid, npyr)) || (r = h->alloc(&t.status, 1))) {
        delete h;
        return r;
    }
    if (cudaMemset(t.leaves, 0, nleaf * 8) != cudaSuccess || cudaMemset(t.pyramid, 0, npyr * 4) != cudaSuccess ||
        cudaMemset(t.status, 0, 4) != cudaSuccess) {
        delete h;
        return fail(RTPG_ECUDA, "rtpg_mqt_create: memset failed");
    }
    cudaError_t e = cudaFuncSetAttribute(k_mqt_build, cudaFuncAttributeMaxDynamicSharedMemorySize, mqt_smem(kMqtMaxLevel));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mqt_build_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, mqt_smem_warp(kMqtWarpLevel));
    if (e != cudaSuccess) {
        delete h;
        return fail(RTPG_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    }
    *out = h;
    return RTPG_OK;
}

int rtpg_mqt_destroy(rtpg_mqt* h) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_destroy: null handle");
    delete h;
    return RTPG_OK;
}

// RTMortonQuadTreeWrapperT::Allocate on an existing wrapper: zero both buffers (MO.h:618-637)
int rtpg_mqt_clear(rtpg_mqt* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_clear: null handle");
    cudaStream_t st = as_stream(stream);
    const MqtDev& t = h->dev;
    RTPG_CUDA(cudaMemsetAsync(t.leaves, 0, ((size_t)t.ncells << (2 * t.level)) * 8, st));
    RTPG_CUDA(cudaMemsetAsync(t.pyramid, 0, (size_t)t.ncells * mqt_level_offset(t.level + 1) * 4, st));
    RTPG_CUDA(cudaMemsetAsync(t.status, 0, 4, st));
    return RTPG_OK;
}

// MortonQuadTreeWrapperT::Record (MO.h:477-484): cell UINT32_MAX is skipped.
int rtpg_mqt_record(rtpg_mqt* h, int64_t n, const uint32_t* cell, const float* dir, int dir_is_canonical,
                    const float* value, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_record: null handle");
    if (n < 0 || (n > 0 && (!cell || !dir || !value))) return fail(RTPG_EINVAL, "rtpg_mqt_record: bad arguments");
    if (dir_is_canonical && !aligned8(dir)) return fail(RTPG_EINVAL, "rtpg_mqt_record: misaligned float2 array");
    if (n == 0) return RTPG_OK;
    k_mqt_record<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(h->dev, n, cell, dir, dir_is_canonical, value);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

// Update + mortonBuildKernel: building leaves -> sampling pyramid, building cleared.
int rtpg_mqt_update(rtpg_mqt* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_update: null handle");
    const int gw = (int)std::min<uint32_t>((h->dev.ncells + kMqtWarps - 1) / kMqtWarps, kSMs * 8);
    if (h->dev.level == 3) {
        k_mqt_build_reg<3><<<gw, 32 * kMqtWarps, 0, as_stream(stream)>>>(h->dev);
    } else if (h->dev.level == 4) {
        k_mqt_build_reg<4><<<gw, 32 * kMqtWarps, 0, as_stream(stream)>>>(h->dev);
    } else if (h->dev.level == 5) {
        k_mqt_build_reg<5><<<gw, 32 * kMqtWarps, 0, as_stream(stream)>>>(h->dev);
    } else if (h->dev.level <= kMqtWarpLevel) {
        k_mqt_build_warp<<<gw, 32 * kMqtWarps, mqt_smem_warp(h->dev.level), as_stream(stream)>>>(h->dev);
    } else {
        const int g = (int)std::min<uint32_t>(h->dev.ncells, kSMs * 8);
        k_mqt_build<<<g, kMqtBuildBlock, mqt_smem(h->dev.level), as_stream(stream)>>>(h->dev);
    }
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

// MortonQuadTreeWrapperT::SampleAndPdf (MO.h:486-500); out_pdf includes the 1/(4 pi) factor,
// out_pdf_tree is MortonQuadTreeT::SampleAndPdf's pdf (MO.h:286-344).
int rtpg_mqt_sample_pdf(rtpg_mqt* h, int64_t n, const uint32_t* cell, const uint32_t* seeds, uint32_t seed_base,
                        float* out_uv, float* out_pdf, float* out_dir, float* out_pdf_tree, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_sample_pdf: null handle");
    if (n < 0 || (n > 0 && !cell)) return fail(RTPG_EINVAL, "rtpg_mqt_sample_pdf: bad arguments");
    if (!aligned8(out_uv)) return fail(RTPG_EINVAL, "rtpg_mqt_sample_pdf: misaligned float2 array");
    if (n == 0) return RTPG_OK;
    k_mqt_sample<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(h->dev, n, cell, seeds, seed_base, out_uv, out_pdf,
                                                                     out_dir, out_pdf_tree);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

// MortonQuadTreeWrapperT::Pdf (MO.h:515-524) or, tree_level = 1, MortonQuadTreeT::Pdf (:401-414).
int rtpg_mqt_pdf(rtpg_mqt* h, int64_t n, const uint32_t* cell, const float* dir, int dir_is_canonical, float* out,
                 int tree_level, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_pdf: null handle");
    if (n < 0 || (n > 0 && (!cell || !dir || !out))) return fail(RTPG_EINVAL, "rtpg_mqt_pdf: bad arguments");
    if (dir_is_canonical && !aligned8(dir)) return fail(RTPG_EINVAL, "rtpg_mqt_pdf: misaligned float2 array");
    if (n == 0) return RTPG_OK;
    k_mqt_pdf<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(h->dev, n, cell, dir, dir_is_canonical, out, tree_level);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_mqt_export(rtpg_mqt* h, int64_t* host_leaves, float* host_pyramid, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mqt_export: null handle");
    cudaStream_t st = as_stream(stream);
    const MqtDev& t = h->dev;
    if (host_leaves)
        RTPG_CUDA(cudaMemcpyAsync(host_leaves, t.leaves, ((size_t)t.ncells << (2 * t.level)) * 8, cudaMemcpyDeviceToHost, st));
    if (host_pyramid)
        RTPG_CUDA(cudaMemcpyAsync(host_pyramid, t.pyramid, (size_t)t.ncells * mqt_level_offset(t.level + 1) * 4,
                                  cudaMemcpyDeviceToHost, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

int rtpg_mqt_status(rtpg_mqt* h, uint32_t* host_status, int clear, void* stream) {
    if (!h || !host_status) return fail(RTPG_EINVAL, "rtpg_mqt_status: null argument");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemcpyAsync(host_status, h->dev.status, 4, cudaMemcpyDeviceToHost, st));
    if (clear) RTPG_CUDA(cudaMemsetAsync(h->dev.status, 0, 4, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

}  // extern "C"

namespace rtpg {
MqtDev mqt_device_view(const rtpg_mqt* h) { return h->dev; }
}

// ================================================================== pass controller
// RTMortonQuadTreeControllerT (OPX7UtilsMorton.h:766-993): the doubling pass schedule of the
// hash-grid guide with a LOCATE phase.  BegTrace at Start clears both quadtree buffers
// (RTMortonQuadTreeWrapperT::Allocate); EndTrace after a finished pass beyond
// iteration_for_built runs Update + mortonBuildKernel (rtpg_mqt_update here).
struct rtpg_mqt_controller {
    rtpg_mqt* tree;
    uint32_t sample_for_budget, samples_per_launch, iteration_for_built, iteration_for_locate;
    float ratio_for_budget;
    bool start = false, executing = false;
    uint32_t per_all = 0, per_tmp = 0, remain = 0, pass = 0, iteration = 0;
    int32_t state = RTPG_MQT_TRACE_RECORD;
};

extern "C" {

int rtpg_mqt_controller_create(rtpg_mqt* tree, uint32_t sample_for_budget, uint32_t iteration_for_built,
                               uint32_t iteration_for_locate, float ratio_for_budget, uint32_t samples_per_launch,
                               rtpg_mqt_controller** out) {
    if (!tree || !out || samples_per_launch == 0) return fail(RTPG_EINVAL, "rtpg_mqt_controller_create: bad arguments");
    auto* c = new (std::nothrow) rtpg_mqt_controller();
    if (!c) return fail(RTPG_ENOMEM, "rtpg_mqt_controller_create: out of host memory");
    c->tree = tree;
    c->sample_for_budget = sample_for_budget;
    c->samples_per_launch = samples_per_launch;
    c->iteration_for_built = iteration_for_built;
    c->iteration_for_locate = iteration_for_locate;
    c->ratio_for_budget = ratio_for_budget;
    *out = c;
    return RTPG_OK;
}
int rtpg_mqt_controller_destroy(rtpg_mqt_controller* c) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_mqt_controller_destroy: null handle");
    delete c;
    return RTPG_OK;
}
int rtpg_mqt_controller_start(rtpg_mqt_controller* c) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_mqt_controller_start: null handle");
    c->start = true;
    return RTPG_OK;
}
// BegTrace (OPX7UtilsMorton.h:818-889)
int rtpg_mqt_controller_begin(rtpg_mqt_controller* c, void* stream) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_mqt_controller_begin: null handle");
    if (c->start) {
        c->per_all = 0;
        c->per_tmp = 0;
        c->iteration = 0;
        c->start = false;
        c->executing = true;
        c->remain = ((c->sample_for_budget - 1 + c->samples_per_launch) / c->samples_per_launch) * c->samples_per_launch;
        c->pass = 0;
        c->state = RTPG_MQT_TRACE_RECORD;
        int r = rtpg_mqt_clear(c->tree, stream);
        if (r) return r;
    }
    if (!c->executing) return RTPG_OK;
    if (c->per_tmp == 0) {
        c->remain -= c->pass;
        c->pass = std::min<uint32_t>(c->remain, (1u << c->iteration) * c->samples_per_launch);
        if ((c->remain - c->pass < 2 * c->pass) ||
            (c->per_all >= c->ratio_for_budget * static_cast<float>(c->sample_for_budget)))
            c->pass = c->remain;
    }
    if (c->iteration > c->iteration_for_built)
        c->state = c->remain > c->pass ? RTPG_MQT_TRACE_RECORD_AND_SAMPLE : RTPG_MQT_TRACE_SAMPLE;
    else if (c->iteration > c->iteration_for_locate)
        c->state = RTPG_MQT_TRACE_RECORD;
    else
        c->state = RTPG_MQT_TRACE_LOCATE;
    return RTPG_OK;
}
// EndTrace (OPX7UtilsMorton.h:891-922)
int rtpg_mqt_controller_end(rtpg_mqt_controller* c, void* stream) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_mqt_controller_end: null handle");
    if (!c->executing) return RTPG_OK;
    c->per_all += c->samples_per_launch;
    c->per_tmp += c->samples_per_launch;
    if (c->per_tmp >= c->pass) {
        c->iteration++;
        if (c->iteration > c->iteration_for_built) {
            int r = rtpg_mqt_update(c->tree, stream);
            if (r) return r;
        }
        c->per_tmp = 0;
    }
    if (c->per_all > c->sample_for_budget) {
        c->executing = false;
        c->per_all = 0;
    }
    return RTPG_OK;
}
int rtpg_mqt_controller_get(rtpg_mqt_controller* c, int32_t* state, uint32_t* iteration, uint32_t* samples_in_pass,
                            int32_t* executing) {
    if (!c) return fail(RTPG_EINVAL, "rtpg_mqt_controller_get: null handle");
    if (state) *state = c->state;
    if (iteration) *iteration = c->iteration;
    if (samples_in_pass) *samples_in_pass = c->per_tmp;
    if (executing) *executing = c->executing ? 1 : 0;
    return RTPG_OK;
}

}  // extern "C"
