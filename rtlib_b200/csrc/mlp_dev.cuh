// Learned directional guide: a 3 x 64 ReLU MLP emitting an 8-lobe von Mises-Fisher mixture,
// run on the 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory, FP32
// accumulators in tensor memory).
//
// One CTA of 128 threads owns a tile of 128 samples: thread t computes the features of sample
// t, one elected thread issues the MMAs of a layer, and thread t reads row t of the
// accumulator back from tensor memory (TMEM lane t) for the epilogue.  Matrices live in shared
// memory in the no-swizzle "core matrix" layout of the UMMA descriptors: 8 rows x 16 bytes
// (8 bf16) per 128-byte core matrix, core matrices of a row group adjacent (128 B apart), row
// groups (C / 8) * 128 B apart for a C-column matrix.  The same storage serves as a K-major
// operand (K = columns) and as an MN-major operand (MN = columns, K = rows), which is how the
// backward GEMMs use the forward activations and weights without a transposed copy.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"
#include "tracer_dev.cuh"  // float3 helpers

namespace rtpg {

constexpr int kMlpTile = 128;   // samples per CTA tile = MMA M = TMEM lanes
constexpr int kMlpIn = 80;      // 72 sin/cos features + normal 3 + outgoing direction 3 + 1 + pad
constexpr int kMlpHidden = 64;  // width of the 3 hidden layers
constexpr int kMlpOut = 48;     // 8 lobes x (mean 3, log kappa 1, logit 1) = 40, padded
constexpr int kMlpLobes = 8;
constexpr int kMlpFreqs = 12;
// parameter block: W0 [80 x 64], W1 [64 x 64], W2 [64 x 64], W3 [64 x 48], row-major [in][out]
constexpr int kW0 = 0, kW1 = kMlpIn * kMlpHidden, kW2 = kW1 + kMlpHidden * kMlpHidden,
              kW3 = kW2 + kMlpHidden * kMlpHidden, kMlpParams = kW3 + kMlpHidden * kMlpOut;  // 16384
constexpr float kLogKappaMin = -2.3f, kLogKappaMax = 6.9f;  // kappa in [0.1, ~1000]
constexpr float kWeightClamp = 20.0f;  // training weights clamped at 20 x their minibatch mean

// element offset of (row, col) of a matrix with `ncols` columns in the core-matrix layout
__host__ __device__ __forceinline__ uint32_t blk(uint32_t row, uint32_t col, uint32_t ncols) {
    return ((row >> 3) * (ncols >> 3) + (col >> 3)) * 64u + (row & 7u) * 8u + (col & 7u);
}

// ------------------------------------------------------------------ tcgen05 plumbing
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, no swizzle: start address, leading / stride byte offsets
// (all >> 4), version 1 at bit 46, layout type 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major operand: rows = M (or N), K = columns kk .. kk+15 of a matrix with `ncols` columns
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t base, uint32_t kk, uint32_t ncols) {
    return umma_desc(base + (kk >> 3) * 128u, 128u, (ncols >> 3) * 128u);
}
// MN-major operand: K = rows kk .. kk+15, MN = columns of a matrix with `ncols` columns
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t base, uint32_t kk, uint32_t ncols) {
    return umma_desc(base + (kk >> 3) * (ncols >> 3) * 128u, (ncols >> 3) * 128u, 128u);
}
// instruction descriptor of kind::f16: D F32, A and B BF16, majors, N >> 3, M >> 4
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t m, uint32_t n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? (1u << 15) : 0u) | (b_mn ? (1u << 16) : 0u) |
           ((n >> 3) << 17) | ((m >> 4) << 24);
}
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// polls of a bounded mbarrier wait before it gives up
constexpr uint32_t kMbarPollLimit = 1u << 22;
// Wait for the phase `parity` of the barrier to complete, at most `limit` polls; returns
// false on a timeout (the caller records an error status, issues no further MMA and leaves,
// so no wait is endless).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit = kMbarPollLimit) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w .. 32w+31);
// the load is asynchronous until tmem_wait_ld()
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    tmem_ld16_async(taddr, r);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// `n` (a multiple of 16, at most 64) columns with the loads in flight together
template <int N>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, float* v) {
    uint32_t r[N];
#pragma unroll
    for (int c = 0; c < N; c += 16) tmem_ld16_async(taddr + c, r + c);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 floats -> 8 bf16 (round to nearest even) stored as one 16-byte core-matrix row chunk
__device__ __forceinline__ void st_bf16x8(__nv_bfloat16* dst, const float* v) {
    __align__(16) __nv_bfloat162 p[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(p);
}

// ------------------------------------------------------------------ features
// Position normalised to the AABB, 12 frequencies of sin / cos of pi 2^j u per axis, then the
// shading normal, the outgoing direction, a constant 1 (the first layer's bias) and a zero.
__device__ __forceinline__ void mlp_features(float3 pos, float3 nrm, float3 wo, float3 mn, float3 inv_ext, float* f) {
    const float u[3] = {(pos.x - mn.x) * inv_ext.x, (pos.y - mn.y) * inv_ext.y, (pos.z - mn.z) * inv_ext.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float a = u[c];
#pragma unroll
        for (int j = 0; j < kMlpFreqs; ++j) {
            float s, co;
            sincospif(a, &s, &co);
            f[c * 24 + 2 * j] = s;
            f[c * 24 + 2 * j + 1] = co;
            a = a * 2.0f;
        }
    }
    f[72] = nrm.x; f[73] = nrm.y; f[74] = nrm.z;
    f[75] = wo.x; f[76] = wo.y; f[77] = wo.z;
    f[78] = 1.0f; f[79] = 0.0f;
}

// ------------------------------------------------------------------ vMF mixture
struct VmfLobe {
    float3 mu;
    float kappa, weight;
};
// raw network outputs of one sample -> lobes (normalised mean, kappa = exp(clamped), softmax)
__device__ __forceinline__ void mlp_head(const float* o, VmfLobe* L) {
    float mx = -1e30f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; ++k) mx = fmaxf(mx, o[5 * k + 4]);
    float se = 0.0f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; ++k) {
        const float3 m = f3(o[5 * k], o[5 * k + 1], o[5 * k + 2]);
        const float len = sqrtf(dot3(m, m));
        L[k].mu = len > 1e-12f ? m * (1.0f / len) : f3(0.f, 0.f, 1.f);
        L[k].kappa = __expf(fminf(fmaxf(o[5 * k + 3], kLogKappaMin), kLogKappaMax));
        L[k].weight = __expf(o[5 * k + 4] - mx);
        se += L[k].weight;
    }
    const float inv = 1.0f / se;
#pragma unroll
    for (int k = 0; k < kMlpLobes; ++k) L[k].weight *= inv;
}
// density of one lobe at w: kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu.w - 1))
__device__ __forceinline__ float vmf_pdf(const VmfLobe& l, float3 w) {
    const float k = l.kappa;
    return k / (6.28318530717958647692f * (1.0f - __expf(-2.0f * k))) * __expf(k * (dot3(l.mu, w) - 1.0f));
}
__device__ __forceinline__ float vmf_mixture_pdf(const VmfLobe* L, float3 w) {
    float p = 0.0f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; ++k) p += L[k].weight * vmf_pdf(L[k], w);
    return p;
}
// lobe by weight, then the vMF sample of W. Jakob's note: cos = 1 + log(u + (1-u) e^{-2k}) / k
__device__ __forceinline__ float3 vmf_mixture_sample(const VmfLobe* L, float u0, float u1, float u2) {
    int sel = kMlpLobes - 1;
    float c = 0.0f;
    for (int k = 0; k < kMlpLobes - 1; ++k) {
        c += L[k].weight;
        if (u0 < c) {
            sel = k;
            break;
        }
    }
    const VmfLobe l = L[sel];
    const float k = l.kappa;
    float cz = 1.0f + __logf(u1 + (1.0f - u1) * __expf(-2.0f * k)) / k;
    cz = fminf(fmaxf(cz, -1.0f), 1.0f);
    const float sz = sqrtf(fmaxf(0.0f, 1.0f - cz * cz));
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    // orthonormal frame around mu (Duff et al. 2017)
    const float3 n = l.mu;
    const float sg = copysignf(1.0f, n.z);
    const float a = -1.0f / (sg + n.z), b = n.x * n.y * a;
    const float3 t = f3(1.0f + sg * n.x * n.x * a, sg * b, -sg * n.x);
    const float3 bt = f3(b, sg + n.y * n.y * a, -n.y);
    return t * (sz * cp) + bt * (sz * sp) + n * cz;
}

// ------------------------------------------------------------------ network building blocks
constexpr int kMlpThreads = kMlpTile;
constexpr size_t kSmemW = size_t(kMlpParams) * 2;             // 32 KB of bf16 weights
constexpr size_t kSmemX = size_t(kMlpTile) * kMlpIn * 2;       // 20 KB input features
constexpr size_t kSmemH = size_t(kMlpTile) * kMlpHidden * 2;   // 16 KB per hidden activation
constexpr size_t kSmemEval = kSmemW + kSmemX + 64;
constexpr size_t kSmemTrain = kSmemW + kSmemX + 4 * kSmemH + 64;  // X0, H1, H2, H3, dY
// TMEM columns of the training kernel: forward / dX accumulator, then dW^T of layers 3..0
constexpr uint32_t kColD = 0, kColW3 = 64, kColW2 = 128, kColW1 = 192, kColW0 = 256, kTrainCols = 512;
constexpr uint32_t kEvalCols = 64;

struct MlpDev {
    const __nv_bfloat16* wq;  // bf16 weights, each matrix in the core-matrix layout
    float3 mn, inv_ext;       // AABB of the positions
    unsigned* status;
    // Test mode of the bounded waits (rtpg_mlp_set_wait_test): skip_mma = 1 issues neither
    // the MMAs nor their commit, so the completion barrier never arrives and the wait runs
    // out after poll_limit polls with nothing in flight.  Normal use: 0 and kMbarPollLimit.
    uint32_t skip_mma;
    uint32_t poll_limit;
};

// After a wait that gave up: one more bounded wait on the same phase, so that an MMA still in
// flight (one that completes after the timeout) has finished before its TMEM is freed.
// Every thread of the CTA calls it.
__device__ __forceinline__ void mma_drain(uint64_t* mbar, uint32_t phase, uint32_t limit) {
    (void)mbar_wait(mbar, phase, limit);
    tc_fence_after();
}

// the learned guide as the tracer sees it: weights and the record buffer it appends to
struct MlpView {
    MlpDev dev;
    float *r_pos, *r_nrm, *r_wo, *r_wi, *r_w;
    float* r_pdf;  // the density the record's direction was sampled with (the vertex's woPdf)
    uint32_t* r_count;
    uint32_t capacity;
};

struct Records {
    const float* pos;  // 3 per record
    const float* nrm;
    const float* wo;
    const float* wi;
    const float* w;    // weight (>= 0)
};

// ------------------------------------------------------------------ shared building blocks
__device__ __forceinline__ void load_weights(__nv_bfloat16* ws, const __nv_bfloat16* wq) {
    const uint4* s = reinterpret_cast<const uint4*>(wq);
    uint4* d = reinterpret_cast<uint4*>(ws);
    for (int i = threadIdx.x; i < kMlpParams / 8; i += blockDim.x) d[i] = __ldg(s + i);
}
// features of sample t into row t of X0
__device__ __forceinline__ void store_features(__nv_bfloat16* x0, int t, const float* f) {
#pragma unroll
    for (int c = 0; c < kMlpIn; c += 8) st_bf16x8(x0 + blk(t, c, kMlpIn), f + c);
}
// all threads: make the shared-memory operands written by this CTA visible to the tensor
// cores and order earlier TMEM loads before the next MMA
__device__ __forceinline__ void mma_barrier() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}
// D[128 x n] (+)= A[128 x k] (K-major, a_cols columns) x W[k x n] (MN-major, n columns)
__device__ __forceinline__ void issue_fwd(uint32_t d, uint32_t a, uint32_t a_cols, uint32_t k, uint32_t w, uint32_t n) {
    const uint32_t id = umma_idesc(128, n, false, true);
    for (uint32_t kk = 0; kk < k; kk += 16) umma_f16(d, desc_kmajor(a, kk, a_cols), desc_mnmajor(w, kk, n), id, kk > 0);
}
// D[128 x nin] = dY[128 x kout] (K-major, 64 columns) x W^T, W stored [nin x kout]
__device__ __forceinline__ void issue_dx(uint32_t d, uint32_t dy, uint32_t kout, uint32_t w, uint32_t nin) {
    const uint32_t id = umma_idesc(128, nin, false, false);
    for (uint32_t kk = 0; kk < kout; kk += 16)
        umma_f16(d, desc_kmajor(dy, kk, kMlpHidden), desc_kmajor(w, kk, kout), id, kk > 0);
}
// D[64 x nin] (+)= dY^T[64 x 128] x X[128 x nin]  (dW^T of a layer over one tile)
__device__ __forceinline__ void issue_dw(uint32_t d, uint32_t dy, uint32_t x, uint32_t x_cols, uint32_t nin, bool acc) {
    const uint32_t id = umma_idesc(64, nin, true, true);
    for (uint32_t kk = 0; kk < kMlpTile; kk += 16)
        umma_f16(d, desc_mnmajor(dy, kk, kMlpHidden), desc_mnmajor(x, kk, x_cols), id, (acc || kk > 0) ? 1u : 0u);
}
// thread t: accumulator row t, columns c0 .. c0+15
__device__ __forceinline__ void ld_row16(uint32_t tmem, uint32_t col, float* v) {
    const uint32_t lane = (threadIdx.x & ~31u);
    tmem_ld16(tmem + (lane << 16) + col, v);
}
// thread t: accumulator row t, columns c0 .. c0+N-1 in one batch of loads
template <int N>
__device__ __forceinline__ void ld_row(uint32_t tmem, uint32_t col, float* v) {
    const uint32_t lane = (threadIdx.x & ~31u);
    tmem_ld_cols<N>(tmem + (lane << 16) + col, v);
}
// hidden epilogue: ReLU, bf16, row t of h [128 x 64]
__device__ __forceinline__ void epilogue_relu(uint32_t tmem, __nv_bfloat16* h) {
    const int t = threadIdx.x;
    float v[kMlpHidden];
    ld_row<kMlpHidden>(tmem, kColD, v);
#pragma unroll
    for (int i = 0; i < kMlpHidden; ++i) v[i] = fmaxf(v[i], 0.0f);
#pragma unroll
    for (int c = 0; c < kMlpHidden; c += 8) st_bf16x8(h + blk(t, c, kMlpHidden), v + c);
}

// Completion of the MMAs thread 0 committed to `mbar`: every thread waits (bounded), and the
// outcome is made uniform over the CTA.  On success the phase flips; on a timeout it stays,
// so mma_drain can wait for the same phase before TMEM is freed.
__device__ __forceinline__ bool mma_complete(uint64_t* mbar, uint32_t& phase, uint32_t limit) {
    const bool ok = __syncthreads_and(mbar_wait(mbar, phase, limit)) != 0;
    if (ok) phase ^= 1u;
    tc_fence_after();
    return ok;
}

// Forward pass of one tile: the features of sample t are in row t of x0 (which the hidden
// activations then overwrite); returns sample t's 48 raw outputs in o.  Every thread of the
// 128-thread CTA calls it; thread 0 issues the MMAs.  False (uniformly over the CTA, with o
// not written) if a wait on the tensor cores gave up: the caller then issues nothing more,
// drains with mma_drain and frees its TMEM.
__device__ __forceinline__ bool mlp_forward_tile(const MlpDev& P, uint32_t tmem, uint32_t sw, __nv_bfloat16* x0,
                                                 uint64_t* mbar, uint32_t& phase, float* o) {
    const uint32_t sx = smem_u32(x0);
    for (int l = 0; l < 4; ++l) {
        mma_barrier();
        if (threadIdx.x == 0 && !P.skip_mma) {
            if (l == 0) issue_fwd(tmem + kColD, sx, kMlpIn, kMlpIn, sw + 2 * kW0, kMlpHidden);
            else if (l < 3) issue_fwd(tmem + kColD, sx, kMlpHidden, kMlpHidden, sw + 2 * (l == 1 ? kW1 : kW2), kMlpHidden);
            else issue_fwd(tmem + kColD, sx, kMlpHidden, kMlpHidden, sw + 2 * kW3, kMlpOut);
            umma_commit(mbar);
        }
        if (!mma_complete(mbar, phase, P.poll_limit)) return false;
        if (l < 3) epilogue_relu(tmem, x0);
    }
    ld_row<kMlpOut>(tmem, kColD, o);
    return true;
}

}  // namespace rtpg
