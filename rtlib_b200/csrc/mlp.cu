// Learned directional guide (rtpg_mlp_*): inference and training of the vMF-mixture MLP on
// the tensor cores (tcgen05), Adam, and the record buffer the tracer fills.
//
// The guide has no counterpart in RTLib; it learns the same quantity the SD-tree records per
// trace vertex (TraceVertexT::Commit, OPX7UtilsPathGuiding.h:830-866: the luminance of the
// incident radiance times |cos| over the sampling pdf, in the sampled direction) and is trained
// to minimise the weighted negative log-likelihood of those directions (the KL divergence of
// the mixture to the recorded radiance distribution).
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "common.cuh"
#include "mlp_dev.cuh"

namespace rtpg {

// ------------------------------------------------------------------ inference
// N floats (a multiple of 4) to dst: 16-byte stores if dst is 16-byte aligned, else scalars
template <int N>
__device__ __forceinline__ void store_row(float* dst, const float* v) {
    if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
#pragma unroll
        for (int c = 0; c < N; c += 4) *reinterpret_cast<float4*>(dst + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
    } else {
#pragma unroll
        for (int c = 0; c < N; ++c) dst[c] = v[c];
    }
}

// out_raw: 48 floats per sample (the network output); out_lobes: 40 floats per sample, lobe k
// = (mu xyz, kappa, weight).  Either may be null.
__global__ void __launch_bounds__(kMlpThreads) k_mlp_eval(MlpDev P, int64_t n, const float* __restrict__ pos,
                                                         const float* __restrict__ nrm, const float* __restrict__ wo,
                                                         float* __restrict__ out_raw, float* __restrict__ out_lobes) {
    extern __shared__ __align__(128) uint8_t sm[];
    __nv_bfloat16* ws = reinterpret_cast<__nv_bfloat16*>(sm);
    __nv_bfloat16* x0 = reinterpret_cast<__nv_bfloat16*>(sm + kSmemW);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kSmemW + kSmemX);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmemW + kSmemX + 8);
    const int t = threadIdx.x;
    if (t < 32) tmem_alloc(tslot, kEvalCols);
    if (t == 0) mbar_init(mbar, 1);
    load_weights(ws, P.wq);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t sw = smem_u32(ws);
    uint32_t phase = 0;
    bool ok = true;
    for (int64_t base = int64_t(blockIdx.x) * kMlpTile; base < n; base += int64_t(gridDim.x) * kMlpTile) {
        const int64_t i = base + t;
        float f[kMlpIn];
        if (i < n) {
            mlp_features(f3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), f3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]),
                         f3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), P.mn, P.inv_ext, f);
        } else {
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) f[k] = 0.0f;
        }
        store_features(x0, t, f);
        float o[kMlpOut];
        if (!mlp_forward_tile(P, tmem, sw, x0, mbar, phase, o)) {
            ok = false;  // uniform over the CTA: issue nothing more
            break;
        }
        if (i < n) {
            // a sample's row (192 or 160 bytes) in 16-byte stores when the array allows it
            if (out_raw) store_row<kMlpOut>(out_raw + i * kMlpOut, o);
            if (out_lobes) {
                VmfLobe L[kMlpLobes];
                mlp_head(o, L);
                float q[40];
#pragma unroll
                for (int k = 0; k < kMlpLobes; ++k) {
                    q[5 * k] = L[k].mu.x; q[5 * k + 1] = L[k].mu.y; q[5 * k + 2] = L[k].mu.z;
                    q[5 * k + 3] = L[k].kappa; q[5 * k + 4] = L[k].weight;
                }
                store_row<40>(out_lobes + i * 40, q);
            }
        }
    }
    if (!ok) {
        if (t == 0) atomicOr(P.status, RTPG_STATUS_TIMEOUT);
        mma_drain(mbar, phase, P.poll_limit);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t < 32) tmem_dealloc(tmem, kEvalCols);
}

// ------------------------------------------------------------------ training
// d(loss)/d(raw outputs) of one record: loss = -w log q(wi) (scaled by inv_wsum), q the mixture
// of mlp_head.  Returns -log q.
__device__ __forceinline__ float head_grad(const float* o, float3 wi, float scale, float* g) {
    VmfLobe L[kMlpLobes];
    mlp_head(o, L);
    float fk[kMlpLobes], q = 0.0f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; ++k) {
        fk[k] = vmf_pdf(L[k], wi);
        q += L[k].weight * fk[k];
    }
    q = fmaxf(q, 1e-30f);
#pragma unroll
    for (int c = 0; c < kMlpOut; ++c) g[c] = 0.0f;
#pragma unroll
    for (int k = 0; k < kMlpLobes; ++k) {
        const float r = L[k].weight * fk[k] / q;  // responsibility
        const float3 m = f3(o[5 * k], o[5 * k + 1], o[5 * k + 2]);
        const float len = fmaxf(sqrtf(dot3(m, m)), 1e-12f);
        const float kap = L[k].kappa, mw = dot3(L[k].mu, wi);
        // d log q / d m = r kappa (wi - (mu.wi) mu) / |m|
        const float3 gm = (wi - L[k].mu * mw) * (r * kap / len);
        const float e = __expf(-2.0f * kap);
        const float dlk = 1.0f / kap - 2.0f * e / (1.0f - e) + (mw - 1.0f);
        const float s = o[5 * k + 3];
        const float gs = (s > kLogKappaMin && s < kLogKappaMax) ? r * kap * dlk : 0.0f;
        g[5 * k] = -scale * gm.x;
        g[5 * k + 1] = -scale * gm.y;
        g[5 * k + 2] = -scale * gm.z;
        g[5 * k + 3] = -scale * gs;
        g[5 * k + 4] = -scale * (r - L[k].weight);
    }
    return -__logf(q);
}

// One pass over n records: forward, loss gradient, backward; dW of all layers accumulate in
// TMEM across the CTA's tiles and are added to grads (fp32, [in][out] per layer) at the end.
__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_train(MlpDev P, int64_t n, Records R, const float* wsum,
                                                            float* __restrict__ grads, float* __restrict__ loss_sum) {
    extern __shared__ __align__(128) uint8_t sm[];
    __nv_bfloat16* ws = reinterpret_cast<__nv_bfloat16*>(sm);
    __nv_bfloat16* x0 = reinterpret_cast<__nv_bfloat16*>(sm + kSmemW);
    __nv_bfloat16* hs[3];
    for (int k = 0; k < 3; ++k) hs[k] = reinterpret_cast<__nv_bfloat16*>(sm + kSmemW + kSmemX + k * kSmemH);
    __nv_bfloat16* dy = reinterpret_cast<__nv_bfloat16*>(sm + kSmemW + kSmemX + 3 * kSmemH);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kSmemW + kSmemX + 4 * kSmemH);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kSmemW + kSmemX + 4 * kSmemH + 8);
    const int t = threadIdx.x;
    if (t < 32) tmem_alloc(tslot, kTrainCols);
    if (t == 0) mbar_init(mbar, 1);
    load_weights(ws, P.wq);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t sw = smem_u32(ws), sx = smem_u32(x0), sdy = smem_u32(dy);
    const uint32_t sh[3] = {smem_u32(hs[0]), smem_u32(hs[1]), smem_u32(hs[2])};
    const float scale = (wsum && *wsum > 0.0f) ? 1.0f / *wsum : 0.0f;
    // record weights are Monte Carlo estimates with a heavy tail: clamp at kWeightClamp times
    // their mean so that single rare paths do not dominate a step
    const float wmax = (wsum && n > 0) ? kWeightClamp * (*wsum / (float)n) : 0.0f;
    uint32_t phase = 0;
    bool ok = true, first = true;
    float lsum = 0.0f;
    // commit the MMAs thread 0 issued and wait for them; false (uniform over the CTA) when the
    // wait gave up, after which nothing more is issued
    auto sync_mma = [&]() -> bool {
        if (t == 0 && !P.skip_mma) umma_commit(mbar);
        return mma_complete(mbar, phase, P.poll_limit);
    };
    for (int64_t base = int64_t(blockIdx.x) * kMlpTile; base < n; base += int64_t(gridDim.x) * kMlpTile) {
        const int64_t i = base + t;
        float f[kMlpIn];
        float3 wi = f3(0.f, 0.f, 1.f);
        float w = 0.0f;
        if (i < n) {
            mlp_features(f3(R.pos[3 * i], R.pos[3 * i + 1], R.pos[3 * i + 2]),
                         f3(R.nrm[3 * i], R.nrm[3 * i + 1], R.nrm[3 * i + 2]),
                         f3(R.wo[3 * i], R.wo[3 * i + 1], R.wo[3 * i + 2]), P.mn, P.inv_ext, f);
            wi = f3(R.wi[3 * i], R.wi[3 * i + 1], R.wi[3 * i + 2]);
            w = fminf(fmaxf(R.w[i], 0.0f), wmax);
        } else {
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) f[k] = 0.0f;
        }
        store_features(x0, t, f);
        // forward, keeping H1..H3
        for (int l = 0; l < 4; ++l) {
            mma_barrier();
            if (t == 0 && !P.skip_mma) {
                if (l == 0) issue_fwd(tmem + kColD, sx, kMlpIn, kMlpIn, sw + 2 * kW0, kMlpHidden);
                else if (l < 3) issue_fwd(tmem + kColD, sh[l - 1], kMlpHidden, kMlpHidden, sw + 2 * (l == 1 ? kW1 : kW2), kMlpHidden);
                else issue_fwd(tmem + kColD, sh[2], kMlpHidden, kMlpHidden, sw + 2 * kW3, kMlpOut);
            }
            if (!(ok = sync_mma())) break;
            if (l < 3) epilogue_relu(tmem, hs[l]);
        }
        if (!ok) break;
        // loss gradient at the outputs -> dY [128 x 64] (columns 40..63 zero)
        {
            float o[kMlpOut], g[kMlpHidden];
            ld_row<kMlpOut>(tmem, kColD, o);
            const float nl = head_grad(o, wi, w * scale, g);
            if (w > 0.0f) lsum += w * nl;
#pragma unroll
            for (int c = kMlpOut; c < kMlpHidden; ++c) g[c] = 0.0f;
#pragma unroll
            for (int c = 0; c < kMlpHidden; c += 8) st_bf16x8(dy + blk(t, c, kMlpHidden), g + c);
        }
        // backward: layer 3 .. 0
        for (int l = 3; l >= 0; --l) {
            mma_barrier();
            if (t == 0 && !P.skip_mma) {
                const uint32_t cw = l == 3 ? kColW3 : (l == 2 ? kColW2 : (l == 1 ? kColW1 : kColW0));
                if (l > 0) {
                    issue_dw(tmem + cw, sdy, sh[l - 1], kMlpHidden, kMlpHidden, !first);
                    const uint32_t wl = l == 3 ? kW3 : (l == 2 ? kW2 : kW1);
                    issue_dx(tmem + kColD, sdy, l == 3 ? kMlpOut : kMlpHidden, sw + 2 * wl, kMlpHidden);
                } else {
                    issue_dw(tmem + cw, sdy, sx, kMlpIn, kMlpIn, !first);
                }
            }
            if (!(ok = sync_mma())) break;
            if (l > 0) {
                // dH = dX masked by ReLU' of the activation it came from, back into dY
                const __nv_bfloat16* hl = hs[l - 1];
                float v[kMlpHidden];
                ld_row<kMlpHidden>(tmem, kColD, v);
#pragma unroll
                for (int c = 0; c < kMlpHidden; c += 8) {
                    // the activation's 8 bf16 of this chunk in one 16-byte load
                    const uint4 hv = *reinterpret_cast<const uint4*>(hl + blk(t, c, kMlpHidden));
                    const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(&hv);
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (!(__bfloat162float(hb[k]) > 0.0f)) v[c + k] = 0.0f;
                    st_bf16x8(dy + blk(t, c, kMlpHidden), v + c);
                }
            }
        }
        if (!ok) break;
        first = false;
    }
    // flush dW^T (M = 64 rows in lanes 16w .. 16w+15 of warp w's quarter) into grads; after a
    // wait gave up the accumulators are incomplete and nothing is flushed
    if (!first && ok) {
        const int warp = t >> 5, lane = t & 31;
        const int row = 16 * warp + lane;  // output feature
        const uint32_t cols[4] = {kColW0, kColW1, kColW2, kColW3};
        const int nin[4] = {kMlpIn, kMlpHidden, kMlpHidden, kMlpHidden};
        const int nout[4] = {kMlpHidden, kMlpHidden, kMlpHidden, kMlpOut};
        const int off[4] = {kW0, kW1, kW2, kW3};
        for (int l = 0; l < 4; ++l) {
            for (int c = 0; c < nin[l]; c += 16) {
                float v[16];
                ld_row16(tmem, cols[l] + c, v);
                if (lane < 16 && row < nout[l])
                    for (int k = 0; k < 16; ++k)
                        if (v[k] != 0.0f) atomicAdd(grads + off[l] + (c + k) * nout[l] + row, v[k]);
            }
        }
    }
    // loss
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((t & 31) == 0 && lsum != 0.0f) atomicAdd(loss_sum, lsum * scale);
    if (!ok) {
        if (t == 0) atomicOr(P.status, RTPG_STATUS_TIMEOUT);
        mma_drain(mbar, phase, P.poll_limit);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (t < 32) tmem_dealloc(tmem, kTrainCols);
}

__global__ void k_wsum(int64_t n, const float* w, float* out) {
    float s = 0.0f;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        s += fmaxf(w[i], 0.0f);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0.0f) atomicAdd(out, s);
}

// fp32 master [in][out] -> bf16 core-matrix layout of each matrix
__device__ __forceinline__ uint32_t packed_index(int i) {
    const int l = i < kW1 ? 0 : (i < kW2 ? 1 : (i < kW3 ? 2 : 3));
    const int off = l == 0 ? kW0 : (l == 1 ? kW1 : (l == 2 ? kW2 : kW3));
    const int nout = l == 3 ? kMlpOut : kMlpHidden;
    const int r = (i - off) / nout, c = (i - off) % nout;
    return off + blk(r, c, nout);
}
__global__ void k_mlp_pack(const float* w, __nv_bfloat16* wq) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x)
        wq[packed_index(i)] = __float2bfloat16_rn(w[i]);
}
// Adam (Kingma & Ba 2015) with bias correction; grads zeroed after use
__global__ void k_mlp_adam(float* w, float* g, float* m, float* v, __nv_bfloat16* wq, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        g[i] = 0.0f;
        wq[packed_index(i)] = __float2bfloat16_rn(wi);
    }
}

}  // namespace rtpg

using namespace rtpg;

struct rtpg_mlp {
    MlpDev dev{};
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr, *scratch = nullptr;  // scratch: wsum, loss
    __nv_bfloat16* wq = nullptr;
    float lr = 1e-3f, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    uint32_t step = 0;
    float mn[3], mx[3];
    // record buffer (filled by the tracer or rtpg_mlp_add_records)
    uint32_t capacity = 0;
    float *r_pos = nullptr, *r_nrm = nullptr, *r_wo = nullptr, *r_wi = nullptr, *r_w = nullptr, *r_pdf = nullptr;
    uint32_t* r_count = nullptr;
    unsigned* status = nullptr;
    std::vector<void*> allocs;
    template <class T>
    int alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(RTPG_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        allocs.push_back(q);
        *p = static_cast<T*>(q);
        return RTPG_OK;
    }
    ~rtpg_mlp() {
        for (void* p : allocs) cudaFree(p);
    }
};

namespace rtpg {
MlpView mlp_view(const rtpg_mlp* h) {
    return MlpView{h->dev, h->r_pos, h->r_nrm, h->r_wo, h->r_wi, h->r_w, h->r_pdf, h->r_count, h->capacity};
}
size_t mlp_eval_smem() { return kSmemEval; }
}

static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static bool g_mlp_attr = false;
static int mlp_set_attrs() {
    if (g_mlp_attr) return RTPG_OK;
    RTPG_CUDA(cudaFuncSetAttribute(k_mlp_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemEval));
    RTPG_CUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTrain));
    g_mlp_attr = true;
    return RTPG_OK;
}

extern "C" {

int rtpg_mlp_create(const float* aabb_min, const float* aabb_max, uint32_t seed, float learning_rate,
                    uint32_t record_capacity, rtpg_mlp** out) {
    if (!aabb_min || !aabb_max || !out) return fail(RTPG_EINVAL, "rtpg_mlp_create: null argument");
    for (int k = 0; k < 3; ++k)
        if (!(aabb_max[k] > aabb_min[k])) return fail(RTPG_EINVAL, "rtpg_mlp_create: empty AABB");
    int r = mlp_set_attrs();
    if (r) return r;
    auto* h = new (std::nothrow) rtpg_mlp();
    if (!h) return fail(RTPG_ENOMEM, "rtpg_mlp_create: out of host memory");
    h->lr = learning_rate > 0.0f ? learning_rate : 1e-3f;
    h->capacity = record_capacity;
    const size_t C = std::max<uint32_t>(record_capacity, 1);
    if ((r = h->alloc(&h->w, kMlpParams)) || (r = h->alloc(&h->g, kMlpParams)) || (r = h->alloc(&h->m, kMlpParams)) ||
        (r = h->alloc(&h->v, kMlpParams)) || (r = h->alloc(&h->wq, kMlpParams)) || (r = h->alloc(&h->scratch, 4)) ||
        (r = h->alloc(&h->r_pos, 3 * C)) || (r = h->alloc(&h->r_nrm, 3 * C)) || (r = h->alloc(&h->r_wo, 3 * C)) ||
        (r = h->alloc(&h->r_wi, 3 * C)) || (r = h->alloc(&h->r_w, C)) || (r = h->alloc(&h->r_pdf, C)) ||
        (r = h->alloc(&h->r_count, 1)) ||
        (r = h->alloc(&h->status, 1))) {
        delete h;
        return r;
    }
    for (int k = 0; k < 3; ++k) {
        h->mn[k] = aabb_min[k];
        h->mx[k] = aabb_max[k];
    }
    h->dev.mn = make_float3(aabb_min[0], aabb_min[1], aabb_min[2]);
    h->dev.inv_ext = make_float3(1.0f / (aabb_max[0] - aabb_min[0]), 1.0f / (aabb_max[1] - aabb_min[1]),
                                 1.0f / (aabb_max[2] - aabb_min[2]));
    h->dev.wq = h->wq;
    h->dev.status = h->status;
    h->dev.skip_mma = 0;
    h->dev.poll_limit = kMbarPollLimit;
    // He-uniform initialisation from a seeded SplitMix64 stream; output padding columns zero
    std::vector<float> w(kMlpParams, 0.0f);
    uint64_t s = 0x5DEECE66Dull ^ (uint64_t(seed) << 17);
    const int nin[4] = {kMlpIn, kMlpHidden, kMlpHidden, kMlpHidden};
    const int nout[4] = {kMlpHidden, kMlpHidden, kMlpHidden, kMlpOut};
    const int off[4] = {kW0, kW1, kW2, kW3};
    for (int l = 0; l < 4; ++l) {
        const float bound = std::sqrt(6.0f / (float)(l == 0 ? 79 : nin[l])) * (l == 3 ? 0.5f : 1.0f);
        for (int i = 0; i < nin[l]; ++i)
            for (int o = 0; o < nout[l]; ++o) {
                const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
                float val = (float)((2.0 * u - 1.0) * bound);
                if ((l == 0 && i >= 79) || (l == 3 && o >= 40)) val = 0.0f;
                w[off[l] + i * nout[l] + o] = val;
            }
    }
    cudaError_t e;
    if ((e = cudaMemcpy(h->w, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice)) ||
        (e = cudaMemset(h->g, 0, sizeof(float) * kMlpParams)) || (e = cudaMemset(h->m, 0, sizeof(float) * kMlpParams)) ||
        (e = cudaMemset(h->v, 0, sizeof(float) * kMlpParams)) || (e = cudaMemset(h->r_count, 0, 4)) ||
        (e = cudaMemset(h->status, 0, 4))) {
        delete h;
        return fail(RTPG_ECUDA, "rtpg_mlp_create: %s", cudaGetErrorString(e));
    }
    k_mlp_pack<<<64, 256>>>(h->w, h->wq);
    if ((e = cudaDeviceSynchronize())) {
        delete h;
        return fail(RTPG_ECUDA, "rtpg_mlp_create: %s", cudaGetErrorString(e));
    }
    *out = h;
    return RTPG_OK;
}

int rtpg_mlp_destroy(rtpg_mlp* h) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mlp_destroy: null handle");
    delete h;
    return RTPG_OK;
}

// Copy the fp32 parameters ([in][out] per layer, 16384 floats) out or in (in: also resets Adam).
int rtpg_mlp_params(rtpg_mlp* h, float* host_get, const float* host_set, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mlp_params: null handle");
    cudaStream_t st = as_stream(stream);
    if (host_set) {
        RTPG_CUDA(cudaMemcpyAsync(h->w, host_set, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, st));
        RTPG_CUDA(cudaMemsetAsync(h->m, 0, sizeof(float) * kMlpParams, st));
        RTPG_CUDA(cudaMemsetAsync(h->v, 0, sizeof(float) * kMlpParams, st));
        RTPG_CUDA(cudaMemsetAsync(h->g, 0, sizeof(float) * kMlpParams, st));
        k_mlp_pack<<<64, 256, 0, st>>>(h->w, h->wq);
        RTPG_LAUNCH_CHECK();
        h->step = 0;
    }
    if (host_get) {
        RTPG_CUDA(cudaMemcpyAsync(host_get, h->w, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, st));
        RTPG_CUDA(cudaStreamSynchronize(st));
    }
    return RTPG_OK;
}

// Network evaluation of n samples (device arrays, 3 floats each): raw outputs (48 per sample)
// and / or the mixture (8 lobes x mu xyz, kappa, weight).
int rtpg_mlp_eval(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, float* out_raw,
                  float* out_lobes, void* stream) {
    if (!h || n < 0 || (n > 0 && (!pos || !nrm || !wo))) return fail(RTPG_EINVAL, "rtpg_mlp_eval: bad arguments");
    if (n == 0) return RTPG_OK;
    const int g = (int)std::min<int64_t>((n + kMlpTile - 1) / kMlpTile, kSMs * 4);
    k_mlp_eval<<<g, kMlpThreads, kSmemEval, as_stream(stream)>>>(h->dev, n, pos, nrm, wo, out_raw, out_lobes);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

// Gradient of the loss over n records (device arrays) ADDED to host_grads-sized device buffer
// `grads` (16384 floats, NULL: the handle's own accumulator); returns the loss through
// host_loss (NULL: none).  The loss is -sum w log q(wi) / sum w.
static int mlp_grad(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, const float* wi,
                    const float* w, float* grads, cudaStream_t st) {
    RTPG_CUDA(cudaMemsetAsync(h->scratch, 0, 8, st));
    k_wsum<<<grid_for(n, 256, 4), 256, 0, st>>>(n, w, h->scratch);
    const int g = (int)std::min<int64_t>((n + kMlpTile - 1) / kMlpTile, kSMs);
    k_mlp_train<<<g, kMlpThreads, kSmemTrain, st>>>(h->dev, n, Records{pos, nrm, wo, wi, w}, h->scratch, grads,
                                                   h->scratch + 1);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_mlp_loss_grad(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, const float* wi,
                       const float* w, float* grads, float* host_loss, void* stream) {
    if (!h || n <= 0 || !pos || !nrm || !wo || !wi || !w) return fail(RTPG_EINVAL, "rtpg_mlp_loss_grad: bad arguments");
    cudaStream_t st = as_stream(stream);
    int r = mlp_grad(h, n, pos, nrm, wo, wi, w, grads ? grads : h->g, st);
    if (r) return r;
    if (host_loss) {
        RTPG_CUDA(cudaMemcpyAsync(host_loss, h->scratch + 1, 4, cudaMemcpyDeviceToHost, st));
        RTPG_CUDA(cudaStreamSynchronize(st));
    }
    return RTPG_OK;
}

// Adam steps over the record buffer (or the given records): the records are split into
// `batch`-sized minibatches, one gradient + Adam update each, `epochs` times.
int rtpg_mlp_train(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, const float* wi,
                   const float* w, uint32_t batch, uint32_t epochs, float* host_last_loss, void* stream) {
    if (!h || batch == 0) return fail(RTPG_EINVAL, "rtpg_mlp_train: bad arguments");
    cudaStream_t st = as_stream(stream);
    if (!pos) {
        uint32_t c = 0;
        RTPG_CUDA(cudaMemcpyAsync(&c, h->r_count, 4, cudaMemcpyDeviceToHost, st));
        RTPG_CUDA(cudaStreamSynchronize(st));
        n = std::min<uint32_t>(c, h->capacity);
        pos = h->r_pos; nrm = h->r_nrm; wo = h->r_wo; wi = h->r_wi; w = h->r_w;
    } else if (!nrm || !wo || !wi || !w) {
        return fail(RTPG_EINVAL, "rtpg_mlp_train: record arrays missing");
    }
    for (uint32_t e = 0; e < epochs; ++e)
        for (int64_t b = 0; b < n; b += batch) {
            const int64_t m = std::min<int64_t>(batch, n - b);
            int r = mlp_grad(h, m, pos + 3 * b, nrm + 3 * b, wo + 3 * b, wi + 3 * b, w + b, h->g, st);
            if (r) return r;
            ++h->step;
            const float c1 = 1.0f - std::pow(h->b1, (float)h->step), c2 = 1.0f - std::pow(h->b2, (float)h->step);
            k_mlp_adam<<<64, 256, 0, st>>>(h->w, h->g, h->m, h->v, h->wq, h->lr, h->b1, h->b2, h->eps, c1, c2);
            RTPG_LAUNCH_CHECK();
        }
    if (host_last_loss) {
        RTPG_CUDA(cudaMemcpyAsync(host_last_loss, h->scratch + 1, 4, cudaMemcpyDeviceToHost, st));
        RTPG_CUDA(cudaStreamSynchronize(st));
    }
    return RTPG_OK;
}

// Record buffer: count (device, may exceed capacity: records beyond it were dropped), clear.
int rtpg_mlp_records(rtpg_mlp* h, uint32_t* host_count, int clear, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mlp_records: null handle");
    cudaStream_t st = as_stream(stream);
    if (host_count) {
        RTPG_CUDA(cudaMemcpyAsync(host_count, h->r_count, 4, cudaMemcpyDeviceToHost, st));
        RTPG_CUDA(cudaStreamSynchronize(st));
    }
    if (clear) RTPG_CUDA(cudaMemsetAsync(h->r_count, 0, 4, st));
    return RTPG_OK;
}

// Device pointers of the record arrays (pos, nrm, wo, wi: 3 floats per record; w: 1).
int rtpg_mlp_record_arrays(rtpg_mlp* h, float** pos, float** nrm, float** wo, float** wi, float** w) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mlp_record_arrays: null handle");
    if (pos) *pos = h->r_pos;
    if (nrm) *nrm = h->r_nrm;
    if (wo) *wo = h->r_wo;
    if (wi) *wi = h->r_wi;
    if (w) *w = h->r_w;
    return RTPG_OK;
}

// Test mode of the bounded tensor-core waits: with skip_mma = 1 the kernels of this guide
// issue neither MMAs nor commits, so each completion wait runs out after poll_limit polls,
// sets RTPG_STATUS_TIMEOUT and the kernel returns with nothing in flight.  skip_mma = 0 and
// poll_limit = 0 restore normal operation.
int rtpg_mlp_set_wait_test(rtpg_mlp* h, int skip_mma, uint32_t poll_limit) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_mlp_set_wait_test: null handle");
    h->dev.skip_mma = skip_mma ? 1u : 0u;
    h->dev.poll_limit = poll_limit ? poll_limit : kMbarPollLimit;
    return RTPG_OK;
}

// Device pointer of the records' sampling densities (1 float per record): the woPdf with which
// the tracer sampled the record's direction, so that a record's integrand value is w * pdf.
int rtpg_mlp_record_pdfs(rtpg_mlp* h, float** wo_pdf) {
    if (!h || !wo_pdf) return fail(RTPG_EINVAL, "rtpg_mlp_record_pdfs: null argument");
    *wo_pdf = h->r_pdf;
    return RTPG_OK;
}

int rtpg_mlp_status(rtpg_mlp* h, uint32_t* host_status, int clear, void* stream) {
    if (!h || !host_status) return fail(RTPG_EINVAL, "rtpg_mlp_status: null argument");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemcpyAsync(host_status, h->status, 4, cudaMemcpyDeviceToHost, st));
    if (clear) RTPG_CUDA(cudaMemsetAsync(h->status, 0, 4, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

}  // extern "C"
