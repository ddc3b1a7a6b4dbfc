// Linear BVH build over triangles and batched hit queries (rtpg_scene_*).
//
// This is the hit-query boundary of the integrator: RTLib answers closest-hit and occlusion
// queries with OptiX (optixTrace in TraceRadiance / TraceOccluded, SimpleKernel.h:347-366,
// over a GAS built in RTLibExtOPX7TestApplication.cpp:170-198).  No OptiX SDK exists on this
// machine, so queries go to this CUDA BVH instead.
#include <cub/cub.cuh>
#include <new>
#include <vector>

#include "common.cuh"
#include "bvh_dev.cuh"
#include "hashgrid_dev.cuh"  // morton3_63

namespace rtpg {

__device__ __forceinline__ unsigned fbits_ord(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_fbits(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_scene_bounds(const float* __restrict__ v, const uint32_t* __restrict__ idx, uint32_t nt,
                               unsigned* __restrict__ bounds) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; ++k) {
            const uint32_t vi = idx[3 * t + k];
            for (int a = 0; a < 3; ++a) {
                // bounds of the centroids are enough for the Morton grid
                const float c = v[3 * vi + a];
                lo[a] = fminf(lo[a], c);
                hi[a] = fmaxf(hi[a], c);
            }
        }
    }
    for (int a = 0; a < 3; ++a) {
        float l = lo[a], h = hi[a];
        for (int o = 16; o > 0; o >>= 1) {
            l = fminf(l, __shfl_xor_sync(0xffffffffu, l, o));
            h = fmaxf(h, __shfl_xor_sync(0xffffffffu, h, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(bounds + a, fbits_ord(l));
            atomicMax(bounds + 3 + a, fbits_ord(h));
        }
    }
}

__global__ void k_scene_morton(const float* __restrict__ v, const uint32_t* __restrict__ idx, uint32_t nt,
                               const unsigned* __restrict__ bounds, unsigned long long* __restrict__ keys,
                               uint32_t* __restrict__ vals) {
    float lo[3], ext[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = ord_fbits(bounds[a]);
        ext[a] = fmaxf(ord_fbits(bounds[3 + a]) - lo[a], 1e-30f);
    }
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            const float c = (v[3 * idx[3 * t] + a] + v[3 * idx[3 * t + 1] + a] + v[3 * idx[3 * t + 2] + a]) / 3.0f;
            const float f = fminf(fmaxf((c - lo[a]) / ext[a], 0.0f), 1.0f);
            q[a] = min((uint32_t)(f * 2097152.0f), 2097151u);
        }
        keys[t] = morton3_63(q[0], q[1], q[2]);
        vals[t] = t;
    }
}

__device__ __forceinline__ int bvh_delta(const unsigned long long* __restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long a = k[i], b = k[j];
    if (a == b) return 64 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clzll(a ^ b);
}

// Karras 2012: node i covers a key range whose split is found by binary search
__global__ void k_scene_hierarchy(const unsigned long long* __restrict__ keys, int n, BvhNode* __restrict__ nodes,
                                  uint32_t* __restrict__ parent_i, uint32_t* __restrict__ parent_l) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (bvh_delta(keys, n, i, i + 1) - bvh_delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = bvh_delta(keys, n, i, i - d);
        int lmax = 2;
        while (bvh_delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (bvh_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = bvh_delta(keys, n, i, j);
        int s = 0;
        for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
            if (bvh_delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int gamma = i + s * d + min(d, 0);
        const int lo = min(i, j), hi = max(i, j);
        uint32_t c0, c1;
        if (lo == gamma) { c0 = kBvhLeafBit | (uint32_t)gamma; parent_l[gamma] = i; }
        else { c0 = (uint32_t)gamma; parent_i[gamma] = i; }
        if (hi == gamma + 1) { c1 = kBvhLeafBit | (uint32_t)(gamma + 1); parent_l[gamma + 1] = i; }
        else { c1 = (uint32_t)(gamma + 1); parent_i[gamma + 1] = i; }
        nodes[i].child[0] = c0;
        nodes[i].child[1] = c1;
        nodes[i].pad[0] = nodes[i].pad[1] = 0;
    }
}

__global__ void k_scene_leaves(const float* __restrict__ v, const uint32_t* __restrict__ idx, uint32_t nt,
                               const uint32_t* __restrict__ order, BvhTri* __restrict__ tris, uint32_t* __restrict__ prim) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
        const uint32_t p = order[k];
        const uint32_t a = idx[3 * p], b = idx[3 * p + 1], c = idx[3 * p + 2];
        float4 r[3];
        tri_transform(v[3 * a], v[3 * a + 1], v[3 * a + 2], v[3 * b], v[3 * b + 1], v[3 * b + 2], v[3 * c], v[3 * c + 1],
                      v[3 * c + 2], r);
        tris[k] = BvhTri{r[0], r[1], r[2]};
        prim[k] = p;
    }
}

// the leaves back in scene order, for small scenes
__global__ void k_scene_flat(const BvhTri* __restrict__ tris, const uint32_t* __restrict__ prim, uint32_t nt,
                             BvhTri* __restrict__ flat) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) flat[prim[k]] = tris[k];
}

// the box of scene triangle p, widened by a relative margin so that it contains the triangle
// as the hit test sees it
__device__ __forceinline__ void tri_box(const float* __restrict__ v, const uint32_t* __restrict__ idx, uint32_t p,
                                        float* lo, float* hi) {
    const uint32_t a = idx[3 * p], b = idx[3 * p + 1], c = idx[3 * p + 2];
    for (int k = 0; k < 3; ++k) {
        const float x0 = v[3 * a + k], x1 = v[3 * b + k], x2 = v[3 * c + k];
        lo[k] = fminf(x0, fminf(x1, x2));
        hi[k] = fmaxf(x0, fmaxf(x1, x2));
        const float m = 1e-6f * fmaxf(fabsf(lo[k]), fabsf(hi[k])) + 1e-12f;
        lo[k] -= m;
        hi[k] += m;
    }
}

// bottom-up boxes: the second thread to reach an interior node merges its children
__global__ void k_scene_boxes(const float* __restrict__ v, const uint32_t* __restrict__ idx,
                              const uint32_t* __restrict__ prim, uint32_t nt, BvhNode* nodes, const uint32_t* parent_i,
                              const uint32_t* parent_l, float4* ibox, unsigned* flags) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
        uint32_t node = parent_l[k];
        for (;;) {
            __threadfence();
            if (atomicAdd(flags + node, 1u) == 0) break;
            __threadfence();
            float lo[2][3], hi[2][3];
            for (int c = 0; c < 2; ++c) {
                const uint32_t ch = nodes[node].child[c];
                if (ch & kBvhLeafBit) {
                    tri_box(v, idx, prim[ch & ~kBvhLeafBit], lo[c], hi[c]);
                } else {
                    const float4 a = __ldcg(ibox + 2 * ch), b = __ldcg(ibox + 2 * ch + 1);
                    lo[c][0] = a.x; lo[c][1] = a.y; lo[c][2] = a.z;
                    hi[c][0] = b.x; hi[c][1] = b.y; hi[c][2] = b.z;
                }
            }
            nodes[node].a = make_float4(lo[0][0], lo[0][1], lo[0][2], hi[0][0]);
            nodes[node].b = make_float4(hi[0][1], hi[0][2], lo[1][0], lo[1][1]);
            nodes[node].c = make_float4(lo[1][2], hi[1][0], hi[1][1], hi[1][2]);
            __stcg(ibox + 2 * node, make_float4(fminf(lo[0][0], lo[1][0]), fminf(lo[0][1], lo[1][1]),
                                                fminf(lo[0][2], lo[1][2]), 0.0f));
            __stcg(ibox + 2 * node + 1, make_float4(fmaxf(hi[0][0], hi[1][0]), fmaxf(hi[0][1], hi[1][1]),
                                                    fmaxf(hi[0][2], hi[1][2]), 0.0f));
            if (node == 0) break;
            node = parent_i[node];
        }
    }
}

template <bool ANY>
__global__ void __launch_bounds__(128) k_scene_intersect(SceneDev s, int64_t n, const float* __restrict__ org,
                                                         const float* __restrict__ dir, const float* __restrict__ tmin,
                                                         const float* __restrict__ tmax, float* __restrict__ out_t,
                                                         uint32_t* __restrict__ out_prim, float* __restrict__ out_uv) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const Hit h = bvh_trace<ANY>(s, org[3 * i], org[3 * i + 1], org[3 * i + 2], dir[3 * i], dir[3 * i + 1],
                                     dir[3 * i + 2], tmin ? tmin[i] : 0.0f, tmax ? tmax[i] : 1e20f);
        if (out_t) out_t[i] = h.prim == 0xffffffffu ? -1.0f : h.t;
        if (out_prim) out_prim[i] = h.prim;
        if (out_uv) reinterpret_cast<float2*>(out_uv)[i] = make_float2(h.u, h.v);
    }
}

}  // namespace rtpg

using namespace rtpg;

struct rtpg_scene {
    SceneDev dev{};
    BvhNode* nodes = nullptr;
    BvhTri* tris = nullptr;
    uint32_t* prim = nullptr;
    BvhTri* flat = nullptr;
    std::vector<void*> allocs;
    size_t bytes = 0;
    template <class T>
    int alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(RTPG_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        allocs.push_back(q);
        bytes += count * sizeof(T);
        *p = static_cast<T*>(q);
        return RTPG_OK;
    }
    ~rtpg_scene() {
        for (void* p : allocs) cudaFree(p);
    }
};

namespace rtpg {
SceneDev scene_device_view(const rtpg_scene* s) { return s->dev; }
}

extern "C" {

int rtpg_scene_create(const float* vertices, uint32_t num_vertices, const uint32_t* indices, uint32_t num_triangles,
                      void* stream, rtpg_scene** out) {
    if (!out || (num_triangles && (!vertices || !indices))) return fail(RTPG_EINVAL, "rtpg_scene_create: bad arguments");
    if (num_triangles >= kBvhLeafBit) return fail(RTPG_EINVAL, "rtpg_scene_create: too many triangles");
    (void)num_vertices;
    cudaStream_t st = as_stream(stream);
    auto* s = new (std::nothrow) rtpg_scene();
    if (!s) return fail(RTPG_ENOMEM, "rtpg_scene_create: out of host memory");
    const uint32_t n = num_triangles;
    int r;
    unsigned* bounds = nullptr;
    unsigned long long *k0 = nullptr, *k1 = nullptr;
    uint32_t *v0 = nullptr, *v1 = nullptr, *pi = nullptr, *pl = nullptr;
    float4* ibox = nullptr;
    unsigned* flags = nullptr;
    void* temp = nullptr;
    size_t tb = 0;
    cub::DoubleBuffer<unsigned long long> dk(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> dv(nullptr, nullptr);
    if ((r = s->alloc(&s->nodes, n > 1 ? n - 1 : 1)) || (r = s->alloc(&s->tris, n)) || (r = s->alloc(&s->prim, n)) ||
        (n > 0 && n <= kFlatTris && (r = s->alloc(&s->flat, n)))) {
        delete s;
        return r;
    }
    s->dev.nodes = s->nodes;
    s->dev.tris = s->tris;
    s->dev.prim = s->prim;
    s->dev.flat = s->flat;
    s->dev.ntris = n;
    if (n == 0) {
        *out = s;
        return RTPG_OK;
    }
    std::vector<void*> tmp;
    auto talloc = [&](size_t bytes, void** p) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) tmp.push_back(*p);
        return e;
    };
    cudaError_t e = cudaSuccess;
    if ((e = talloc(6 * 4, (void**)&bounds)) || (e = talloc(8ull * n, (void**)&k0)) || (e = talloc(8ull * n, (void**)&k1)) ||
        (e = talloc(4ull * n, (void**)&v0)) || (e = talloc(4ull * n, (void**)&v1)) || (e = talloc(4ull * n, (void**)&pi)) ||
        (e = talloc(4ull * n, (void**)&pl)) || (e = talloc(32ull * n, (void**)&ibox)) || (e = talloc(4ull * n, (void**)&flags))) {
        for (void* p : tmp) cudaFree(p);
        delete s;
        cudaGetLastError();
        return fail(RTPG_ENOMEM, "rtpg_scene_create: scratch allocation failed");
    }
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    const int g = grid_for(n, 256, 8);
    int rc = RTPG_OK;
    do {
        if ((e = cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st))) break;
        k_scene_bounds<<<g, 256, 0, st>>>(vertices, indices, n, bounds);
        k_scene_morton<<<g, 256, 0, st>>>(vertices, indices, n, bounds, k0, v0);
        dk = cub::DoubleBuffer<unsigned long long>(k0, k1);
        dv = cub::DoubleBuffer<uint32_t>(v0, v1);
        if ((e = cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)n, 0, 63, st))) break;
        if ((e = talloc(tb, &temp))) break;
        if ((e = cub::DeviceRadixSort::SortPairs(temp, tb, dk, dv, (int)n, 0, 63, st))) break;
        k_scene_leaves<<<g, 256, 0, st>>>(vertices, indices, n, dv.Current(), s->tris, s->prim);
        if (s->flat) k_scene_flat<<<1, 64, 0, st>>>(s->tris, s->prim, n, s->flat);
        if (n > 1) {
            k_scene_hierarchy<<<g, 256, 0, st>>>(dk.Current(), (int)n, s->nodes, pi, pl);
            if ((e = cudaMemsetAsync(flags, 0, 4ull * n, st))) break;
            k_scene_boxes<<<g, 256, 0, st>>>(vertices, indices, s->prim, n, s->nodes, pi, pl, ibox, flags);
        }
        if ((e = cudaGetLastError())) break;
        if ((e = cudaStreamSynchronize(st))) break;
    } while (0);
    for (void* p : tmp) cudaFree(p);
    if (e != cudaSuccess) {
        delete s;
        return fail(RTPG_ECUDA, "rtpg_scene_create: %s", cudaGetErrorString(e));
    }
    *out = s;
    return rc;
}

int rtpg_scene_destroy(rtpg_scene* s) {
    if (!s) return fail(RTPG_EINVAL, "rtpg_scene_destroy: null handle");
    delete s;
    return RTPG_OK;
}

// Batched TraceRadiance (any_hit = 0, closest hit) / TraceOccluded (any_hit = 1).
int rtpg_scene_intersect(rtpg_scene* s, int64_t n, const float* org, const float* dir, const float* tmin,
                         const float* tmax, int any_hit, float* out_t, uint32_t* out_prim, float* out_uv, void* stream) {
    if (!s) return fail(RTPG_EINVAL, "rtpg_scene_intersect: null handle");
    if (n < 0 || (n > 0 && (!org || !dir))) return fail(RTPG_EINVAL, "rtpg_scene_intersect: bad arguments");
    if (n == 0) return RTPG_OK;
    const int g = grid_for(n, 128, 16);
    if (any_hit)
        k_scene_intersect<true><<<g, 128, 0, as_stream(stream)>>>(s->dev, n, org, dir, tmin, tmax, out_t, out_prim, out_uv);
    else
        k_scene_intersect<false><<<g, 128, 0, as_stream(stream)>>>(s->dev, n, org, dir, tmin, tmax, out_t, out_prim, out_uv);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

}  // extern "C"
