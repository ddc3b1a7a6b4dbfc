// Shared host/device helpers of rtlib_b200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <string>

#include "../../include/rtpg.h"

namespace rtpg {

// ------------------------------------------------------------------ host error plumbing
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define RTPG_CUDA(call)                                                                     \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return ::rtpg::fail(RTPG_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,     \
                                cudaGetErrorString(e_));                                    \
    } while (0)

#define RTPG_LAUNCH_CHECK() RTPG_CUDA(cudaGetLastError())

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// float2 arrays are read and written as 8-byte vectors: their base must be 8-byte aligned
inline bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }
inline bool aligned4(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 3u) == 0; }

constexpr int kSMs = 148;  // B200: 148 SMs on two dies

inline int grid_for(int64_t n, int block, int per_sm = 8) {
    int64_t g = (n + block - 1) / block;
    int64_t cap = int64_t(kSMs) * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return int(g);
}

// ------------------------------------------------------------------ constants
constexpr float kInv2Pi = 0.15915494309189533576888376337251436203445964574046f;
constexpr float k2Pi = 6.283185307179586476925286766559f;
constexpr float kPi = 3.14159265358979323846264338327950288f;
constexpr float kInvPi = 0.318309886183790691216444201927515678107738494873046875f;

// ------------------------------------------------------------------ RNG (host + device)
// Xorshift32 and the 23-bit mantissa uniform float: the generator RTLib's kernels carry in
// their per-pixel seed buffers (Random.h:37-51, Math.h:682-694).
__host__ __device__ __forceinline__ uint32_t xs32_next(uint32_t& s) {
    uint32_t y = s;
    y = y ^ (y << 13);
    y = y ^ (y >> 17);
    return s = y ^ (y << 5);
}
__host__ __device__ __forceinline__ float to_uniform_float(uint32_t v) {
    uint32_t b = (v >> 9) | (0x7Fu << 23);
#ifdef __CUDA_ARCH__
    return __fsub_rn(__uint_as_float(b), 1.0f);
#else
    float f;
    memcpy(&f, &b, 4);
    return f - 1.0f;
#endif
}
__host__ __device__ __forceinline__ float rnd1(uint32_t& s) { return to_uniform_float(xs32_next(s)); }

// pcg1d (Hash.h:13-18)
__host__ __device__ __forceinline__ uint32_t pcg1d(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

// ------------------------------------------------------------------ fixed point
// Radiance and stat-weight sums are int64(value * 2^bits), rounded to nearest, so that the
// sum of a batch does not depend on the order in which atomics land.
struct FixedPoint {
    float scale;      // 2^bits
    float inv_scale;  // 2^-bits
};
__device__ __forceinline__ unsigned long long to_fx(float v, FixedPoint fx, unsigned* status) {
    float s = __fmul_rn(v, fx.scale);
    if (!(s < 9.2233720368547758e18f)) {
        atomicOr(status, RTPG_STATUS_FX_SATURATED);
        return 0x7fffffffffffffffull;
    }
    return (unsigned long long)__float2ll_rn(s);
}
__device__ __forceinline__ float fx_to_float(unsigned long long x, FixedPoint fx) {
    return __fmul_rn(__ll2float_rn((long long)x), fx.inv_scale);
}

// Warp-aggregated 64-bit atomic add: lanes with equal keys (match.any) reduce their values
// with three 21-bit redux.sync partial sums (exact for 32 lanes of 63-bit values) and one
// lane issues the atomic.  All 32 lanes must call this converged; key == ~0 means no-op.
__device__ __forceinline__ void warp_add_u64(unsigned long long key, unsigned long long val,
                                             unsigned long long* base) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key == ~0ull) return;
    const unsigned lo = unsigned(val & 0x1FFFFFull);
    const unsigned mid = unsigned((val >> 21) & 0x1FFFFFull);
    const unsigned hi = unsigned(val >> 42);
    const unsigned slo = __reduce_add_sync(peers, lo);
    const unsigned smid = __reduce_add_sync(peers, mid);
    const unsigned shi = __reduce_add_sync(peers, hi);
    const int lane = threadIdx.x & 31;
    if (lane == __ffs(peers) - 1) {
        unsigned long long total = (unsigned long long)slo + ((unsigned long long)smid << 21) +
                                   ((unsigned long long)shi << 42);
        atomicAdd(base + key, total);
    }
}

// ------------------------------------------------------------------ block scan
// Exclusive prefix sum over a block (blockDim.x multiple of 32, <= 1024); returns the
// exclusive prefix of `v` and writes the block total to *total (all threads).
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = BLOCK / 32;
        uint32_t w = lane < NW ? smem_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NW) smem_warp[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const uint32_t before = warp ? smem_warp[warp - 1] : 0u;
    total = smem_warp[BLOCK / 32 - 1];
    __syncthreads();
    return before + x - v;
}

// ------------------------------------------------------------------ device-count scan
// Exclusive scan of in[0, *n) -> out, *total_out = sum; n lives in device memory so the
// sequence can be captured in a CUDA graph.  `partials` needs ceil(cap / kScanTile) + 1
// words of scratch.  Three launches: tile sums, scan of tile sums, tile scans.
constexpr int kScanBlock = 512;
constexpr int kScanTile = kScanBlock * 4;
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint32_t cap, uint32_t* partials,
                       uint32_t* total_out, cudaStream_t st);
inline size_t scan_partials_words(uint32_t cap) { return size_t(cap + kScanTile - 1) / kScanTile + 1; }
// Two arrays of the same length n (in one pass of three launches); `partials` needs
// 2 * scan_partials_words(cap) words.
int scan_exclusive_u32x2(const uint32_t* in0, uint32_t* out0, uint32_t* total0, const uint32_t* in1, uint32_t* out1,
                         uint32_t* total1, const uint32_t* n_dev, uint32_t cap, uint32_t* partials, cudaStream_t st);

// Programmatic dependent launch.  A kernel started with launch_dependent() may be scheduled
// while the kernel before it in the stream is still running, which hides the launch gap of
// chains of short kernels; it must call grid_dependency_wait() before it touches memory, which
// returns once the preceding grid has completed and its writes are visible.  For a kernel
// launched the ordinary way the wait returns at once.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                    Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace rtpg
