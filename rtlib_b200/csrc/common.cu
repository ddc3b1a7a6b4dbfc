// Error plumbing, limits and the device-count-aware scan shared by the kernels.
#include "common.cuh"
#include "limits.cuh"

namespace rtpg {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// ---------------------------------------------------------------- scan
// Up to two arrays of the same device-side length per launch: blockIdx.y picks the array, each
// with its own region of `partials` (ceil(cap / kScanTile) + 1 words apart).
struct ScanPair {
    const uint32_t* in[2];
    uint32_t* out[2];
    uint32_t* total[2];
    uint32_t stride;  // words between the two partials regions
};

__global__ void __launch_bounds__(kScanBlock) scan_tile_sums(ScanPair a, const uint32_t* n_dev, uint32_t* partials) {
    grid_dependency_wait();
    const uint32_t y = blockIdx.y;
    const uint32_t* __restrict__ in = y ? a.in[1] : a.in[0];
    partials += y * a.stride;
    const uint32_t n = *n_dev;
    const uint32_t base = blockIdx.x * kScanTile;
    if (base >= n) return;
    uint32_t s = 0;
    for (uint32_t i = base + threadIdx.x; i < base + kScanTile && i < n; i += kScanBlock) s += in[i];
    s = __reduce_add_sync(0xffffffffu, s);
    __shared__ uint32_t ws[kScanBlock / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < kScanBlock / 32 ? ws[threadIdx.x] : 0u;
        v = __reduce_add_sync(0xffffffffu, v);
        if (threadIdx.x == 0) partials[blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(kScanBlock) scan_partials(ScanPair a, const uint32_t* n_dev, uint32_t* partials) {
    grid_dependency_wait();
    const uint32_t y = blockIdx.y;
    uint32_t* total_out = y ? a.total[1] : a.total[0];
    partials += y * a.stride;
    __shared__ uint32_t ws[kScanBlock / 32];
    const uint32_t n = *n_dev;
    const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    uint32_t carry = 0;
    for (uint32_t b = 0; b < tiles; b += kScanBlock) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < tiles ? partials[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<kScanBlock>(v, ws, tot);
        if (i < tiles) partials[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void __launch_bounds__(kScanBlock) scan_tiles(ScanPair a, const uint32_t* n_dev, const uint32_t* partials) {
    grid_dependency_wait();
    const uint32_t y = blockIdx.y;
    const uint32_t* __restrict__ in = y ? a.in[1] : a.in[0];
    uint32_t* __restrict__ out = y ? a.out[1] : a.out[0];
    partials += y * a.stride;
    __shared__ uint32_t ws[kScanBlock / 32];
    const uint32_t n = *n_dev;
    const uint32_t base = blockIdx.x * kScanTile;
    if (base >= n) return;
    // each thread owns 4 consecutive elements
    const uint32_t i0 = base + threadIdx.x * 4;
    uint32_t v[4];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = (i0 + k < n) ? in[i0 + k] : 0u;
        s += v[k];
    }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan<kScanBlock>(s, ws, tot) + partials[blockIdx.x];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (i0 + k < n) out[i0 + k] = ex;
        ex += v[k];
    }
}

static int scan_launch(const ScanPair& a, uint32_t arrays, const uint32_t* n_dev, uint32_t cap, uint32_t* partials,
                       cudaStream_t st) {
    const uint32_t tiles = (cap + kScanTile - 1) / kScanTile;
    const dim3 g(tiles ? tiles : 1, arrays);
    // launched as dependent grids: each may be scheduled while its predecessor finishes
    RTPG_CUDA(launch_dependent(scan_tile_sums, g, kScanBlock, 0, st, a, n_dev, partials));
    RTPG_CUDA(launch_dependent(scan_partials, dim3(1, arrays), kScanBlock, 0, st, a, n_dev, partials));
    RTPG_CUDA(launch_dependent(scan_tiles, g, kScanBlock, 0, st, a, n_dev, (const uint32_t*)partials));
    return RTPG_OK;
}

int scan_exclusive_u32(const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint32_t cap, uint32_t* partials,
                       uint32_t* total_out, cudaStream_t st) {
    const ScanPair a{{in, in}, {out, out}, {total_out, total_out}, 0};
    return scan_launch(a, 1, n_dev, cap, partials, st);
}

int scan_exclusive_u32x2(const uint32_t* in0, uint32_t* out0, uint32_t* total0, const uint32_t* in1, uint32_t* out1,
                         uint32_t* total1, const uint32_t* n_dev, uint32_t cap, uint32_t* partials, cudaStream_t st) {
    const ScanPair a{{in0, in1}, {out0, out1}, {total0, total1}, (uint32_t)scan_partials_words(cap)};
    return scan_launch(a, 2, n_dev, cap, partials, st);
}

}  // namespace rtpg

extern "C" {

const char* rtpg_last_error(void) { return rtpg::g_last_error.c_str(); }

int rtpg_version(void) { return 100; }

int rtpg_query_limits(uint32_t* dtree_node_cap, uint32_t* max_dtree_depth, uint32_t* hash_block) {
    if (dtree_node_cap) *dtree_node_cap = rtpg::kDTreeNodeCap;
    if (max_dtree_depth) *max_dtree_depth = rtpg::kMaxDTreeDepth;
    if (hash_block) *hash_block = rtpg::kHashBlock;
    return RTPG_OK;
}

}  // extern "C"
