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
__global__ void __launch_bounds__(kScanBlock) scan_tile_sums(const uint32_t* __restrict__ in, const uint32_t* n_dev,
                                                            uint32_t* __restrict__ partials) {
    grid_dependency_wait();
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

__global__ void __launch_bounds__(kScanBlock) scan_partials(uint32_t* partials, const uint32_t* n_dev, uint32_t* total_out) {
    grid_dependency_wait();
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

__global__ void __launch_bounds__(kScanBlock) scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                        const uint32_t* n_dev, const uint32_t* __restrict__ partials) {
    grid_dependency_wait();
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

int scan_exclusive_u32(const uint32_t* in, uint32_t* out, const uint32_t* n_dev, uint32_t cap, uint32_t* partials,
                       uint32_t* total_out, cudaStream_t st) {
    const uint32_t tiles = (cap + kScanTile - 1) / kScanTile;
    const uint32_t g = tiles ? tiles : 1;
    // launched as dependent grids: each may be scheduled while its predecessor finishes
    RTPG_CUDA(launch_dependent(scan_tile_sums, g, kScanBlock, 0, st, in, n_dev, partials));
    RTPG_CUDA(launch_dependent(scan_partials, 1, kScanBlock, 0, st, partials, n_dev, total_out));
    RTPG_CUDA(launch_dependent(scan_tiles, g, kScanBlock, 0, st, in, out, n_dev, partials));
    return RTPG_OK;
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
