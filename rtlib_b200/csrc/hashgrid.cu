// Double-buffered spatial hash grid (RTLib's DoubleBufferedHashGrid3T, OPX7UtilsGrid.h:157-353,
// and its host buffer DoubleBufferedHashGrid3Buffer, RTLibExtOPX7Test.h:1472-1570).
//
// Cell (ix,iy,iz) = clamp(uint(bounds * (p - off) / size), 0, bounds - 1).  Two keyings:
//   RTPG_HASH_KEY_REFERENCE: bucket = pcg1d(size + iz + pcg1d(iy + pcg1d(ix))) % (slots / 32),
//       key = 1 + bx*by*iz + bx*iy + ix (uint32, RTLib's checksum);
//   RTPG_HASH_KEY_MORTON: key = morton63(ix, iy, iz) + 1 (21 bits per axis),
//       bucket = splitmix64(key) % (slots / 32).
// Each bucket holds 32 slots filled front to back; a key's slot is found by linear probing.
//
// RTLib inserts with atomicCAS, so which key wins which slot depends on thread timing.  Here
// a batch insert reproduces the slots of inserting the batch sequentially in index order:
// new keys are sorted (stable radix sort), each distinct key takes its first occurrence, the
// keys of a bucket are ranked by first occurrence and appended after the bucket's occupied
// prefix.  Lookups (FindFromPrv) read the previous snapshot and stop at the first empty slot.
#include <cub/cub.cuh>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "limits.cuh"
#include "hashgrid_dev.cuh"

namespace rtpg {

constexpr uint32_t kFull = 0xffffffffu;

__global__ void k_hash_prepare(HashGridDev g, int64_t base, int64_t n, const float* __restrict__ pos,
                               unsigned long long* __restrict__ skey, uint32_t* __restrict__ sval,
                               uint32_t* __restrict__ bucket_of, uint8_t* __restrict__ occ_of,
                               uint32_t* __restrict__ out_slot, unsigned long long* __restrict__ out_key) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = base + j;
        uint32_t b;
        const unsigned long long key = hash_key(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], b);
        if (out_key) out_key[i] = key;
        const unsigned long long* row = g.cur + size_t(b) * kHashBlock;
        uint32_t k = 0;
        bool found = false;
        for (; k < kHashBlock; ++k) {
            const unsigned long long v = row[k];
            if (v == 0ull) break;
            if (v == key) { found = true; break; }
        }
        bucket_of[j] = b;
        occ_of[j] = (uint8_t)k;
        if (found) {
            out_slot[i] = b * kHashBlock + k;
            skey[j] = ~0ull;
        } else {
            skey[j] = key;
        }
        sval[j] = (uint32_t)j;
    }
}

// run heads of the key-sorted batch: composite (bucket << 32 | first index) for ranking
__global__ void k_hash_heads(int64_t n, const unsigned long long* __restrict__ key_sorted,
                             const uint32_t* __restrict__ val_sorted, const uint32_t* __restrict__ bucket_of,
                             unsigned long long* __restrict__ comp, uint32_t* __restrict__ comp_val) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        const unsigned long long k = key_sorted[p];
        const bool head = k != ~0ull && (p == 0 || key_sorted[p - 1] != k);
        const uint32_t j = val_sorted[p];
        comp[p] = head ? ((unsigned long long)bucket_of[j] << 32) | j : ~0ull;
        comp_val[p] = (uint32_t)p;
    }
}

__device__ __forceinline__ int64_t lower_bound_u64(const unsigned long long* a, int64_t n, unsigned long long x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (a[m] < x) lo = m + 1;
        else hi = m;
    }
    return lo;
}

// rank of each distinct new key among the bucket's new keys (by first occurrence) -> slot
__global__ void k_hash_assign(HashGridDev g, int64_t n, const unsigned long long* __restrict__ comp_sorted,
                              const uint32_t* __restrict__ comp_val_sorted, const unsigned long long* __restrict__ key_sorted,
                              const uint8_t* __restrict__ occ_of, uint32_t* __restrict__ run_slot) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n; r += int64_t(gridDim.x) * blockDim.x) {
        const unsigned long long c = comp_sorted[r];
        if (c == ~0ull) continue;
        const uint32_t b = uint32_t(c >> 32), j = uint32_t(c & 0xffffffffu);
        const int64_t start = lower_bound_u64(comp_sorted, n, (unsigned long long)b << 32);
        const uint32_t slot_in_bucket = occ_of[j] + uint32_t(r - start);
        const uint32_t p = comp_val_sorted[r];
        if (slot_in_bucket < kHashBlock) {
            const uint32_t slot = b * kHashBlock + slot_in_bucket;
            g.cur[slot] = key_sorted[p];
            run_slot[p] = slot;
        } else {
            run_slot[p] = kFull;
            atomicOr(g.status, RTPG_STATUS_HASH_FULL);
        }
    }
}

__global__ void k_hash_scatter(int64_t base, int64_t n, const unsigned long long* __restrict__ key_sorted,
                               const uint32_t* __restrict__ val_sorted, const uint32_t* __restrict__ run_slot,
                               uint32_t* __restrict__ out_slot) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n; p += int64_t(gridDim.x) * blockDim.x) {
        const unsigned long long k = key_sorted[p];
        if (k == ~0ull) continue;
        const int64_t h = lower_bound_u64(key_sorted, n, k);
        out_slot[base + val_sorted[p]] = run_slot[h];
    }
}

__global__ void k_hash_lookup(HashGridDev g, int64_t n, const float* __restrict__ pos, uint32_t* __restrict__ out_slot) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out_slot[i] = hash_find_prv(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
}

__global__ void k_hash_cells(HashGridDev g, int64_t n, const float* __restrict__ pos, uint32_t* __restrict__ out_cell,
                             unsigned long long* __restrict__ out_key) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        uint32_t c[3];
        hash_cell(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], c);
        if (out_cell) {
            out_cell[3 * i] = c[0];
            out_cell[3 * i + 1] = c[1];
            out_cell[3 * i + 2] = c[2];
        }
        if (out_key) {
            uint32_t b;
            out_key[i] = hash_key(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], b);
        }
    }
}

}  // namespace rtpg

using namespace rtpg;

struct rtpg_hashgrid {
    HashGridDev dev{};
    uint32_t max_batch = 0;
    unsigned long long *skey[2] = {nullptr, nullptr}, *comp[2] = {nullptr, nullptr};
    uint32_t *sval[2] = {nullptr, nullptr}, *cval[2] = {nullptr, nullptr};
    uint32_t *bucket_of = nullptr, *run_slot = nullptr;
    uint8_t* occ_of = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
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
    ~rtpg_hashgrid() {
        for (void* p : allocs) cudaFree(p);
    }
};

extern "C" {

int rtpg_hashgrid_create(const float* aabb_min, const float* aabb_max, const uint32_t* bounds, uint32_t num_slots,
                         int32_t keying, uint32_t max_batch, rtpg_hashgrid** out) {
    if (!aabb_min || !aabb_max || !bounds || !out) return fail(RTPG_EINVAL, "rtpg_hashgrid_create: null argument");
    if (num_slots < kHashBlock || num_slots % kHashBlock)
        return fail(RTPG_EINVAL, "rtpg_hashgrid_create: num_slots must be a positive multiple of %u", kHashBlock);
    if (keying != RTPG_HASH_KEY_REFERENCE && keying != RTPG_HASH_KEY_MORTON)
        return fail(RTPG_EINVAL, "rtpg_hashgrid_create: unknown keying %d", keying);
    for (int k = 0; k < 3; ++k) {
        if (bounds[k] == 0) return fail(RTPG_EINVAL, "rtpg_hashgrid_create: zero bound");
        if (keying == RTPG_HASH_KEY_MORTON && bounds[k] > (1u << 21))
            return fail(RTPG_EINVAL, "rtpg_hashgrid_create: Morton keying supports at most 2^21 cells per axis");
        if (!(aabb_max[k] > aabb_min[k])) return fail(RTPG_EINVAL, "rtpg_hashgrid_create: empty AABB");
    }
    auto* h = new (std::nothrow) rtpg_hashgrid();
    if (!h) return fail(RTPG_ENOMEM, "rtpg_hashgrid_create: out of host memory");
    HashGridDev& g = h->dev;
    // DoubleBufferedHashGrid3Buffer::GetHandle (RTLibExtOPX7Test.h:1561-1568)
    g.off = make_float3(aabb_min[0], aabb_min[1], aabb_min[2]);
    g.size = make_float3(aabb_max[0] - aabb_min[0], aabb_max[1] - aabb_min[1], aabb_max[2] - aabb_min[2]);
    g.bounds = make_uint3(bounds[0], bounds[1], bounds[2]);
    g.nslots = num_slots;
    g.nbuckets = num_slots / kHashBlock;
    g.keying = keying;
    h->max_batch = max_batch ? max_batch : (1u << 22);
    const size_t B = h->max_batch;
    int r;
    if ((r = h->alloc(&g.cur, num_slots)) || (r = h->alloc(&g.prv, num_slots)) || (r = h->alloc(&g.status, 1)) ||
        (r = h->alloc(&h->skey[0], B)) || (r = h->alloc(&h->skey[1], B)) || (r = h->alloc(&h->comp[0], B)) ||
        (r = h->alloc(&h->comp[1], B)) || (r = h->alloc(&h->sval[0], B)) || (r = h->alloc(&h->sval[1], B)) ||
        (r = h->alloc(&h->cval[0], B)) || (r = h->alloc(&h->cval[1], B)) || (r = h->alloc(&h->bucket_of, B)) ||
        (r = h->alloc(&h->run_slot, B)) || (r = h->alloc(&h->occ_of, B))) {
        delete h;
        return r;
    }
    cub::DoubleBuffer<unsigned long long> dk(h->skey[0], h->skey[1]);
    cub::DoubleBuffer<uint32_t> dv(h->sval[0], h->sval[1]);
    size_t tb = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)B);
    if (e != cudaSuccess || (r = h->alloc(reinterpret_cast<uint8_t**>(&h->temp), tb))) {
        delete h;
        return e != cudaSuccess ? fail(RTPG_ECUDA, "cub temp size: %s", cudaGetErrorString(e)) : r;
    }
    h->temp_bytes = tb;
    if (cudaMemset(g.cur, 0, num_slots * 8ull) != cudaSuccess || cudaMemset(g.prv, 0, num_slots * 8ull) != cudaSuccess ||
        cudaMemset(g.status, 0, 4) != cudaSuccess) {
        delete h;
        return fail(RTPG_ECUDA, "rtpg_hashgrid_create: memset failed");
    }
    *out = h;
    return RTPG_OK;
}

int rtpg_hashgrid_destroy(rtpg_hashgrid* h) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_destroy: null handle");
    delete h;
    return RTPG_OK;
}

// DoubleBufferedHashGrid3Buffer::Clear (RTLibExtOPX7Test.h:1529-1543)
int rtpg_hashgrid_clear(rtpg_hashgrid* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_clear: null handle");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemsetAsync(h->dev.cur, 0, h->dev.nslots * 8ull, st));
    RTPG_CUDA(cudaMemsetAsync(h->dev.prv, 0, h->dev.nslots * 8ull, st));
    RTPG_CUDA(cudaMemsetAsync(h->dev.status, 0, 4, st));
    return RTPG_OK;
}

// DoubleBufferedHashGrid3Buffer::Update (RTLibExtOPX7Test.h:1544-1559): the previous table
// becomes a copy of the current one; the current table keeps its keys.
int rtpg_hashgrid_swap(rtpg_hashgrid* h, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_swap: null handle");
    RTPG_CUDA(cudaMemcpyAsync(h->dev.prv, h->dev.cur, h->dev.nslots * 8ull, cudaMemcpyDeviceToDevice, as_stream(stream)));
    return RTPG_OK;
}

int rtpg_hashgrid_insert(rtpg_hashgrid* h, int64_t n, const float* pos, uint32_t* out_slot, uint64_t* out_key,
                         void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_insert: null handle");
    if (n < 0 || (n > 0 && (!pos || !out_slot))) return fail(RTPG_EINVAL, "rtpg_hashgrid_insert: bad arguments");
    cudaStream_t st = as_stream(stream);
    // chunks are inserted in order, which keeps the sequential-insertion semantics
    for (int64_t base = 0; base < n; base += h->max_batch) {
        const int64_t m = std::min<int64_t>(h->max_batch, n - base);
        const int g = grid_for(m, 256, 8);
        k_hash_prepare<<<g, 256, 0, st>>>(h->dev, base, m, pos, h->skey[0], h->sval[0], h->bucket_of, h->occ_of,
                                           out_slot, reinterpret_cast<unsigned long long*>(out_key));
        RTPG_LAUNCH_CHECK();
        cub::DoubleBuffer<unsigned long long> dk(h->skey[0], h->skey[1]);
        cub::DoubleBuffer<uint32_t> dv(h->sval[0], h->sval[1]);
        size_t tb = h->temp_bytes;
        RTPG_CUDA(cub::DeviceRadixSort::SortPairs(h->temp, tb, dk, dv, (int)m, 0, 64, st));
        k_hash_heads<<<g, 256, 0, st>>>(m, dk.Current(), dv.Current(), h->bucket_of, h->comp[0], h->cval[0]);
        RTPG_LAUNCH_CHECK();
        cub::DoubleBuffer<unsigned long long> ck(h->comp[0], h->comp[1]);
        cub::DoubleBuffer<uint32_t> cv(h->cval[0], h->cval[1]);
        tb = h->temp_bytes;
        RTPG_CUDA(cub::DeviceRadixSort::SortPairs(h->temp, tb, ck, cv, (int)m, 0, 64, st));
        k_hash_assign<<<g, 256, 0, st>>>(h->dev, m, ck.Current(), cv.Current(), dk.Current(), h->occ_of, h->run_slot);
        k_hash_scatter<<<g, 256, 0, st>>>(base, m, dk.Current(), dv.Current(), h->run_slot, out_slot);
        RTPG_LAUNCH_CHECK();
    }
    return RTPG_OK;
}

int rtpg_hashgrid_lookup(rtpg_hashgrid* h, int64_t n, const float* pos, uint32_t* out_slot, void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_lookup: null handle");
    if (n < 0 || (n > 0 && (!pos || !out_slot))) return fail(RTPG_EINVAL, "rtpg_hashgrid_lookup: bad arguments");
    if (n == 0) return RTPG_OK;
    k_hash_lookup<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(h->dev, n, pos, out_slot);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_hashgrid_cells(rtpg_hashgrid* h, int64_t n, const float* pos, uint32_t* out_cell_xyz, uint64_t* out_key,
                        void* stream) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_cells: null handle");
    if (n < 0 || (n > 0 && !pos)) return fail(RTPG_EINVAL, "rtpg_hashgrid_cells: bad arguments");
    if (n == 0) return RTPG_OK;
    k_hash_cells<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(h->dev, n, pos, out_cell_xyz,
                                                                     reinterpret_cast<unsigned long long*>(out_key));
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}

int rtpg_hashgrid_export(rtpg_hashgrid* h, int previous, uint64_t* host_table, void* stream) {
    if (!h || !host_table) return fail(RTPG_EINVAL, "rtpg_hashgrid_export: null argument");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemcpyAsync(host_table, previous ? h->dev.prv : h->dev.cur, h->dev.nslots * 8ull,
                              cudaMemcpyDeviceToHost, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

int rtpg_hashgrid_status(rtpg_hashgrid* h, uint32_t* host_status, int clear, void* stream) {
    if (!h || !host_status) return fail(RTPG_EINVAL, "rtpg_hashgrid_status: null argument");
    cudaStream_t st = as_stream(stream);
    RTPG_CUDA(cudaMemcpyAsync(host_status, h->dev.status, 4, cudaMemcpyDeviceToHost, st));
    if (clear) RTPG_CUDA(cudaMemsetAsync(h->dev.status, 0, 4, st));
    RTPG_CUDA(cudaStreamSynchronize(st));
    return RTPG_OK;
}

int rtpg_hashgrid_device_view(rtpg_hashgrid* h, void** dev_cur, void** dev_prv) {
    if (!h) return fail(RTPG_EINVAL, "rtpg_hashgrid_device_view: null handle");
    if (dev_cur) *dev_cur = h->dev.cur;
    if (dev_prv) *dev_prv = h->dev.prv;
    return RTPG_OK;
}

}  // extern "C"

namespace rtpg {
HashGridDev hashgrid_device_view(const rtpg_hashgrid* h) { return h->dev; }
}

// ================================================================ allocation-free insert
// The batch insert above keeps its sort buffers in the handle, allocated by
// rtpg_hashgrid_create.  Some callers cannot allocate device memory at all: a renderer or
// simulation that hands this library a fixed memory budget and owns every allocation, code
// that enqueues work while another component captures the stream into a CUDA graph (where
// cudaMalloc is not allowed), or a real-time loop that must never block in the allocator.
// rtpg_hashgrid_insert_noalloc serves them: the caller passes the table and the outputs, and
// the scratch lives in one file-scope device array of fixed size, reserved in every GPU's
// memory when the library loads and held until the process exits.
namespace rtpg {

constexpr uint32_t kNoAllocMaxPoints = 1u << 16;  // points per call
constexpr size_t kNoAllocSortBytes = size_t(4) << 20;  // radix-sort temporary storage
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kNA_skey = 0;
constexpr size_t kNA_sval = kNA_skey + align256(2ull * 8 * kNoAllocMaxPoints);
constexpr size_t kNA_comp = kNA_sval + align256(2ull * 4 * kNoAllocMaxPoints);
constexpr size_t kNA_cval = kNA_comp + align256(2ull * 8 * kNoAllocMaxPoints);
constexpr size_t kNA_bucket = kNA_cval + align256(2ull * 4 * kNoAllocMaxPoints);
constexpr size_t kNA_run = kNA_bucket + align256(4ull * kNoAllocMaxPoints);
constexpr size_t kNA_occ = kNA_run + align256(4ull * kNoAllocMaxPoints);
constexpr size_t kNA_status = kNA_occ + align256(kNoAllocMaxPoints);
constexpr size_t kNA_temp = kNA_status + 256;
constexpr size_t kNoAllocScratchBytes = kNA_temp + kNoAllocSortBytes;  // about 7.8 MB

static __device__ __align__(256) unsigned char g_insert_scratch[kNoAllocScratchBytes];

// Device address of g_insert_scratch per device, looked up once per device with that device
// current (host code cannot use the symbol itself as a device address).
static std::mutex g_na_mutex;
static unsigned char* g_na_ptr[64] = {};

static int noalloc_scratch(unsigned char** out) {
    int dev = 0;
    RTPG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_insert_scratch);
        if (e != cudaSuccess)
            return fail(RTPG_ECUDA, "rtpg_hashgrid_insert_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        // the sort's temporary storage for the largest batch must fit the reserved bytes
        cub::DoubleBuffer<unsigned long long> dk(nullptr, nullptr);
        cub::DoubleBuffer<uint32_t> dv(nullptr, nullptr);
        size_t tb = 0;
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)kNoAllocMaxPoints, 0, 64);
        if (e != cudaSuccess) return fail(RTPG_ECUDA, "rtpg_hashgrid_insert_noalloc: %s", cudaGetErrorString(e));
        if (tb > kNoAllocSortBytes)
            return fail(RTPG_ECAPACITY, "rtpg_hashgrid_insert_noalloc: sort needs %zu bytes, %zu reserved", tb,
                        kNoAllocSortBytes);
        g_na_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_na_ptr[dev];
    return RTPG_OK;
}

}  // namespace rtpg

extern "C" int rtpg_hashgrid_insert_noalloc(const float* aabb_min, const float* aabb_max, const uint32_t* bounds,
                                            uint32_t num_slots, int32_t keying, uint64_t* table, uint32_t* status,
                                            int64_t n, const float* pos, uint32_t* out_slot, void* stream) {
    if (!aabb_min || !aabb_max || !bounds || !table) return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: null argument");
    if (n < 0 || (n > 0 && (!pos || !out_slot))) return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: bad arguments");
    if (n > (int64_t)kNoAllocMaxPoints)
        return fail(RTPG_ECAPACITY, "rtpg_hashgrid_insert_noalloc: %lld points exceed the limit of %u per call",
                    (long long)n, kNoAllocMaxPoints);
    if (num_slots < kHashBlock || num_slots % kHashBlock)
        return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: num_slots must be a positive multiple of %u", kHashBlock);
    if (keying != RTPG_HASH_KEY_REFERENCE && keying != RTPG_HASH_KEY_MORTON)
        return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: unknown keying %d", keying);
    if (!aligned8(table) || !aligned4(pos) || !aligned4(out_slot) || (status && !aligned4(status)))
        return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: misaligned array");
    for (int k = 0; k < 3; ++k) {
        if (bounds[k] == 0 || !(aabb_max[k] > aabb_min[k]))
            return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: empty grid or AABB");
        if (keying == RTPG_HASH_KEY_MORTON && bounds[k] > (1u << 21))
            return fail(RTPG_EINVAL, "rtpg_hashgrid_insert_noalloc: Morton keying supports at most 2^21 cells per axis");
    }
    unsigned char* s = nullptr;
    int r = noalloc_scratch(&s);
    if (r) return r;
    if (n == 0) return RTPG_OK;
    HashGridDev g{};
    g.off = make_float3(aabb_min[0], aabb_min[1], aabb_min[2]);
    g.size = make_float3(aabb_max[0] - aabb_min[0], aabb_max[1] - aabb_min[1], aabb_max[2] - aabb_min[2]);
    g.bounds = make_uint3(bounds[0], bounds[1], bounds[2]);
    g.nslots = num_slots;
    g.nbuckets = num_slots / kHashBlock;
    g.keying = keying;
    g.cur = reinterpret_cast<unsigned long long*>(table);
    g.prv = nullptr;
    g.status = status ? reinterpret_cast<unsigned*>(status) : reinterpret_cast<unsigned*>(s + kNA_status);
    auto* skey = reinterpret_cast<unsigned long long*>(s + kNA_skey);
    auto* sval = reinterpret_cast<uint32_t*>(s + kNA_sval);
    auto* comp = reinterpret_cast<unsigned long long*>(s + kNA_comp);
    auto* cval = reinterpret_cast<uint32_t*>(s + kNA_cval);
    auto* bucket_of = reinterpret_cast<uint32_t*>(s + kNA_bucket);
    auto* run_slot = reinterpret_cast<uint32_t*>(s + kNA_run);
    auto* occ_of = reinterpret_cast<uint8_t*>(s + kNA_occ);
    void* temp = s + kNA_temp;
    // every scratch word read below is written earlier in the same call, so nothing left
    // by a previous call needs clearing
    cudaStream_t st = as_stream(stream);
    const int64_t m = n;
    const int grid = grid_for(m, 256, 8);
    k_hash_prepare<<<grid, 256, 0, st>>>(g, 0, m, pos, skey, sval, bucket_of, occ_of, out_slot, nullptr);
    RTPG_LAUNCH_CHECK();
    cub::DoubleBuffer<unsigned long long> dk(skey, skey + kNoAllocMaxPoints);
    cub::DoubleBuffer<uint32_t> dv(sval, sval + kNoAllocMaxPoints);
    size_t tb = kNoAllocSortBytes;
    RTPG_CUDA(cub::DeviceRadixSort::SortPairs(temp, tb, dk, dv, (int)m, 0, 64, st));
    k_hash_heads<<<grid, 256, 0, st>>>(m, dk.Current(), dv.Current(), bucket_of, comp, cval);
    RTPG_LAUNCH_CHECK();
    cub::DoubleBuffer<unsigned long long> ck(comp, comp + kNoAllocMaxPoints);
    cub::DoubleBuffer<uint32_t> cv(cval, cval + kNoAllocMaxPoints);
    tb = kNoAllocSortBytes;
    RTPG_CUDA(cub::DeviceRadixSort::SortPairs(temp, tb, ck, cv, (int)m, 0, 64, st));
    k_hash_assign<<<grid, 256, 0, st>>>(g, m, ck.Current(), cv.Current(), dk.Current(), occ_of, run_slot);
    k_hash_scatter<<<grid, 256, 0, st>>>(0, m, dk.Current(), dv.Current(), run_slot, out_slot);
    RTPG_LAUNCH_CHECK();
    return RTPG_OK;
}
