// Device-side hash-grid routines shared by the hash-grid kernels and the tracer.
#pragma once
#include "common.cuh"
#include "limits.cuh"

namespace rtpg {

struct HashGridDev {
    float3 off, size;
    uint3 bounds;
    uint32_t nslots, nbuckets;
    int32_t keying;
    unsigned long long* cur;  // slots (key 0 = empty)
    unsigned long long* prv;
    unsigned* status;
};

// cell of DoubleBufferedHashGrid3T::FindFromCur/Prv (OPX7UtilsGrid.h:189-199, 228-237):
// uint(bounds * (p - off) / size) clamped to bounds - 1; the float-to-unsigned conversion
// saturates (negative -> 0), which is the device semantics of the reference.
__device__ __forceinline__ void hash_cell(const HashGridDev& g, float px, float py, float pz, uint32_t* c) {
    const float f[3] = {__fdiv_rn(__fsub_rn(px, g.off.x), g.size.x), __fdiv_rn(__fsub_rn(py, g.off.y), g.size.y),
                        __fdiv_rn(__fsub_rn(pz, g.off.z), g.size.z)};
    const uint32_t b[3] = {g.bounds.x, g.bounds.y, g.bounds.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t v = __float2uint_rz(__fmul_rn((float)b[k], f[k]));
        c[k] = v > b[k] - 1 ? b[k] - 1 : v;
    }
}

__device__ __forceinline__ unsigned long long part1by2_21(unsigned long long x) {
    x &= 0x1fffffull;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
__device__ __forceinline__ unsigned long long morton3_63(uint32_t x, uint32_t y, uint32_t z) {
    return part1by2_21(x) | (part1by2_21(y) << 1) | (part1by2_21(z) << 2);
}
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// key and bucket of a position.  Reference keying: DoubleBufferedHashGrid3T::Hash1 and the
// checksum of GetCurCellIndex (OPX7UtilsGrid.h:241-252).
__device__ __forceinline__ unsigned long long hash_key(const HashGridDev& g, float px, float py, float pz,
                                                       uint32_t& bucket) {
    uint32_t c[3];
    hash_cell(g, px, py, pz, c);
    if (g.keying == RTPG_HASH_KEY_REFERENCE) {
        bucket = pcg1d(g.nslots + c[2] + pcg1d(c[1] + pcg1d(c[0]))) % g.nbuckets;
        return (unsigned long long)(1u + g.bounds.x * g.bounds.y * c[2] + g.bounds.x * c[1] + c[0]);
    }
    const unsigned long long key = morton3_63(c[0], c[1], c[2]) + 1ull;
    bucket = (uint32_t)(mix64(key) % g.nbuckets);
    return key;
}

// FindFromPrv (OPX7UtilsGrid.h:278-300): probe the previous snapshot, stop at the first empty
// slot; UINT32_MAX when absent.
__device__ __forceinline__ uint32_t hash_find_prv_key(const HashGridDev& g, unsigned long long key, uint32_t b) {
    const unsigned long long* row = g.prv + size_t(b) * kHashBlock;
    for (uint32_t k = 0; k < kHashBlock; ++k) {
        const unsigned long long v = row[k];
        if (v == 0ull) return 0xffffffffu;
        if (v == key) return b * kHashBlock + k;
    }
    return 0xffffffffu;
}
__device__ __forceinline__ uint32_t hash_find_prv(const HashGridDev& g, float px, float py, float pz) {
    uint32_t b;
    const unsigned long long key = hash_key(g, px, py, pz, b);
    return hash_find_prv_key(g, key, b);
}

// FindFromCur (OPX7UtilsGrid.h:189-226): claim the first empty slot of the bucket with a
// compare-and-swap or find the key already there; slots only ever go from empty to a key,
// so the occupied slots of a bucket stay a prefix and lookups may stop at the first empty
// one.  A full bucket returns UINT32_MAX and raises RTPG_STATUS_HASH_FULL.
__device__ __forceinline__ uint32_t hash_insert_cur_key(const HashGridDev& g, unsigned long long key, uint32_t b) {
    unsigned long long* row = g.cur + size_t(b) * kHashBlock;
    for (uint32_t k = 0; k < kHashBlock; ++k) {
        const unsigned long long old = atomicCAS(row + k, 0ull, key);
        if (old == 0ull || old == key) return b * kHashBlock + k;
    }
    atomicOr(g.status, RTPG_STATUS_HASH_FULL);
    return 0xffffffffu;
}

}  // namespace rtpg
