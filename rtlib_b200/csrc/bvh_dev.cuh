// Triangle BVH for closest-hit / any-hit queries (the part RTLib delegates to OptiX:
// TraceRadiance / TraceOccluded, SimpleKernel.h:347-366).  A linear BVH: 63-bit Morton codes
// of the triangle centroids, radix-sorted, hierarchy by Karras' split search, boxes by a
// bottom-up pass.  Each interior node stores both children's boxes (64 bytes, two sectors),
// so a traversal step fetches one node and tests two boxes.
#pragma once
#include "common.cuh"

namespace rtpg {

constexpr uint32_t kBvhLeafBit = 0x80000000u;
constexpr int kBvhStack = 64;

struct __align__(16) BvhNode {
    float4 a;  // c0.lo.xyz, c0.hi.x
    float4 b;  // c0.hi.yz, c1.lo.xy
    float4 c;  // c1.lo.z, c1.hi.xyz
    uint32_t child[2];  // kBvhLeafBit | leaf index, or interior node index
    uint32_t pad[2];
};

struct __align__(16) BvhTri {
    float4 v0;  // xyz + original primitive index (as bits) in w
    float4 e1;  // v1 - v0
    float4 e2;  // v2 - v0
};

// Scenes of at most kFlatTris triangles are also kept as a flat list in their own order and
// traced by testing every triangle: all lanes of a warp then run the same loop over the same
// triangle (one broadcast load per triangle), where the BVH walk leaves most lanes idle, and the
// lowest index wins a tie of equal distances, as in a brute-force test.
constexpr uint32_t kFlatTris = 64;

struct SceneDev {
    const BvhNode* nodes;  // n - 1 interior nodes (root 0); n == 1: no interior node
    const BvhTri* tris;    // n triangles in leaf order
    const BvhTri* flat;    // n <= kFlatTris: the triangles in scene order, else null
    uint32_t ntris;
};

struct Hit {
    float t, u, v;
    uint32_t prim;  // 0xffffffff: miss
};

// Slab test with the ray's origin pre-scaled (oix = ox * ix, ...): each slab distance is one
// fused multiply-add, lo * ix - ox * ix with a single rounding.  Box tests only prune the
// traversal (the hit itself comes from tri_hit), so this arithmetic need not follow the
// oracle's rounding, which intersects triangles by brute force.
__device__ __forceinline__ bool box_hit(float lox, float loy, float loz, float hix, float hiy, float hiz, float oix,
                                        float oiy, float oiz, float ix, float iy, float iz, float tmin, float tmax,
                                        float& tnear) {
    const float tx0 = __fmaf_rn(lox, ix, -oix), tx1 = __fmaf_rn(hix, ix, -oix);
    const float ty0 = __fmaf_rn(loy, iy, -oiy), ty1 = __fmaf_rn(hiy, iy, -oiy);
    const float tz0 = __fmaf_rn(loz, iz, -oiz), tz1 = __fmaf_rn(hiz, iz, -oiz);
    const float t0 = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    const float t1 = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    tnear = t0;
    return t0 <= t1;
}

// Moller-Trumbore; returns t in (tmin, tmax) or a negative value
__device__ __forceinline__ float tri_hit(const BvhTri& tr, float ox, float oy, float oz, float dx, float dy, float dz,
                                         float tmin, float tmax, float& u, float& v) {
    const float px = dy * tr.e2.z - dz * tr.e2.y;
    const float py = dz * tr.e2.x - dx * tr.e2.z;
    const float pz = dx * tr.e2.y - dy * tr.e2.x;
    const float det = tr.e1.x * px + tr.e1.y * py + tr.e1.z * pz;
    if (fabsf(det) < 1e-20f) return -1.0f;
    const float inv = __frcp_rn(det);  // the correctly rounded 1 / det, without a full division
    const float sx = ox - tr.v0.x, sy = oy - tr.v0.y, sz = oz - tr.v0.z;
    u = (sx * px + sy * py + sz * pz) * inv;
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const float qx = sy * tr.e1.z - sz * tr.e1.y;
    const float qy = sz * tr.e1.x - sx * tr.e1.z;
    const float qz = sx * tr.e1.y - sy * tr.e1.x;
    v = (dx * qx + dy * qy + dz * qz) * inv;
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = (tr.e2.x * qx + tr.e2.y * qy + tr.e2.z * qz) * inv;
    return (t > tmin && t < tmax) ? t : -1.0f;
}

// closest hit (ANY = false) or any hit (ANY = true) in (tmin, tmax) by testing every triangle
// of a small scene, in scene order
template <bool ANY>
__device__ __forceinline__ Hit flat_trace(const SceneDev& s, float ox, float oy, float oz, float dx, float dy, float dz,
                                          float tmin, float tmax) {
    Hit h;
    h.t = tmax;
    h.prim = 0xffffffffu;
    h.u = h.v = 0.0f;
    // unrolled so that the next triangles' loads issue while this one is tested; the hit is
    // still updated in scene order
#pragma unroll 4
    for (uint32_t k = 0; k < s.ntris; ++k) {
        const BvhTri tr = s.flat[k];
        float u, v;
        const float t = tri_hit(tr, ox, oy, oz, dx, dy, dz, tmin, h.t, u, v);
        if (t > 0.0f) {
            h.t = t;
            h.u = u;
            h.v = v;
            h.prim = k;
            if (ANY) return h;
        }
    }
    return h;
}

// closest hit (ANY = false) or any hit (ANY = true) in (tmin, tmax)
template <bool ANY>
__device__ __forceinline__ Hit bvh_trace(const SceneDev& s, float ox, float oy, float oz, float dx, float dy, float dz,
                                         float tmin, float tmax) {
    if (s.flat) return flat_trace<ANY>(s, ox, oy, oz, dx, dy, dz, tmin, tmax);
    Hit h;
    h.t = tmax;
    h.prim = 0xffffffffu;
    h.u = h.v = 0.0f;
    const float ix = 1.0f / (fabsf(dx) > 1e-30f ? dx : copysignf(1e-30f, dx));
    const float iy = 1.0f / (fabsf(dy) > 1e-30f ? dy : copysignf(1e-30f, dy));
    const float iz = 1.0f / (fabsf(dz) > 1e-30f ? dz : copysignf(1e-30f, dz));
    if (s.ntris == 0) return h;
    const float oix = ox * ix, oiy = oy * iy, oiz = oz * iz;
    uint32_t stack[kBvhStack];
    int sp = 0;
    uint32_t cur = s.ntris == 1 ? kBvhLeafBit : 0u;
    for (;;) {
        if (cur & kBvhLeafBit) {
            const uint32_t li = cur & ~kBvhLeafBit;
            const BvhTri tr = s.tris[li];
            float u, v;
            const float t = tri_hit(tr, ox, oy, oz, dx, dy, dz, tmin, h.t, u, v);
            if (t > 0.0f) {
                h.t = t;
                h.u = u;
                h.v = v;
                h.prim = __float_as_uint(tr.v0.w);
                if (ANY) return h;
            }
        } else {
            const BvhNode nd = s.nodes[cur];
            float t0, t1;
            const bool h0 = box_hit(nd.a.x, nd.a.y, nd.a.z, nd.a.w, nd.b.x, nd.b.y, oix, oiy, oiz, ix, iy, iz, tmin, h.t, t0);
            const bool h1 = box_hit(nd.b.z, nd.b.w, nd.c.x, nd.c.y, nd.c.z, nd.c.w, oix, oiy, oiz, ix, iy, iz, tmin, h.t, t1);
            if (h0 && h1) {
                const bool first0 = t0 <= t1;
                const uint32_t near = first0 ? nd.child[0] : nd.child[1];
                const uint32_t far = first0 ? nd.child[1] : nd.child[0];
                if (sp < kBvhStack) stack[sp++] = far;
                cur = near;
                continue;
            }
            if (h0) { cur = nd.child[0]; continue; }
            if (h1) { cur = nd.child[1]; continue; }
        }
        if (sp == 0) break;
        cur = stack[--sp];
    }
    return h;
}

}  // namespace rtpg
