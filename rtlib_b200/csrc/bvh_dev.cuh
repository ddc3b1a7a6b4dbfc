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

// A triangle as the affine map of world space onto its own frame (Baldwin and Weber, "Fast
// Ray-Triangle Intersections by Coordinate Transformation", JCGT 5(3), 2016): a point x has
// barycentric coordinates u = dot(r0.xyz, x) + r0.w and v = dot(r1.xyz, x) + r1.w, and
// dot(r2.xyz, x) + r2.w is its offset along the face normal in units of the normal's length.
// tri_transform forms the rows in double precision from the vertices, once per scene.
struct __align__(16) BvhTri {
    float4 r0, r1, r2;
};

// The rows of triangle (a, b, c): with e1 = b - a, e2 = c - a, n = e1 x e2, the inverse of the
// matrix [e1 e2 n] is [e2 x n; n x e1; n] / |n|^2, translated by -a.  Every operation is a
// double operation rounded as written (the file is built without contraction), then the rows
// are rounded to float: the CPU restatement forms them the same way, bit for bit.
__host__ __device__ inline void tri_transform(float ax_, float ay_, float az_, float bx_, float by_, float bz_, float cx_,
                                              float cy_, float cz_, float4* r) {
    const double ax = ax_, ay = ay_, az = az_;
    const double e1x = (double)bx_ - ax, e1y = (double)by_ - ay, e1z = (double)bz_ - az;
    const double e2x = (double)cx_ - ax, e2y = (double)cy_ - ay, e2z = (double)cz_ - az;
    const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const double nn = nx * nx + ny * ny + nz * nz;
    const double m[3][3] = {{e2y * nz - e2z * ny, e2z * nx - e2x * nz, e2x * ny - e2y * nx},
                            {ny * e1z - nz * e1y, nz * e1x - nx * e1z, nx * e1y - ny * e1x},
                            {nx, ny, nz}};
    for (int k = 0; k < 3; ++k) {
        const double w = -(m[k][0] * ax + m[k][1] * ay + m[k][2] * az);
        r[k] = make_float4((float)(m[k][0] / nn), (float)(m[k][1] / nn), (float)(m[k][2] / nn), (float)(w / nn));
    }
}

// Scenes of at most kFlatTris triangles are also kept as a flat list in their own order and
// traced by testing every triangle: all lanes of a warp then run the same loop over the same
// triangle (one broadcast load per triangle), where the BVH walk leaves most lanes idle, and the
// lowest index wins a tie of equal distances, as in a brute-force test.
constexpr uint32_t kFlatTris = 64;

struct SceneDev {
    const BvhNode* nodes;  // n - 1 interior nodes (root 0); n == 1: no interior node
    const BvhTri* tris;    // n triangles in leaf order
    const uint32_t* prim;  // scene index of each leaf
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

// The hit of ray o + t d on triangle tr: the ray meets the triangle's plane at
// t = -(dot(r2.xyz, o) + r2.w) / dot(r2.xyz, d), where u and v follow as o's coordinates plus
// t times d's.  Each dot product is a chain of fused multiply-adds and 1 / den the correctly
// rounded reciprocal, so the CPU restatement (fmaf, 1.0f / den) reproduces every value; the
// test runs without a branch, as every lane of a warp tests the same triangle.  Returns t in
// (tmin, tmax) or a negative value (also for a ray parallel to the plane: t is then infinite
// or NaN).
__device__ __forceinline__ float tri_hit(const BvhTri& tr, float ox, float oy, float oz, float dx, float dy, float dz,
                                         float tmin, float tmax, float& u, float& v) {
    const float den = __fmaf_rn(tr.r2.x, dx, __fmaf_rn(tr.r2.y, dy, __fmul_rn(tr.r2.z, dz)));
    const float num = __fmaf_rn(tr.r2.x, ox, __fmaf_rn(tr.r2.y, oy, __fmaf_rn(tr.r2.z, oz, tr.r2.w)));
    const float t = __fmul_rn(-num, __frcp_rn(den));
    const float ud = __fmaf_rn(tr.r0.x, dx, __fmaf_rn(tr.r0.y, dy, __fmul_rn(tr.r0.z, dz)));
    const float uo = __fmaf_rn(tr.r0.x, ox, __fmaf_rn(tr.r0.y, oy, __fmaf_rn(tr.r0.z, oz, tr.r0.w)));
    const float vd = __fmaf_rn(tr.r1.x, dx, __fmaf_rn(tr.r1.y, dy, __fmul_rn(tr.r1.z, dz)));
    const float vo = __fmaf_rn(tr.r1.x, ox, __fmaf_rn(tr.r1.y, oy, __fmaf_rn(tr.r1.z, oz, tr.r1.w)));
    u = __fmaf_rn(t, ud, uo);
    v = __fmaf_rn(t, vd, vo);
    const bool hit = (t > tmin) & (t < tmax) & (u >= 0.0f) & (v >= 0.0f) & (__fadd_rn(u, v) <= 1.0f);
    return hit ? t : -1.0f;
}

// closest hit (ANY = false) or any hit (ANY = true) in (tmin, tmax) by testing every triangle
// of a small scene (tris[0, n), in scene order)
template <bool ANY>
__device__ __forceinline__ Hit flat_trace(const BvhTri* tris, uint32_t n, float ox, float oy, float oz, float dx,
                                          float dy, float dz, float tmin, float tmax) {
    Hit h;
    h.t = tmax;
    h.prim = 0xffffffffu;
    h.u = h.v = 0.0f;
    // unrolled so that the next triangles' loads issue while this one is tested; the hit is
    // still updated in scene order
#pragma unroll 4
    for (uint32_t k = 0; k < n; ++k) {
        const BvhTri tr = tris[k];
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
    if (s.flat) return flat_trace<ANY>(s.flat, s.ntris, ox, oy, oz, dx, dy, dz, tmin, tmax);
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
                h.prim = li;  // the leaf; its scene index is looked up once, at the end
                if (ANY) break;
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
    if (h.prim != 0xffffffffu) h.prim = s.prim[h.prim];
    return h;
}

}  // namespace rtpg
