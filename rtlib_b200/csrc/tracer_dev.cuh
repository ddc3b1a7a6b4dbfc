// Shading math of RTLib's closest-hit programs (SimpleGuide.cu / SimpleTrace.cu /
// SimpleKernel.h), shared by the wavefront kernels and the adjoint.
#pragma once
#include "common.cuh"
#include "canonical.cuh"

namespace rtpg {

// Hit-group types (SimpleKernel.h:232-239)
enum : int { MAT_PHONG = 0, MAT_GLASS = 1, MAT_NEE_LIGHT = 2, MAT_DEF_LIGHT = 3 };
// Hit-record flags (SimpleKernel.h:246-253)
enum : uint32_t { HF_MISS = 1, HF_DELTA = 2, HF_PHONG = 4, HF_COUNT_EMITTED = 8, HF_FINISH = 16 };

struct __align__(16) Material {
    float3 diffuse;
    int32_t tex;  // diffuse texture index, -1 = none
    float3 specular;
    float shininess;
    float3 emission;
    float ref_index;
    int32_t type;
    int32_t pad[3];
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float a, float3 b) { return f3(a * b.x, a * b.y, a * b.z); }
__device__ __forceinline__ float3 operator*(float3 b, float a) { return f3(a * b.x, a * b.y, a * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float b) { return f3(a.x / b, a.y / b, a.z / b); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 unit3(float3 a) { return a / len3(a); }
__device__ __forceinline__ float avg3(float3 a) { return (a.x + a.y + a.z) / 3.0f; }
__device__ __forceinline__ bool any_nan3(float3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }

// ONB (VectorFunction.h:5666-5697)
struct Onb {
    float3 t, b, n;
    __device__ __forceinline__ explicit Onb(float3 normal) {
        n = unit3(normal);
        if (fabsf(n.x) > fabsf(n.z)) b = f3(-n.y, n.x, 0.0f);
        else b = f3(0.0f, -n.z, n.y);
        b = unit3(b);
        t = unit3(cross3(n, b));
    }
    __device__ __forceinline__ Onb(float3 t_, float3 b_, float3 n_) : t(t_), b(b_), n(n_) {}
    __device__ __forceinline__ float3 local(float3 d) const { return d.x * t + d.y * b + d.z * n; }
};

// What shading needs of a triangle that does not depend on the ray, formed once per triangle
// with the same operations the per-hit code would perform (so bit-identical):
//   fr[0] = face normal unit3(cross(v1 - v0, v2 - v0)) and half its cross length (the area
//           MeshLight::Sample weighs by, SimpleKernel.h:96);
//   fr[1..3] = the ONB of that normal (its n, t, b), as sampleCosinePDF builds it.
struct TriFrame {
    float4 fr[4];
};
__device__ __forceinline__ TriFrame make_tri_frame(float3 v0, float3 v1, float3 v2) {
    const float3 nf = cross3(v1 - v0, v2 - v0);
    const float3 fn = unit3(nf);
    const Onb o(fn);
    TriFrame f;
    f.fr[0] = make_float4(fn.x, fn.y, fn.z, len3(nf) / 2.0f);
    f.fr[1] = make_float4(o.n.x, o.n.y, o.n.z, 0.0f);
    f.fr[2] = make_float4(o.t.x, o.t.y, o.t.z, 0.0f);
    f.fr[3] = make_float4(o.b.x, o.b.y, o.b.z, 0.0f);
    return f;
}
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }

// random_cosine_direction (Random.h:321-334); draws x then y
__device__ __forceinline__ float3 sample_cosine(const Onb& onb, uint32_t& rng) {
    const float a = rnd1(rng);
    const float c = rnd1(rng);
    const float r = sqrtf(a), z = sqrtf(1.0f - a);
    float sp, cp;
    sincospif(2.0f * c, &sp, &cp);
    return onb.local(f3(r * cp, r * sp, z));
}
__device__ __forceinline__ float3 sample_cosine(float3 normal, uint32_t& rng) { return sample_cosine(Onb(normal), rng); }
// samplePhongPDF (SimpleGuide.cu:34-41)
__device__ __forceinline__ float3 sample_phong(float3 refl, float s, uint32_t& rng) {
    const float cosT = powf(rnd1(rng), 1.0f / (s + 1.0f));
    const float sinT = sqrtf(fmaxf(1.0f - cosT * cosT, 0.0f));
    const float phi = k2Pi * rnd1(rng);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return Onb(refl).local(f3(sinT * cp, sinT * sp, cosT));
}
// getValPhongPDF (SimpleGuide.cu:42-46)
__device__ __forceinline__ float phong_pdf(float3 d, float3 refl, float s) {
    const float c = fmaxf(dot3(refl, d), 0.0f);
    return (s + 1.0f) * powf(c, s) * kInv2Pi;
}
__device__ __forceinline__ float3 reflect3(float3 d, float3 n) { return d - 2.0f * dot3(d, n) * n; }
// BSDF value of the Phong material (SimpleGuide.cu:345-354)
__device__ __forceinline__ float3 phong_bsdf(float3 kd, float3 ks, float s, float3 d, float3 refl) {
    return kd * kInvPi + ks * ((s + 2.0f) / (s + 1.0f)) * phong_pdf(d, refl, s);
}

}  // namespace rtpg
