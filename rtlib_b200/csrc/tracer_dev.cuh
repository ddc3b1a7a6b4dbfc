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
    __device__ __forceinline__ float3 local(float3 d) const { return d.x * t + d.y * b + d.z * n; }
};

// random_cosine_direction (Random.h:321-334); draws x then y
__device__ __forceinline__ float3 sample_cosine(float3 normal, uint32_t& rng) {
    const float a = rnd1(rng);
    const float c = rnd1(rng);
    const float r = sqrtf(a), z = sqrtf(1.0f - a);
    float sp, cp;
    sincospif(2.0f * c, &sp, &cp);
    return Onb(normal).local(f3(r * cp, r * sp, z));
}
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
