// Equal-area cylindrical map between unit directions and [0,1]^2 (RTLib's canonical_to_dir /
// dir_to_canonical, VectorFunction.h:5698-5720).
#pragma once
#include "common.cuh"

namespace rtpg {

// canonical_to_dir / dir_to_canonical (VectorFunction.h:5698-5720)
// phi = 2 pi v is evaluated as sincospi(2 v): no range reduction, within 1 ulp.
__device__ __forceinline__ float3 canonical_to_dir(float u, float v) {
    const float cosTheta = 2.0f * u - 1.0f;
    const float sinTheta = sqrtf(fmaxf(1.0f - cosTheta * cosTheta, 0.0f));
    float sp, cp;
    sincospif(2.0f * v, &sp, &cp);
    return make_float3(sinTheta * cp, sinTheta * sp, cosTheta);
}
__device__ __forceinline__ float2 dir_to_canonical(float x, float y, float z) {
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) return make_float2(0.0f, 0.0f);
    z = fminf(fmaxf(z, -1.0f), 1.0f);
    float phi = atan2f(y, x);
    while (phi < 0.0f) phi += k2Pi;
    return make_float2((z + 1.0f) / 2.0f, phi * kInv2Pi);
}
__device__ __forceinline__ float3 normalize3(float3 v) {
    const float r = rsqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x * r, v.y * r, v.z * r);
}

}  // namespace rtpg
