// Small float3 helpers for the cloth kernels.
//
// Every helper fixes its evaluation order so the kernels compute exactly the
// float expressions of the FP32 restatement (the library is built with
// -fmad=false, so no product is fused into an add behind our back).  The
// order follows the reference's Vec3 algebra (tools/cloth_bag.cpp:104-214):
// dot = (x*x + y*y) + z*z, a/s = a*(1/s), rotation by q as
// v + w*(2 q.xyz x v) + q.xyz x (2 q.xyz x v).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 xyz(float4 a) { return V3{a.x, a.y, a.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
// Division through the reciprocal, as the reference's Vec3 operator/ does.
__device__ __forceinline__ V3 vdiv(V3 a, float s) { return a * (1.0f / s); }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float lsq(V3 a) { return dot3(a, a); }
__device__ __forceinline__ float len3(V3 a) { return sqrtf(lsq(a)); }
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 normalized3(V3 a) {
    const float m = len3(a);
    return m > 1.0e-14f ? vdiv(a, m) : V3{1.0f, 0.0f, 0.0f};
}
__device__ __forceinline__ bool finite3(V3 a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}
// q = (x, y, z, w).
__device__ __forceinline__ V3 rotate_q(float4 q, V3 v) {
    const V3 u{q.x, q.y, q.z};
    const V3 twice = cross3(u, v) * 2.0f;
    return (v + twice * q.w) + cross3(u, twice);
}
__device__ __forceinline__ V3 inverse_rotate_q(float4 q, V3 v) {
    return rotate_q(make_float4(-q.x, -q.y, -q.z, q.w), v);
}
__device__ __forceinline__ float4 with_xyz(float4 a, V3 p) { return make_float4(p.x, p.y, p.z, a.w); }
template <class T>
__device__ __forceinline__ T nf4(float x, float y, float z, float w) {
    T r;
    r.x = x;
    r.y = y;
    r.z = z;
    r.w = w;
    return r;
}
