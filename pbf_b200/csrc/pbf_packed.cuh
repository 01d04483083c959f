// Packed FP32 arithmetic for sm_100a: T = float (one value) or float2 (two values
// per instruction, the PTX f32x2 instructions). Each float2 operation is, per
// component, the scalar IEEE operation with round-to-nearest.
#pragma once
#include <cuda_runtime.h>

namespace pbf {

// The float2 forms are the PTX f32x2 instructions with an explicit .rn rounding
// modifier, which the compiler never contracts (a multiply feeding an add stays
// two rounded operations, as in the scalar code built with -fmad=false).
__device__ __forceinline__ unsigned long long as_u64(float2 a) {
    return (unsigned long long)__float_as_uint(a.x) | ((unsigned long long)__float_as_uint(a.y) << 32);
}
__device__ __forceinline__ float2 as_f2(unsigned long long u) {
    return make_float2(__uint_as_float((unsigned)u), __uint_as_float((unsigned)(u >> 32)));
}
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)), "l"(as_u64(c)));
    return as_f2(d);
}
__device__ __forceinline__ float vneg(float a) { return -a; }
__device__ __forceinline__ float2 vneg(float2 a) { return make_float2(-a.x, -a.y); }
// a - b is a + (-b) exactly, signed zeros included
template <typename T> __device__ __forceinline__ T vsub(T a, T b) { return vadd(a, vneg(b)); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float2 vmax(float2 a, float b) { return make_float2(fmaxf(a.x, b), fmaxf(a.y, b)); }

template <typename T> __device__ __forceinline__ T bc(float s);
template <> __device__ __forceinline__ float bc<float>(float s) { return s; }
template <> __device__ __forceinline__ float2 bc<float2>(float s) { return make_float2(s, s); }

}  // namespace pbf
