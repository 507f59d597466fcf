// packed.cuh — packed FP32 pair arithmetic (sm_100 f32x2 instructions).
//
// Each function applies one IEEE operation to each lane of a float2 and never
// mixes the lanes: fma.rn.f32x2, add.rn.f32x2 and mul.rn.f32x2 issue one
// instruction for two single-precision operations.
#pragma once

#include <cuda_runtime.h>

namespace sirius {

__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 max2(float2 a, float b) { return make_float2(fmaxf(a.x, b), fmaxf(a.y, b)); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
// 2^x by the special-function unit (PTX ex2.approx.ftz.f32: a few ulp of
// relative error, subnormal results flushed to zero)
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// square root of a positive argument from the reciprocal square root (single-
// precision relative accuracy, not correct rounding)
__device__ __forceinline__ float2 sqrt2(float2 a) { return mul2(a, make_float2(rsqrtf(a.x), rsqrtf(a.y))); }

}  // namespace sirius
