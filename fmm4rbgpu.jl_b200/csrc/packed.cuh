// packed.cuh -- packed FP32x2 arithmetic for the mixed-form M2L / P2P kernels.
//
// sm_100 executes two FP32 adds, multiplies or FMAs per lane in one instruction
// (FADD2 / FMUL2 / FFMA2, reached through __fadd2_rn / __fmul2_rn / __ffma2_rn),
// each lane of the pair rounded exactly as the scalar operation would be.  The
// kernels evaluate two targets per thread in the two halves of a float2, so one
// instruction stream serves both; per-source operands are stored duplicated
// ((v, v) pairs) in shared memory, so a 128-bit shared load yields two packed
// operands without register moves.
#pragma once

#include <cuda_runtime.h>

namespace fmmb200 {

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

__device__ __forceinline__ float rsqrt_approx_f32(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 rsqrt2(float2 d) { return make_float2(rsqrt_approx_f32(d.x), rsqrt_approx_f32(d.y)); }

// Kahan-compensated accumulation of v into (sum, comp), lane by lane; the value
// held is sum - comp.
__device__ __forceinline__ void kahan_add2(float2 &sum, float2 &comp, float2 v) {
  const float2 y = sub2(v, comp);
  const float2 t = add2(sum, y);
  comp = sub2(sub2(t, sum), y);
  sum = t;
}

}  // namespace fmmb200
