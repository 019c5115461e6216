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

// Mixed P2P and P2P^T tiles whose source and target boxes are apart by more than
// 1/kHiOnlyGap of the larger extent form every pair difference R from the hi parts of the
// coordinates alone (the lo parts are skipped).  Every pair of such a tile is at least the gap
// apart while the coordinates (in the source leaf's frame) are at most about 1.5 extents, so R
// keeps a relative error below about 3 kHiOnlyGap FP32 ulps (1e-4 at 256), reached only by
// pairs at the gap itself.  At 256, 87 % of the P2P tiles of the N = 2^24 Gaussian bunch
// (n = 4, N0 = 125) take the hi path (55 % at 16): the P2P stage drops from 57.0 to 51.7 ms,
// and the mixed-vs-FP64 error over all particles moves from 2.233e-7 to 2.238e-7 (2^22: Gaussian
// 1.91e-7 -> 2.04e-7, uniform 2.44e-7 -> 2.45e-7, beamlets 1.84e-7 -> 2.02e-7).
constexpr double kHiOnlyGap = 256.0;

__device__ __forceinline__ bool p2p_tile_needs_lo(const double *sb, const double *tb) {
  double gap = 0.0, ext = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    gap = fmax(gap, fmax(sb[d] - tb[3 + d], tb[d] - sb[3 + d]));
    ext = fmax(ext, fmax(sb[3 + d] - sb[d], tb[3 + d] - tb[d]));
  }
  return !(kHiOnlyGap * gap > ext);
}

// The FP32 M2L kernels factor their sums over the source nodes y_b around the target
// centre (E = x' G - Q and the like), which loses a factor (|x'| + |y|) / |x' - y| of
// precision for a target node x' and a source node y.  True when that factor stays
// below kFactoredMaxCancel for every node pair of the target box (centre c, corners
// tb[0..2], tb[3..5]) and the source box (corners sb[0..2], sb[3..5]): |x'| <= |h_t|,
// |y| <= |c_s - c| + |h_s|, and |x' - y| is at least the distance between the boxes.
// Pairs of boxes that nearly touch fail it.
constexpr double kFactoredMaxCancel = 16.0;

__device__ __forceinline__ bool factored_ok(const double *sb, const double *tb, double cx, double cy, double cz) {
  double R2 = 0.0, gap2 = 0.0, rt2 = 0.0, rs2 = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = sb[d], hi = sb[3 + d];
    const double hs = 0.5 * (hi - lo), ht = 0.5 * (tb[3 + d] - tb[d]);
    const double dc = fabs(0.5 * (lo + hi) - (d == 0 ? cx : (d == 1 ? cy : cz)));
    const double g = fmax(0.0, dc - hs - ht);
    R2 += dc * dc;
    gap2 += g * g;
    rt2 += ht * ht;
    rs2 += hs * hs;
  }
  const double span = sqrt(rt2) + sqrt(R2) + sqrt(rs2);
  return span * span < kFactoredMaxCancel * kFactoredMaxCancel * gap2;
}

}  // namespace fmmb200
