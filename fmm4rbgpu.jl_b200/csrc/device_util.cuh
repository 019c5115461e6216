// device_util.cuh -- device helpers: warp/block scans, order-preserving keys,
// and the sm_100a bulk-copy (TMA) + mbarrier primitives used for staging.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace fmmb200 {

// ---------------------------------------------------------------- keys
// Order-preserving map double -> uint64 (IEEE total order on finite values);
// -0.0 is folded onto +0.0 so that the two compare equal, as `<` does.
__device__ __forceinline__ uint64_t double_key(double v) {
  uint64_t b = (uint64_t)__double_as_longlong(v);
  if (b == 0x8000000000000000ull) b = 0;
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// ---------------------------------------------------------------- scans
__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one int per thread (blockDim.x multiple of 32,
// <= 1024).  s_warp must hold 33 ints.  Returns the exclusive prefix; *total
// receives the block sum.
__device__ __forceinline__ int block_excl_scan(int v, int *s_warp, int *total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int inc = warp_incl_scan(v);
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? s_warp[lane] : 0;
    int wi = warp_incl_scan(w);
    if (lane < nw) s_warp[lane] = wi - w;
    if (lane == nw - 1) s_warp[32] = wi;
  }
  __syncthreads();
  int res = s_warp[wid] + inc - v;
  if (total) *total = s_warp[32];
  __syncthreads();
  return res;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------- bulk copy (TMA) + mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar` (bytes % 16 == 0,
// both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase: gives up after `limit` polls, raises the
// device status word and returns false (the caller skips the work; no trap).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status,
                                                  uint32_t limit = (1u << 24)) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (status) atomicCAS(status, kDevOk, kDevQueueOverflow);
  return false;
}

// ---------------------------------------------------------------- exact (uncontracted) FP64 ops
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
// norm of a 3-vector as sqrt((a^2 + b^2) + c^2), each operation rounded
__device__ __forceinline__ double norm3_exact(double a, double b, double c) {
  return __dsqrt_rn(rn_add(rn_add(rn_mul(a, a), rn_mul(b, b)), rn_mul(c, c)));
}

}  // namespace fmmb200
