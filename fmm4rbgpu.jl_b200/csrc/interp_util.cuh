// interp_util.cuh -- barycentric Lagrange weights on Chebyshev points of the
// second kind (and their derivatives, for the adjoint).
//   w_i(x) = (ws_i / (x - x_i)) / sum_j ws_j / (x - x_j),  ws = (1/2, -1, 1, ..., (-1)^n/2)
// with the reference's exact-node rule: |x - x_i| < eps(Float64) -> indicator of
// the last such node (gpu_upwardpass.jl:48-76).
#pragma once

#include "device_util.cuh"

namespace fmmb200 {

// second-kind barycentric weights: 1/2, -1, 1, ..., (-1)^n/2
__device__ __forceinline__ double bary_ws(int i, int M) {
  double w = (i & 1) ? -1.0 : 1.0;
  return (i == 0 || i == M - 1) ? 0.5 * w : w;
}

// FP64 weights of the M nodes at x (GPU exact-node semantics).
template <int M, typename TW>
__device__ __forceinline__ void weights64(double x, const double *nodes, TW *w) {
  double q[M];
  double sum = 0.0;
  int flag = -1;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const double dx = x - nodes[i];
    flag = fabs(dx) < kEps64 ? i : flag;
    q[i] = bary_ws(i, M) / dx;
    sum += q[i];
  }
  if (flag >= 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = (TW)(i == flag ? 1.0 : 0.0);
  } else {
    const double inv = 1.0 / sum;
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = (TW)(q[i] * inv);
  }
}

// FP32 weights from leaf-local FP32 coordinates (exact hit: dx == 0 or subnormal).
template <int M>
__device__ __forceinline__ void weights32(float x, const float *nodes, float *w) {
  float q[M];
  float sum = 0.f;
  int flag = -1;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const float dx = x - nodes[i];
    flag = fabsf(dx) < 1.17549435e-38f ? i : flag;
    q[i] = (float)bary_ws(i, M) / dx;
    sum += q[i];
  }
  if (flag >= 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = i == flag ? 1.f : 0.f;
  } else {
    const float inv = 1.f / sum;
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = q[i] * inv;
  }
}

// As weights32 with the approximate FP32 division (__fdividef, ~2 ulp): the
// normalisation by the sum of the q_i carries that error into every weight
// alike, so the weights still sum to 1 to FP32 rounding.
template <int M>
__device__ __forceinline__ void weights32_fast(float x, const float *nodes, float *w) {
  float q[M];
  float sum = 0.f;
  int flag = -1;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const float dx = x - nodes[i];
    flag = fabsf(dx) < 1.17549435e-38f ? i : flag;
    q[i] = __fdividef((float)bary_ws(i, M), dx);
    sum += q[i];
  }
  if (flag >= 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = i == flag ? 1.f : 0.f;
  } else {
    const float inv = __fdividef(1.f, sum);
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = q[i] * inv;
  }
}

// Weights and their x-derivatives (FP64).  Off the nodes
//   w_i' = w_i (S2/S - 1/(x - x_i)),  S = sum_j ws_j/(x-x_j), S2 = sum_j ws_j/(x-x_j)^2;
// on node k the barycentric differentiation matrix row
//   w_i'(x_k) = (ws_i/ws_k)/(x_k - x_i) (i != k),  w_k'(x_k) = -sum_{i!=k} w_i'(x_k).
// A degenerate axis (all nodes equal) has zero derivatives.
template <int M>
__device__ __forceinline__ void weights_d64(double x, const double *nodes, double *w, double *dw) {
  double q[M], dx[M];
  double sum = 0.0, sum2 = 0.0;
  int flag = -1;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    dx[i] = x - nodes[i];
    flag = fabs(dx[i]) < kEps64 ? i : flag;
    q[i] = bary_ws(i, M) / dx[i];
    sum += q[i];
    sum2 += q[i] / dx[i];
  }
  const bool degenerate = nodes[0] == nodes[M - 1];
  if (flag >= 0) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      w[i] = i == flag ? 1.0 : 0.0;
      double d = 0.0;
      if (i != flag && !degenerate) d = (bary_ws(i, M) / bary_ws(flag, M)) / (nodes[flag] - nodes[i]);
      dw[i] = d;
      acc += d;
    }
#pragma unroll
    for (int i = 0; i < M; ++i)
      if (i == flag) dw[i] = -acc;
  } else {
    const double inv = 1.0 / sum, r = sum2 * inv;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      w[i] = q[i] * inv;
      dw[i] = degenerate ? 0.0 : w[i] * (r - 1.0 / dx[i]);
    }
  }
}

// Chebyshev fractions t_i = (cos(pi i/n) + 1)/2: node i of [a, b] is a + t_i (b - a).
struct ChebT {
  double t[kMaxNodes1D];
};

}  // namespace fmmb200
