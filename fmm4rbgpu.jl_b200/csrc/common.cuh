// common.cuh -- shared definitions of libfmmb200 (B200 / sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/fmmb200.h"

namespace fmmb200 {

// eps(Float64): the kernel regulariser of every K(R; p) evaluation and the
// absolute exact-node threshold of the Lagrange weights.
constexpr double kEps64 = 2.220446049250313e-16;
// classical electron radius in amp = r_e * q / lambda
constexpr double kRe = 2.8179403699772166e-15;

constexpr int kMaxDegree = 10;  // n+1 <= 11 Chebyshev nodes per axis
constexpr int kMaxNodes1D = kMaxDegree + 1;

// Status raised from device code into ctx->d_status (never __trap()).
enum DeviceStatus : int {
  kDevOk = 0,
  kDevBadIndex = 1,
  kDevQueueOverflow = 2,
  kDevTreeShape = 3,
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Stretched-metric cluster geometry used by the traversal, computed once per
// cluster with the reference's operation order (no contraction).
struct ClusterGeom {
  double xc[3];
  double r;     // norm(stretch .* (bmax - xc))
  double diam;  // norm(stretch .* (bmax - bmin) ./ 2)
  int leaf;
  int pad;
};

}  // namespace fmmb200

#define FMM_CUDA_TRY(ctx, expr)                                                         \
  do {                                                                                  \
    cudaError_t e__ = (expr);                                                           \
    if (e__ != cudaSuccess) {                                                           \
      return (ctx)->fail(FMMB200_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
    }                                                                                   \
  } while (0)

#define FMM_TRY(expr)        \
  do {                       \
    int s__ = (expr);        \
    if (s__ != 0) return s__; \
  } while (0)
