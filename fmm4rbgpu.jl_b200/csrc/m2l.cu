// m2l.cu -- M2L: local fields of every target cluster from the moments of the
// sources in its interaction list (the reference's gpu_M2L!,
// src/gpu_fmm/gpu_interaction.jl:3-41, and M2L!, src/fmm/interaction.jl:3-46):
//   E_t[a] += sum_b Gamma_s[b] K(x_a - x_b; p_avg),  B_t[a] += sum_b M_s[b] x K
//   K(R; p) = R / (R.R + (p.R)^2 + eps)^(3/2)
//
// Design: one CTA per target cluster, one thread per target Chebyshev node.
// The CTA walks the target's CSR source list; each source's moment record
// (Gamma, Mx, My, Mz) and node coordinates are staged in shared memory by a
// bulk-copy (TMA) into a double buffer guarded by two mbarriers, so the next
// source streams in while the current one is evaluated.  The kernel matrix is
// generated on the fly; per-axis target-source offsets are hoisted so that one
// evaluation costs three adds/FMAs for the denominator.  (The reference
// re-stages into one shared buffer without a barrier after the compute loop --
// a write-after-read race; here the end-of-iteration barrier orders it.)
//
// FP64 form: double throughout.  Mixed form: FP32 moments and arithmetic, the
// node offsets are formed in FP64 and rounded, per-source partial sums are
// folded into Kahan-compensated FP32 accumulators.
#include "device_util.cuh"
#include "kernels.cuh"

namespace fmmb200 {

namespace {

template <int NDEG>
struct M2LShape {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int TPT = (NN + 511) / 512;
  static constexpr int BT = (((NN + TPT - 1) / TPT) + 31) / 32 * 32;
};

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  float y = v - comp;
  float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

template <int NDEG, bool MIXED>
__global__ void __launch_bounds__(M2LShape<NDEG>::BT)
    m2l_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const double *__restrict__ nodes,
               const void *__restrict__ mom_v, void *__restrict__ loc_v, const double *__restrict__ consts,
               int accumulate, int *__restrict__ status) {
  using S = M2LShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, TPT = S::TPT, BT = S::BT;
  using T = typename std::conditional<MIXED, float, double>::type;
  constexpr int MOM_BYTES = 4 * NN * (int)sizeof(T);
  constexpr int REC_BYTES = MOM_BYTES + NS * 8;  // moments then node coordinates
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[2];

  const T *mom = (const T *)mom_v;
  T *loc = (T *)loc_v;
  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;

  // accumulators: FP64 sums, or FP32 Kahan (sum, compensation) pairs
  double acc[TPT][6];
  float ks[TPT][6], kc[TPT][6];
#pragma unroll
  for (int q = 0; q < TPT; ++q)
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      acc[q][c] = 0.0;
      ks[q][c] = 0.f;
      kc[q][c] = 0.f;
    }

  if (np > 0) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int k, int bb) {
      const int s = src[p0 + k];
      unsigned char *dst = smem + bb * REC_BYTES;
      mbar_arrive_expect_tx(&bar[bb], REC_BYTES);
      bulk_g2s(dst, mom + (int64_t)s * 4 * NN, MOM_BYTES, &bar[bb]);
      bulk_g2s(dst + MOM_BYTES, nodes + (int64_t)s * NS, NS * 8, &bar[bb]);
    };
    if (tid == 0) issue(0, 0);
    const T px = (T)consts[0], py = (T)consts[1], pz = (T)consts[2];
    for (int i = 0; i < np; ++i) {
      const int bb = i & 1;
      if (tid == 0 && i + 1 < np) {
        fence_proxy_async_smem();
        issue(i + 1, bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((i >> 1) & 1), status);
      if (ok) {
        const T *G = (const T *)(smem + bb * REC_BYTES);
        const T *MX = G + NN, *MY = G + 2 * NN, *MZ = G + 3 * NN;
        const double *SN = (const double *)(smem + bb * REC_BYTES + MOM_BYTES);
#pragma unroll
        for (int q = 0; q < TPT; ++q) {
          const int a = tid + q * BT;
          if (a < NN) {
            const int ai = a % M, aj = (a / M) % M, ak = a / (M * M);
            const double tx = tn[ai], ty = tn[M + aj], tz = tn[2 * M + ak];
            T rx[M], prx[M], rx2[M];
#pragma unroll
            for (int bi = 0; bi < M; ++bi) {
              rx[bi] = (T)(tx - SN[bi]);
              prx[bi] = px * rx[bi];
              rx2[bi] = rx[bi] * rx[bi];
            }
            T e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
#pragma unroll 1
            for (int bk = 0; bk < M; ++bk) {
              const T rz = (T)(tz - SN[2 * M + bk]);
              const T prz = pz * rz;
              const T rz2 = rz * rz + (T)kEps64;
#pragma unroll
              for (int bj = 0; bj < M; ++bj) {
                const T ry = (T)(ty - SN[M + bj]);
                const T P = py * ry + prz;
                const T A = ry * ry + rz2;
                const int b0i = M * (bj + M * bk);
#pragma unroll
                for (int bi = 0; bi < M; ++bi) {
                  const T tt = P + prx[bi];
                  const T u = A + rx2[bi];
                  const T d = tt * tt + u;
                  T s;
                  if constexpr (MIXED)
                    s = rsqrt_approx(d);
                  else
                    s = rsqrt(d);
                  const T s3 = s * s * s;
                  const T g = G[b0i + bi] * s3;
                  e0 += g * rx[bi];
                  e1 += g * ry;
                  e2 += g * rz;
                  const T hx = MX[b0i + bi] * s3, hy = MY[b0i + bi] * s3, hz = MZ[b0i + bi] * s3;
                  b0 += hy * rz - hz * ry;
                  b1 += hz * rx[bi] - hx * rz;
                  b2 += hx * ry - hy * rx[bi];
                }
              }
            }
            if constexpr (MIXED) {
              kahan_add(ks[q][0], kc[q][0], e0);
              kahan_add(ks[q][1], kc[q][1], e1);
              kahan_add(ks[q][2], kc[q][2], e2);
              kahan_add(ks[q][3], kc[q][3], b0);
              kahan_add(ks[q][4], kc[q][4], b1);
              kahan_add(ks[q][5], kc[q][5], b2);
            } else {
              acc[q][0] += e0;
              acc[q][1] += e1;
              acc[q][2] += e2;
              acc[q][3] += b0;
              acc[q][4] += b1;
              acc[q][5] += b2;
            }
          }
        }
      }
      __syncthreads();  // everyone is done with buffer bb before it is refilled
    }
  }
  T *out = loc + (int64_t)t * 6 * NN;
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    const int a = tid + q * BT;
    if (a < NN) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        T v;
        if constexpr (MIXED)
          v = ks[q][c];
        else
          v = acc[q][c];
        if (accumulate) v += out[c * NN + a];
        out[c * NN + a] = v;
      }
    }
  }
}

template <int NDEG, bool MIXED>
int launch_m2l_t(Ctx *ctx, bool accumulate) {
  using S = M2LShape<NDEG>;
  using T = typename std::conditional<MIXED, float, double>::type;
  const int rec = 4 * S::NN * (int)sizeof(T) + S::NS * 8;
  const int smem = 2 * rec;
  auto kern = m2l_kernel<NDEG, MIXED>;
  FMM_TRY(opt_in_smem(ctx, kern, smem));
  if (ctx->nc > 0)
    kern<<<(unsigned)ctx->nc, S::BT, smem, ctx->stream>>>(
        ctx->get<int>("m2l_ptr"), ctx->get<int>("m2l_src"), ctx->get<double>("nodes"),
        MIXED ? (const void *)ctx->get<float>("mom32") : (const void *)ctx->get<double>("mom64"),
        MIXED ? (void *)ctx->get<float>("loc32") : (void *)ctx->get<double>("loc64"), ctx->get<double>("consts"),
        accumulate ? 1 : 0, ctx->d_status);
  return ctx->check_launch("m2l_kernel");
}

}  // namespace

int launch_m2l(Ctx *ctx, int n, bool mixed, bool accumulate) {
#define FMM_M2L_CASE(D) \
  case D:               \
    return mixed ? launch_m2l_t<D, true>(ctx, accumulate) : launch_m2l_t<D, false>(ctx, accumulate);
  switch (n) {
    FMM_M2L_CASE(1)
    FMM_M2L_CASE(2)
    FMM_M2L_CASE(3)
    FMM_M2L_CASE(4)
    FMM_M2L_CASE(5)
    FMM_M2L_CASE(6)
    FMM_M2L_CASE(7)
    FMM_M2L_CASE(8)
    FMM_M2L_CASE(9)
    FMM_M2L_CASE(10)
    default:
      return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "degree n must be in 1..10");
  }
#undef FMM_M2L_CASE
}

}  // namespace fmmb200
