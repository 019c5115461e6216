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
// evaluation costs three adds/FMAs for the denominator, and the E/B sums are
// factored through per-source-node vectors packed once per source (below), so
// that an evaluation accumulates with 10 FMAs.  (The reference
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

// Packed per-source-node data (x' = node - target centre):
//   P0 = (Gamma, Gamma x', Gamma y', Gamma z'), P1 = (Mx, My, Mz, 0), P2 = M x x' (3), 0
// so that, with s3 = d^{-3/2},
//   E_a = sum s3 Gamma_b (x_a - x_b) = x_a' G - Q,     G = sum s3 Gamma_b,  Q = sum s3 Gamma_b x_b'
//   B_a = sum s3 M_b x (x_a - x_b)   = W x x_a' - V,   W = sum s3 M_b,      V = sum s3 M_b x x_b'
// and one evaluation costs the denominator (3), rsqrt, s3 (2) and 10 FMAs.
// MASK: zero K at coincident nodes (R = 0), possible only for eta > 1/2.
template <int NDEG, bool MIXED, bool MASK>
__global__ void __launch_bounds__(M2LShape<NDEG>::BT)
    m2l_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const double *__restrict__ nodes,
               const double *__restrict__ bbox, const void *__restrict__ mom_v, void *__restrict__ loc_v,
               const double *__restrict__ consts, int accumulate, int *__restrict__ status) {
  using S = M2LShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, TPT = S::TPT, BT = S::BT;
  using T = typename std::conditional<MIXED, float, double>::type;
  using T4 = typename std::conditional<MIXED, float4, double4>::type;
  constexpr int MOM_BYTES = 4 * NN * (int)sizeof(T);
  constexpr int REC_BYTES = MOM_BYTES + NS * 8;  // raw moments then node coordinates
  extern __shared__ __align__(16) unsigned char smem[];
  T4 *pk = (T4 *)(smem + 2 * REC_BYTES);  // 3*NN packed entries
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_sn[3 * M];           // source node offsets from the target centre

  const T *mom = (const T *)mom_v;
  T *loc = (T *)loc_v;
  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);

  // E(3), B(3) accumulated over source pairs: FP64 sums, or FP32 Kahan (sum, compensation)
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
    const double pxd = consts[0], pyd = consts[1], pzd = consts[2];
    const T px = (T)pxd, py = (T)pyd, pz = (T)pzd;
    for (int i = 0; i < np; ++i) {
      const int bb = i & 1;
      if (tid == 0 && i + 1 < np) {
        fence_proxy_async_smem();
        issue(i + 1, bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((i >> 1) & 1), status);
      // pack the source's node data relative to the target centre
      const T *G = (const T *)(smem + bb * REC_BYTES);
      const double *SN = (const double *)(smem + bb * REC_BYTES + MOM_BYTES);
      if (ok) {
        for (int e = tid; e < 3 * M; e += BT) {
          const int d = e / M;
          s_sn[e] = SN[e] - (d == 0 ? cx : (d == 1 ? cy : cz));
        }
        for (int b = tid; b < NN; b += BT) {
          const int bi = b % M, bj = (b / M) % M, bk = b / (M * M);
          const T xb = (T)(SN[bi] - cx), yb = (T)(SN[M + bj] - cy), zb = (T)(SN[2 * M + bk] - cz);
          const T g = G[b], m0 = G[NN + b], m1 = G[2 * NN + b], m2 = G[3 * NN + b];
          T4 a, c, e;
          a.x = g; a.y = g * xb; a.z = g * yb; a.w = g * zb;
          c.x = m0; c.y = m1; c.z = m2; c.w = 0;
          e.x = m1 * zb - m2 * yb; e.y = m2 * xb - m0 * zb; e.z = m0 * yb - m1 * xb; e.w = 0;
          pk[3 * b] = a;
          pk[3 * b + 1] = c;
          pk[3 * b + 2] = e;
        }
      }
      __syncthreads();
      if (ok) {
#pragma unroll
        for (int q = 0; q < TPT; ++q) {
          const int a = tid + q * BT;
          if (a < NN) {
            const int ai = a % M, aj = (a / M) % M, ak = a / (M * M);
            const double tx = tn[ai] - cx, ty = tn[M + aj] - cy, tz = tn[2 * M + ak] - cz;
            T prx[M], rx2[M];
#pragma unroll
            for (int bi = 0; bi < M; ++bi) {
              const T rx = (T)(tx - s_sn[bi]);
              prx[bi] = px * rx;
              rx2[bi] = rx * rx;
            }
            T g0 = 0, q0 = 0, q1 = 0, q2 = 0, w0 = 0, w1 = 0, w2 = 0, v0 = 0, v1 = 0, v2 = 0;
#pragma unroll 1
            for (int bk = 0; bk < M; ++bk) {
              const T rz = (T)(tz - s_sn[2 * M + bk]);
              const T prz = pz * rz;
              const T rz2 = rz * rz + (T)kEps64;
#pragma unroll
              for (int bj = 0; bj < M; ++bj) {
                const T ry = (T)(ty - s_sn[M + bj]);
                const T P = py * ry + prz;
                const T A = ry * ry + rz2;
                const T4 *pb = pk + 3 * M * (bj + M * bk);
#pragma unroll
                for (int bi = 0; bi < M; ++bi) {
                  const T tt = P + prx[bi];
                  const T d = tt * tt + (A + rx2[bi]);
                  T s;
                  if constexpr (MIXED)
                    s = rsqrt_approx(d);
                  else
                    s = rsqrt(d);
                  T s3 = s * s * s;
                  if constexpr (MASK) s3 = d > (T)kEps64 ? s3 : (T)0;
                  const T4 a4 = pb[3 * bi], m4 = pb[3 * bi + 1], c4 = pb[3 * bi + 2];
                  g0 += s3 * a4.x;
                  q0 += s3 * a4.y;
                  q1 += s3 * a4.z;
                  q2 += s3 * a4.w;
                  w0 += s3 * m4.x;
                  w1 += s3 * m4.y;
                  w2 += s3 * m4.z;
                  v0 += s3 * c4.x;
                  v1 += s3 * c4.y;
                  v2 += s3 * c4.z;
                }
              }
            }
            // this source's E and B at the node: E = x' G - Q, B = W x x' - V.  Folding per
            // source keeps the cancellation between sources in the compensated sum.
            const T xa = (T)tx, ya = (T)ty, za = (T)tz;
            const T part[6] = {xa * g0 - q0, ya * g0 - q1, za * g0 - q2,
                               (w1 * za - w2 * ya) - v0, (w2 * xa - w0 * za) - v1, (w0 * ya - w1 * xa) - v2};
#pragma unroll
            for (int c = 0; c < 6; ++c) {
              if constexpr (MIXED)
                kahan_add(ks[q][c], kc[q][c], part[c]);
              else
                acc[q][c] += part[c];
            }
          }
        }
      }
      __syncthreads();  // the packed data and buffer bb are rewritten later
    }
  }
  T *out = loc + (int64_t)t * 6 * NN;
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    const int a = tid + q * BT;
    if (a < NN) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        T o = MIXED ? (T)((double)ks[q][c] - (double)kc[q][c]) : (T)acc[q][c];
        if (accumulate) o += out[c * NN + a];
        out[c * NN + a] = o;
      }
    }
  }
}

template <int NDEG, bool MIXED, bool MASK>
int launch_m2l_t(Ctx *ctx, bool accumulate) {
  using S = M2LShape<NDEG>;
  using T = typename std::conditional<MIXED, float, double>::type;
  const int rec = 4 * S::NN * (int)sizeof(T) + S::NS * 8;
  const int smem = 2 * rec + 3 * S::NN * 4 * (int)sizeof(T);
  auto kern = m2l_kernel<NDEG, MIXED, MASK>;
  FMM_TRY(opt_in_smem(ctx, kern, smem));
  if (ctx->nc > 0)
    kern<<<(unsigned)ctx->nc, S::BT, smem, ctx->stream>>>(
        ctx->get<int>("m2l_ptr"), ctx->get<int>("m2l_src"), ctx->get<double>("nodes"), ctx->get<double>("bbox"),
        MIXED ? (const void *)ctx->get<float>("mom32") : (const void *)ctx->get<double>("mom64"),
        MIXED ? (void *)ctx->get<float>("loc32") : (void *)ctx->get<double>("loc64"), ctx->get<double>("consts"),
        accumulate ? 1 : 0, ctx->d_status);
  return ctx->check_launch("m2l_kernel");
}

template <int NDEG>
int launch_m2l_n(Ctx *ctx, bool mixed, bool accumulate) {
  // coincident target/source nodes need eta > 1/2 (admissible: max(r1,r2) < eta R)
  const bool mask = !(ctx->eta <= 0.5);
  if (mixed) return mask ? launch_m2l_t<NDEG, true, true>(ctx, accumulate) : launch_m2l_t<NDEG, true, false>(ctx, accumulate);
  return mask ? launch_m2l_t<NDEG, false, true>(ctx, accumulate) : launch_m2l_t<NDEG, false, false>(ctx, accumulate);
}

}  // namespace

int launch_m2l(Ctx *ctx, int n, bool mixed, bool accumulate) {
#define FMM_M2L_CASE(D) \
  case D:               \
    return launch_m2l_n<D>(ctx, mixed, accumulate);
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
