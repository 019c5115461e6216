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
// FP64 form (m2l_kernel): double throughout, one target node per thread.
// Mixed form (m2l_x2_kernel): FP32 moments and arithmetic in packed FP32x2
// instructions, two target nodes per thread in the two lanes of a float2; the
// node offsets are formed in FP64 and rounded, and per-source partial sums are
// folded into Kahan-compensated FP32 accumulators.
#include "device_util.cuh"
#include "kernels.cuh"
#include "packed.cuh"

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

// Packed per-source-node data (x' = node - target centre):
//   P0 = (Gamma, Gamma x', Gamma y', Gamma z'), P1 = (Mx, My, Mz, 0), P2 = M x x' (3), 0
// so that, with s3 = d^{-3/2},
//   E_a = sum s3 Gamma_b (x_a - x_b) = x_a' G - Q,     G = sum s3 Gamma_b,  Q = sum s3 Gamma_b x_b'
//   B_a = sum s3 M_b x (x_a - x_b)   = W x x_a' - V,   W = sum s3 M_b,      V = sum s3 M_b x x_b'
// and one evaluation costs the denominator (3), rsqrt, s3 (2) and 10 FMAs.
// MASK: zero K at coincident nodes (R = 0), possible only for eta > 1/2.
template <int NDEG, bool MASK>
__global__ void __launch_bounds__(M2LShape<NDEG>::BT)
    m2l_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const double *__restrict__ nodes,
               const double *__restrict__ bbox, const double *__restrict__ mom, double *__restrict__ loc,
               const double *__restrict__ consts, int accumulate, int *__restrict__ status) {
  using S = M2LShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, TPT = S::TPT, BT = S::BT;
  using T = double;
  using T4 = double4;
  constexpr int MOM_BYTES = 4 * NN * (int)sizeof(T);
  constexpr int REC_BYTES = MOM_BYTES + NS * 8;  // raw moments then node coordinates
  extern __shared__ __align__(16) unsigned char smem[];
  T4 *pk = (T4 *)(smem + 2 * REC_BYTES);  // 3*NN packed entries
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_sn[3 * M];           // source node offsets from the target centre

  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);

  // E(3), B(3) accumulated over source pairs
  double acc[TPT][6];
#pragma unroll
  for (int q = 0; q < TPT; ++q)
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[q][c] = 0.0;

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
                  const T s = rsqrt(d);
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
            // this source's E and B at the node: E = x' G - Q, B = W x x' - V
            const T part[6] = {tx * g0 - q0, ty * g0 - q1, tz * g0 - q2,
                               (w1 * tz - w2 * ty) - v0, (w2 * tx - w0 * tz) - v1, (w0 * ty - w1 * tx) - v2};
#pragma unroll
            for (int c = 0; c < 6; ++c) acc[q][c] += part[c];
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
        T o = acc[q][c];
        if (accumulate) o += out[c * NN + a];
        out[c * NN + a] = o;
      }
    }
  }
}

// Mixed form: two target nodes per thread (a0 = k, a1 = k + NP with NP = ceil(NN/2)),
// evaluated in the two lanes of packed FP32x2 instructions.  The per-source-node
// data of the factored sums is stored duplicated, five float4 per node:
//   (G,G, Gx',Gx') (Gy',Gy', Gz',Gz') (M0,M0, M1,M1) (M2,M2, C0,C0) (C1,C1, C2,C2)
// with C = M x x', so that one evaluation pair costs 3 packed ops for the
// denominator, 2 rsqrt, 2 packed ops for s^3, 10 FFMA2 and 5 shared loads.
template <int NDEG>
struct M2LShape2 {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int NP = (NN + 1) / 2;             // target-node pairs
  static constexpr int TPP = (NP + 511) / 512;        // pairs per thread
  static constexpr int BT = (((NP + TPP - 1) / TPP) + 31) / 32 * 32;
  static constexpr int REC = 4 * NN * 4 + NS * 8;     // raw FP32 moments then node coordinates
  static constexpr int SMEM = 2 * REC + 5 * NN * 16;  // double buffer + packed node data
};

template <int NDEG, bool MASK>
__global__ void __launch_bounds__(M2LShape2<NDEG>::BT)
    m2l_x2_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const double *__restrict__ nodes,
                  const double *__restrict__ bbox, const float *__restrict__ mom, float *__restrict__ loc,
                  const double *__restrict__ consts, int accumulate, int *__restrict__ status) {
  using S = M2LShape2<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, NP = S::NP, TPP = S::TPP, BT = S::BT, REC = S::REC;
  constexpr int MOM_BYTES = 4 * NN * 4;
  extern __shared__ __align__(16) unsigned char smem[];
  float4 *pk = (float4 *)(smem + 2 * REC);  // 5*NN packed entries
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_sn[3 * M];  // source node offsets from the target centre

  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);

  // per pair: E(3), B(3) of both targets as Kahan (sum, compensation) pairs
  float2 ks[TPP][6], kc[TPP][6];
#pragma unroll
  for (int q = 0; q < TPP; ++q)
#pragma unroll
    for (int c = 0; c < 6; ++c) ks[q][c] = kc[q][c] = make_float2(0.f, 0.f);

  if (np > 0) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int k, int bb) {
      const int s = src[p0 + k];
      unsigned char *dst = smem + bb * REC;
      mbar_arrive_expect_tx(&bar[bb], REC);
      bulk_g2s(dst, mom + (int64_t)s * 4 * NN, MOM_BYTES, &bar[bb]);
      bulk_g2s(dst + MOM_BYTES, nodes + (int64_t)s * NS, NS * 8, &bar[bb]);
    };
    if (tid == 0) issue(0, 0);
    const float2 px = dup2((float)consts[0]), py = dup2((float)consts[1]), pz = dup2((float)consts[2]);
    const float2 eps = dup2((float)kEps64);
    for (int i = 0; i < np; ++i) {
      const int bb = i & 1;
      if (tid == 0 && i + 1 < np) {
        fence_proxy_async_smem();
        issue(i + 1, bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((i >> 1) & 1), status);
      const float *G = (const float *)(smem + bb * REC);
      const double *SN = (const double *)(smem + bb * REC + MOM_BYTES);
      if (ok) {
        for (int e = tid; e < 3 * M; e += BT) {
          const int d = e / M;
          s_sn[e] = SN[e] - (d == 0 ? cx : (d == 1 ? cy : cz));
        }
        for (int b = tid; b < NN; b += BT) {
          const int bi = b % M, bj = (b / M) % M, bk = b / (M * M);
          const float xb = (float)(SN[bi] - cx), yb = (float)(SN[M + bj] - cy), zb = (float)(SN[2 * M + bk] - cz);
          const float g = G[b], m0 = G[NN + b], m1 = G[2 * NN + b], m2 = G[3 * NN + b];
          const float c0 = m1 * zb - m2 * yb, c1 = m2 * xb - m0 * zb, c2 = m0 * yb - m1 * xb;
          float4 *o = pk + 5 * b;
          o[0] = make_float4(g, g, g * xb, g * xb);
          o[1] = make_float4(g * yb, g * yb, g * zb, g * zb);
          o[2] = make_float4(m0, m0, m1, m1);
          o[3] = make_float4(m2, m2, c0, c0);
          o[4] = make_float4(c1, c1, c2, c2);
        }
      }
      __syncthreads();
      if (ok) {
#pragma unroll
        for (int q = 0; q < TPP; ++q) {
          const int k = tid + q * BT;
          if (k < NP) {
            // the pair's targets (a1 past the end repeats a0 and is not written)
            const int a0 = k, a1 = k + NP < NN ? k + NP : k;
            const double tx0 = tn[a0 % M] - cx, ty0 = tn[M + (a0 / M) % M] - cy, tz0 = tn[2 * M + a0 / (M * M)] - cz;
            const double tx1 = tn[a1 % M] - cx, ty1 = tn[M + (a1 / M) % M] - cy, tz1 = tn[2 * M + a1 / (M * M)] - cz;
            float2 prx[M], rx2[M], ryv[M];
#pragma unroll
            for (int b = 0; b < M; ++b) {
              const float2 rx = make_float2((float)(tx0 - s_sn[b]), (float)(tx1 - s_sn[b]));
              prx[b] = mul2(px, rx);
              rx2[b] = mul2(rx, rx);
              ryv[b] = make_float2((float)(ty0 - s_sn[M + b]), (float)(ty1 - s_sn[M + b]));
            }
            float2 g0 = make_float2(0.f, 0.f), q0 = g0, q1 = g0, q2 = g0, w0 = g0, w1 = g0, w2 = g0, v0 = g0,
                   v1 = g0, v2 = g0;
#pragma unroll 1
            for (int bk = 0; bk < M; ++bk) {
              const float2 rz = make_float2((float)(tz0 - s_sn[2 * M + bk]), (float)(tz1 - s_sn[2 * M + bk]));
              const float2 prz = mul2(pz, rz);
              const float2 rzz = fma2(rz, rz, eps);
#pragma unroll
              for (int bj = 0; bj < M; ++bj) {
                const float2 P = fma2(py, ryv[bj], prz);
                const float2 A = fma2(ryv[bj], ryv[bj], rzz);
                const float4 *pb = pk + 5 * M * (bj + M * bk);
#pragma unroll
                for (int bi = 0; bi < M; ++bi) {
                  const float2 tt = add2(P, prx[bi]);
                  const float2 d = fma2(tt, tt, add2(A, rx2[bi]));
                  const float2 sv = rsqrt2(d);
                  float2 s3 = mul2(mul2(sv, sv), sv);
                  if constexpr (MASK) {
                    s3.x = d.x > (float)kEps64 ? s3.x : 0.f;
                    s3.y = d.y > (float)kEps64 ? s3.y : 0.f;
                  }
                  const float4 e0 = pb[5 * bi], e1 = pb[5 * bi + 1], e2 = pb[5 * bi + 2], e3 = pb[5 * bi + 3],
                               e4 = pb[5 * bi + 4];
                  g0 = fma2(s3, lo2(e0), g0);
                  q0 = fma2(s3, hi2(e0), q0);
                  q1 = fma2(s3, lo2(e1), q1);
                  q2 = fma2(s3, hi2(e1), q2);
                  w0 = fma2(s3, lo2(e2), w0);
                  w1 = fma2(s3, hi2(e2), w1);
                  w2 = fma2(s3, lo2(e3), w2);
                  v0 = fma2(s3, hi2(e3), v0);
                  v1 = fma2(s3, lo2(e4), v1);
                  v2 = fma2(s3, hi2(e4), v2);
                }
              }
            }
            // this source's E and B at both nodes: E = x' G - Q, B = W x x' - V, folded per
            // source into the compensated sums
            const float2 xa = make_float2((float)tx0, (float)tx1), ya = make_float2((float)ty0, (float)ty1),
                         za = make_float2((float)tz0, (float)tz1);
            kahan_add2(ks[q][0], kc[q][0], sub2(mul2(xa, g0), q0));
            kahan_add2(ks[q][1], kc[q][1], sub2(mul2(ya, g0), q1));
            kahan_add2(ks[q][2], kc[q][2], sub2(mul2(za, g0), q2));
            kahan_add2(ks[q][3], kc[q][3], sub2(sub2(mul2(w1, za), mul2(w2, ya)), v0));
            kahan_add2(ks[q][4], kc[q][4], sub2(sub2(mul2(w2, xa), mul2(w0, za)), v1));
            kahan_add2(ks[q][5], kc[q][5], sub2(sub2(mul2(w0, ya), mul2(w1, xa)), v2));
          }
        }
      }
      __syncthreads();  // the packed data and buffer bb are rewritten later
    }
  }
  float *out = loc + (int64_t)t * 6 * NN;
#pragma unroll
  for (int q = 0; q < TPP; ++q) {
    const int k = tid + q * BT;
    if (k < NP) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        float o0 = (float)((double)ks[q][c].x - (double)kc[q][c].x);
        if (accumulate) o0 += out[c * NN + k];
        out[c * NN + k] = o0;
        if (k + NP < NN) {
          float o1 = (float)((double)ks[q][c].y - (double)kc[q][c].y);
          if (accumulate) o1 += out[c * NN + k + NP];
          out[c * NN + k + NP] = o1;
        }
      }
    }
  }
}

template <int NDEG, bool MASK>
int launch_m2l_fp64(Ctx *ctx, bool accumulate) {
  using S = M2LShape<NDEG>;
  const int rec = 4 * S::NN * 8 + S::NS * 8;
  const int smem = 2 * rec + 3 * S::NN * 4 * 8;
  auto kern = m2l_kernel<NDEG, MASK>;
  FMM_TRY(opt_in_smem(ctx, kern, smem));
  if (ctx->nc > 0)
    kern<<<(unsigned)ctx->nc, S::BT, smem, ctx->stream>>>(
        ctx->get<int>("m2l_ptr"), ctx->get<int>("m2l_src"), ctx->get<double>("nodes"), ctx->get<double>("bbox"),
        ctx->get<double>("mom64"), ctx->get<double>("loc64"), ctx->get<double>("consts"), accumulate ? 1 : 0,
        ctx->d_status);
  return ctx->check_launch("m2l_kernel");
}

template <int NDEG, bool MASK>
int launch_m2l_mixed(Ctx *ctx, bool accumulate) {
  using S = M2LShape2<NDEG>;
  auto kern = m2l_x2_kernel<NDEG, MASK>;
  FMM_TRY(opt_in_smem(ctx, kern, S::SMEM));
  if (ctx->nc > 0)
    kern<<<(unsigned)ctx->nc, S::BT, S::SMEM, ctx->stream>>>(
        ctx->get<int>("m2l_ptr"), ctx->get<int>("m2l_src"), ctx->get<double>("nodes"), ctx->get<double>("bbox"),
        ctx->get<float>("mom32"), ctx->get<float>("loc32"), ctx->get<double>("consts"), accumulate ? 1 : 0,
        ctx->d_status);
  return ctx->check_launch("m2l_x2_kernel");
}

template <int NDEG>
int launch_m2l_n(Ctx *ctx, bool mixed, bool accumulate) {
  // coincident target/source nodes need eta > 1/2 (admissible: max(r1,r2) < eta R)
  const bool mask = !(ctx->eta <= 0.5);
  if (mixed) return mask ? launch_m2l_mixed<NDEG, true>(ctx, accumulate) : launch_m2l_mixed<NDEG, false>(ctx, accumulate);
  return mask ? launch_m2l_fp64<NDEG, true>(ctx, accumulate) : launch_m2l_fp64<NDEG, false>(ctx, accumulate);
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
