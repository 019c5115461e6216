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
// node offsets are formed in FP64 and rounded, and per-source FP32 partial sums
// are added into per-thread FP64 sums held in shared memory.
//
// Mixed form on the tensor cores (m2l_tc_kernel, degree n <= 4, eta <= 1/2; an
// opt-in engine -- at n = 4 the M2L stage measures 102 ms against 95 ms for the
// packed CUDA-core kernel on 2^24 particles: the tensor cores take only the 71 %
// of the pairs whose factored sums are accurate, the CUDA-core kernel still runs
// the rest, and the per-chunk hand-off between the evaluating warps and the MMA
// issuer keeps the rsqrt pipe at about a third of its rate): per source the
// M2L is a (target nodes) x (source nodes) kernel matrix K times the 10 packed
// per-source-node columns V below, so the 10 accumulations per evaluation run
// as tcgen05 TF32 MMAs.  Each thread owns one target node = one TMEM lane: it
// evaluates its row of K two source nodes per packed FP32x2 instruction (3 for
// the denominator, rsqrt, 2 for s^3) in chunks of 16 source nodes, splits every
// value into TF32 hi + lo and stores both into a TMEM A buffer (three in
// rotation); one thread issues the MMAs
// D += [K_hi; K_lo] x [V_hi | V_lo] (M = 128, N = 32, K = 8) against V held in
// shared memory.  After each source D is read back (tcgen05.ld), its four
// hi/lo products are summed and E = x'G - Q, B = W x x' - V is folded into
// Kahan-compensated FP32 accumulators.
#include "device_util.cuh"
#include "kernels.cuh"
#include "packed.cuh"
#include "tcgen05.cuh"

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
// MASK (eta > 1/2, coincident nodes admissible): the factored sums x'G - Q would
// cancel catastrophically for nodes much closer than the box size, so E and B
// are accumulated directly (s^3 Gamma R, s^3 M x R) from (G,G,M0,M0) (M1,M1,M2,M2).
template <int NDEG>
struct M2LShape2 {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int NP = (NN + 1) / 2;             // target-node pairs
  static constexpr int TPP = (NP + 511) / 512;        // pairs per thread
  static constexpr int BT = (((NP + TPP - 1) / TPP) + 31) / 32 * 32;
  static constexpr int REC = 4 * NN * 4 + NS * 8;     // raw FP32 moments then node coordinates
  // double buffer + packed node data (MASK uses 2/5) + per-thread FP64 sums of E, B of both targets
  static constexpr int SMEM = 2 * REC + 5 * NN * 16 + TPP * 12 * BT * 8;
};

template <int NDEG, bool MASK>
__global__ void __launch_bounds__(M2LShape2<NDEG>::BT)
    m2l_x2_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const double *__restrict__ nodes,
                  const double *__restrict__ bbox, const float *__restrict__ mom, float *__restrict__ loc,
                  const double *__restrict__ consts, int accumulate, int *__restrict__ status,
                  const uint32_t *__restrict__ srcf) {
  using S = M2LShape2<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, NP = S::NP, TPP = S::TPP, BT = S::BT, REC = S::REC;
  constexpr int MOM_BYTES = 4 * NN * 4;
  extern __shared__ __align__(16) unsigned char smem[];
  float4 *pk = (float4 *)(smem + 2 * REC);  // 5*NN packed entries
  // [q][c][BT]: c < 6 the first target's E, B, c >= 6 the second's (FP64 sums over sources)
  double *s_acc = (double *)(smem + 2 * REC + 5 * NN * 16);
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_sn[3 * M];  // source node offsets from the target centre
  __shared__ int s_dir[2];        // per staged source: direct sums (the boxes nearly touch)

  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);

  for (int e = 0; e < TPP * 12; ++e) s_acc[e * BT + tid] = 0.0;
  // one source's FP32 partial sums (both targets) into the FP64 sums
  auto fold = [&](int q, int c, float2 v) {
    s_acc[(q * 12 + c) * BT + tid] += (double)v.x;
    s_acc[(q * 12 + 6 + c) * BT + tid] += (double)v.y;
  };

  if (np > 0) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int k, int bb) {
      // factored sums unless the two boxes nearly touch (factored_ok); at N = 2^24 the
      // direct pairs make the M2L about 2 % slower and its error ~20x smaller.  srcf, when
      // given, holds the source with that decision in its top bit (m2l_dirflag_kernel), so
      // that this thread does not evaluate it between its own sweeps.  Written before the
      // arrive, whose release orders it for the threads that wait on bar[bb].
      int s;
      if (srcf) {
        const uint32_t v = srcf[p0 + k];
        s = (int)(v & 0x7FFFFFFFu);
        s_dir[bb] = MASK || (v >> 31) != 0u;
      } else {
        s = src[p0 + k];
        s_dir[bb] = MASK || !factored_ok(bbox + 6 * (int64_t)s, tb, cx, cy, cz);
      }
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
      const bool dir = s_dir[bb] != 0;
      if (ok) {
        for (int e = tid; e < 3 * M; e += BT) {
          const int d = e / M;
          s_sn[e] = SN[e] - (d == 0 ? cx : (d == 1 ? cy : cz));
        }
        for (int b = tid; b < NN; b += BT) {
          const int bi = b % M, bj = (b / M) % M, bk = b / (M * M);
          const float xb = (float)(SN[bi] - cx), yb = (float)(SN[M + bj] - cy), zb = (float)(SN[2 * M + bk] - cz);
          const float g = G[b], m0 = G[NN + b], m1 = G[2 * NN + b], m2 = G[3 * NN + b];
          if (dir) {
            float4 *o = pk + 2 * b;
            o[0] = make_float4(g, g, m0, m0);
            o[1] = make_float4(m1, m1, m2, m2);
          } else {
            const float c0 = m1 * zb - m2 * yb, c1 = m2 * xb - m0 * zb, c2 = m0 * yb - m1 * xb;
            float4 *o = pk + 5 * b;
            o[0] = make_float4(g, g, g * xb, g * xb);
            o[1] = make_float4(g * yb, g * yb, g * zb, g * zb);
            o[2] = make_float4(m0, m0, m1, m1);
            o[3] = make_float4(m2, m2, c0, c0);
            o[4] = make_float4(c1, c1, c2, c2);
          }
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
            // this source's sweep over its nodes (bk outer, bi inner)
            auto sweep = [&](auto DIRECT) {
              constexpr bool D = decltype(DIRECT)::value;
              float2 prx[M], rx2[M], ryv[M];
              float2 rxv[D ? M : 1];
#pragma unroll
              for (int b = 0; b < M; ++b) {
                const float2 rx = make_float2((float)(tx0 - s_sn[b]), (float)(tx1 - s_sn[b]));
                prx[b] = mul2(px, rx);
                rx2[b] = mul2(rx, rx);
                ryv[b] = make_float2((float)(ty0 - s_sn[M + b]), (float)(ty1 - s_sn[M + b]));
                if constexpr (D) rxv[b] = rx;
              }
              // factored: (G, Q, W, V) sums; direct: E and B accumulated
              float2 g0 = make_float2(0.f, 0.f), q0 = g0, q1 = g0, q2 = g0, w0 = g0, w1 = g0, w2 = g0, v0 = g0,
                     v1 = g0, v2 = g0;
#pragma unroll 1
              for (int bk = 0; bk < M; ++bk) {
                const float2 rz = make_float2((float)(tz0 - s_sn[2 * M + bk]), (float)(tz1 - s_sn[2 * M + bk]));
                const float2 prz = mul2(pz, rz);
                const float2 rzz = fma2(rz, rz, eps);
#pragma unroll
                for (int bj = 0; bj < M; ++bj) {
                  const float2 ry = ryv[bj];
                  const float2 P = fma2(py, ry, prz);
                  const float2 A = fma2(ry, ry, rzz);
#pragma unroll
                  for (int bi = 0; bi < M; ++bi) {
                    const float2 tt = add2(P, prx[bi]);
                    const float2 d = fma2(tt, tt, add2(A, rx2[bi]));
                    const float2 sv = rsqrt2(d);
                    float2 s3 = mul2(mul2(sv, sv), sv);
                    if constexpr (D) {
                      if constexpr (MASK) {
                        s3.x = d.x > (float)kEps64 ? s3.x : 0.f;
                        s3.y = d.y > (float)kEps64 ? s3.y : 0.f;
                      }
                      const float4 *pb = pk + 2 * (bi + M * (bj + M * bk));
                      const float4 e0 = pb[0], e1 = pb[1];
                      const float2 G = lo2(e0), M0 = hi2(e0), M1 = lo2(e1), M2 = hi2(e1);
                      const float2 kx = mul2(s3, rxv[bi]), ky = mul2(s3, ry), kz = mul2(s3, rz);  // K
                      g0 = fma2(G, kx, g0);  // E = G K
                      q0 = fma2(G, ky, q0);
                      q1 = fma2(G, kz, q1);
                      w0 = fma2(M1, kz, w0);  // B = M x K as (w - v)
                      v0 = fma2(M2, ky, v0);
                      w1 = fma2(M2, kx, w1);
                      v1 = fma2(M0, kz, v1);
                      w2 = fma2(M0, ky, w2);
                      v2 = fma2(M1, kx, v2);
                    } else {
                      const float4 *pb = pk + 5 * (bi + M * (bj + M * bk));
                      const float4 e0 = pb[0], e1 = pb[1], e2 = pb[2], e3 = pb[3], e4 = pb[4];
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
              }
              if constexpr (D) {
                fold(q, 0, g0);
                fold(q, 1, q0);
                fold(q, 2, q1);
                fold(q, 3, sub2(w0, v0));
                fold(q, 4, sub2(w1, v1));
                fold(q, 5, sub2(w2, v2));
              } else {
                // this source's E and B at both nodes: E = x' G - Q, B = W x x' - V
                const float2 xa = make_float2((float)tx0, (float)tx1), ya = make_float2((float)ty0, (float)ty1),
                             za = make_float2((float)tz0, (float)tz1);
                fold(q, 0, sub2(mul2(xa, g0), q0));
                fold(q, 1, sub2(mul2(ya, g0), q1));
                fold(q, 2, sub2(mul2(za, g0), q2));
                fold(q, 3, sub2(sub2(mul2(w1, za), mul2(w2, ya)), v0));
                fold(q, 4, sub2(sub2(mul2(w2, xa), mul2(w0, za)), v1));
                fold(q, 5, sub2(sub2(mul2(w0, ya), mul2(w1, xa)), v2));
              }
            };
            if (dir)
              sweep(std::integral_constant<bool, true>{});
            else if constexpr (!MASK)
              sweep(std::integral_constant<bool, false>{});
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
        float o0 = (float)s_acc[(q * 12 + c) * BT + tid];
        if (accumulate) o0 += out[c * NN + k];
        out[c * NN + k] = o0;
        if (k + NP < NN) {
          float o1 = (float)s_acc[(q * 12 + 6 + c) * BT + tid];
          if (accumulate) o1 += out[c * NN + k + NP];
          out[c * NN + k + NP] = o1;
        }
      }
    }
  }
}

// srcf[k] = src[k] with the top bit set when target t's pair with it takes the direct sums
// (factored_ok false), for every row t of the CSR lists; one thread per target.
__global__ void m2l_dirflag_kernel(int64_t nc, const int *__restrict__ ptr, const int *__restrict__ src,
                                   const double *__restrict__ bbox, uint32_t *__restrict__ srcf) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc) return;
  const double *tb = bbox + 6 * t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);
  for (int k = ptr[t]; k < ptr[t + 1]; ++k) {
    const int s = src[k];
    srcf[k] = (uint32_t)s | (factored_ok(bbox + 6 * (int64_t)s, tb, cx, cy, cz) ? 0u : 0x80000000u);
  }
}

// ---------------------------------------------------------------- tensor-core mixed form
// The K dimension (source nodes) is ordered for packed FP32x2 evaluation.  Node b lies
// on x-row r = b / M = bj + M bk at bi = b % M.  The rows are paired (2 rp, 2 rp + 1), and
// column 2 q + lane with q = M rp + bi holds row 2 rp + lane at bi.  One packed
// evaluation then forms both columns of a pair: the two lanes share bi (the hoisted
// x-parts of the denominator) and take their rows' y/z parts.  A row past the last
// (M^2 odd) and the columns past 2 M NRP are zero in V.
template <int NDEG>
struct M2LShapeTC {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;                 // <= 125
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int CH = 16;                        // K columns per chunk (one tcgen05.st.x16)
  static constexpr int NR = M * M;                     // x-rows
  static constexpr int NRP = (NR + 1) / 2;             // row pairs
  static constexpr int NQ = M * NRP;                   // packed column pairs
  static constexpr int NCH = (2 * NQ + CH - 1) / CH;
  static constexpr int KP = NCH * CH;                  // padded K
  static constexpr int NBUF = 3;                       // TMEM A buffers in rotation
  static constexpr int NMMA = 32;                      // D columns: 0..9 V_hi products, 16..25 V_lo
  static constexpr uint32_t LBO = (NMMA / 8) * 128;    // bytes between 4-element K groups of V
  static constexpr uint32_t SBO = 128;                 // bytes between 8-row groups of V
  static constexpr int BBYTES = (KP / 4) * (int)LBO;   // one V operand
  static constexpr int MOM_BYTES = 4 * NN * 4;
  static constexpr int REC = MOM_BYTES + NS * 8;       // raw FP32 moments then node coordinates
  static constexpr int SMEM_USED = 2 * BBYTES + 2 * REC;
  // at most 4 CTAs per SM (3 by registers), so that 4 x 128 TMEM columns never exceed the SM's 512
  static constexpr int SMEM = SMEM_USED > 48 * 1024 ? SMEM_USED : 48 * 1024;
  static constexpr uint32_t TMEM_COLS = 128;           // D [0,32), A buffer b at 32 + 32 b (hi 16, lo 16)
  __host__ __device__ static constexpr int col(int b) {
    return 2 * (M * ((b / M) / 2) + b % M) + (b / M) % 2;
  }
};

// Warp roles: warps 0-3 evaluate K (thread = target node = TMEM lane) and
// arrive on full[b] once their slice of A buffer b is in TMEM; warp 4 waits on
// full[b], issues the chunk's MMAs and commits them to empty[b], which the
// evaluating warps wait on before reusing buffer b.  The evaluating warps meet
// in one named barrier per source (V and the node offsets written); they read
// a source's D while evaluating the next source's first chunk, which the MMAs
// overwrite only after every warp has arrived for that chunk.
constexpr int kTcThreads = 160;

template <int NDEG>
// Three CTAs per SM: 125 registers without spills (a bound of four spilled and ran 9 % slower).
__global__ void __launch_bounds__(kTcThreads, 3)
    m2l_tc_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const double *__restrict__ nodes,
                  const double *__restrict__ bbox, const float *__restrict__ mom, float *__restrict__ loc,
                  const double *__restrict__ consts, int accumulate, int *__restrict__ status) {
  using S = M2LShapeTC<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, CH = S::CH, NR = S::NR, NQ = S::NQ, NCH = S::NCH;
  constexpr int NBUF = S::NBUF, REC = S::REC, MOM_BYTES = S::MOM_BYTES;
  constexpr uint32_t LBO = S::LBO, SBO = S::SBO;
  constexpr uint32_t IDESC = idesc_tf32(128, S::NMMA);
  constexpr int kEvalBar = 1;  // named barrier of the 128 evaluating threads
  static_assert(NN <= 128 && 2 * NQ <= S::KP, "one target node per TMEM lane, every column pair in a chunk");
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sRaw = smem + 2 * S::BBYTES;  // 2 raw source records (TMA double buffer)
  __shared__ __align__(8) uint64_t bar_tma[2];
  __shared__ __align__(8) uint64_t bar_full[NBUF];
  __shared__ __align__(8) uint64_t bar_empty[NBUF];
  __shared__ __align__(8) uint64_t bar_drain;
  __shared__ uint32_t s_tmem;
  __shared__ float s_sn[2][3 * M];  // source node offsets from the target centre, by source parity

  const int tid = threadIdx.x, warp = tid >> 5;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);
  const int a = tid < NN ? tid : NN - 1;  // rows past NN repeat a node and are not written
  const float xa = (float)(tn[a % M] - cx), ya = (float)(tn[M + (a / M) % M] - cy),
              za = (float)(tn[2 * M + a / (M * M)] - cz);

  float ks[6], kc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) ks[c] = kc[c] = 0.f;

  if (np > 0) {
    for (int e = tid; e < 2 * S::BBYTES / 16; e += kTcThreads)
      reinterpret_cast<float4 *>(smem)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (warp == 0) {
      tmem_alloc(&s_tmem, S::TMEM_COLS);
      tmem_relinquish();
    }
    auto issue = [&](int k, int rb) {
      const int s = src[p0 + k];
      unsigned char *dst = sRaw + rb * REC;
      mbar_arrive_expect_tx(&bar_tma[rb], REC);
      bulk_g2s(dst, mom + (int64_t)s * 4 * NN, MOM_BYTES, &bar_tma[rb]);
      bulk_g2s(dst + MOM_BYTES, nodes + (int64_t)s * NS, NS * 8, &bar_tma[rb]);
    };
    int issued = 0;  // TMA copies issued (thread 0)
    if (tid == 0) {
      mbar_init(&bar_tma[0], 1);
      mbar_init(&bar_tma[1], 1);
      for (int b = 0; b < NBUF; ++b) {
        mbar_init(&bar_full[b], 4);  // one arrival per evaluating warp
        mbar_init(&bar_empty[b], 1);
      }
      mbar_init(&bar_drain, 1);
      fence_mbar_init();
      issue(0, 0);
      issued = 1;
      if (np > 1) {
        issue(1, 1);
        issued = 2;
      }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = s_tmem;

    if (warp == 4) {
      // ---------------- MMA issuer
      if ((tid & 31) == 0) {
        bool ok = true;
        int k = 0;
        for (int i = 0; i < np && ok; ++i) {
          const unsigned char *sV = smem + (i & 1) * S::BBYTES;
          for (int c = 0; c < NCH; ++c, ++k) {
            const int b = k % NBUF;
            if (!mbar_wait_bounded(&bar_full[b], (uint32_t)((k / NBUF) & 1), status)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t acol = 32 + 32 * (uint32_t)b;
#pragma unroll
            for (int kstep = 0; kstep < CH / 8; ++kstep) {
              const uint64_t bd = smem_desc_noswizzle(sV + ((CH * c + 8 * kstep) / 4) * LBO, LBO, SBO);
              mma_tf32_ts(tbase, tbase + acol + 8 * kstep, bd, IDESC, (c > 0 || kstep > 0) ? 1u : 0u);
              mma_tf32_ts(tbase, tbase + acol + 16 + 8 * kstep, bd, IDESC, 1u);
            }
            mma_commit(&bar_empty[b]);
          }
        }
        // every MMA issued has completed before TMEM is released
        mma_commit(&bar_drain);
        mbar_wait_bounded(&bar_drain, 0, status);
      }
    } else {
      // ---------------- K evaluation (128 threads)
      const uint32_t lane = (uint32_t)(32 * warp) << 16;
      const float px = (float)consts[0], py = (float)consts[1], pz = (float)consts[2];
      const float eps = (float)kEps64;
      bool fail = false;  // a bounded wait gave up (uniform after each per-source barrier)

      // D holds one source's sums: D[n] + D[16 + n] = (K_hi + K_lo)(V_hi + V_lo)
      auto readout = [&](int last_chunk) {
        if (fail) return;
        if (!mbar_wait_bounded(&bar_empty[last_chunk % NBUF], (uint32_t)((last_chunk / NBUF) & 1), status)) {
          fail = true;
          return;
        }
        tc_fence_after();
        uint32_t d0[16], d1[16];
        tmem_ld16(tbase + lane, d0);
        tmem_ld16(tbase + lane + 16, d1);
        tmem_wait_ld();
        float sum[10];
#pragma unroll
        for (int n = 0; n < 10; ++n) sum[n] = __uint_as_float(d0[n]) + __uint_as_float(d1[n]);
        const float g0 = sum[0], q0 = sum[1], q1 = sum[2], q2 = sum[3], w0 = sum[4], w1 = sum[5], w2 = sum[6];
        const float v0 = sum[7], v1 = sum[8], v2 = sum[9];
        const float part[6] = {xa * g0 - q0, ya * g0 - q1, za * g0 - q2,
                               (w1 * za - w2 * ya) - v0, (w2 * xa - w0 * za) - v1, (w0 * ya - w1 * xa) - v2};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const float y = part[q] - kc[q];
          const float tsum = ks[q] + y;
          kc[q] = (tsum - ks[q]) - y;
          ks[q] = tsum;
        }
      };

      int g = 0;         // chunks evaluated so far (global over sources)
      int consumed = 0;  // TMA copies waited for
      for (int i = 0; i < np; ++i) {
        const int rb = i & 1;
        unsigned char *sV = smem + rb * S::BBYTES;  // V of source i (source i-1's MMAs may still read the other)
        float *sn = s_sn[rb];
        const bool got = !fail && mbar_wait_bounded(&bar_tma[rb], (uint32_t)((i >> 1) & 1), status);
        ++consumed;
        fail |= !got;
        if (got) {
          const float *G = (const float *)(sRaw + rb * REC);
          const double *SN = (const double *)(sRaw + rb * REC + MOM_BYTES);
          if (tid < 3 * M) {
            const int d = tid / M;
            sn[tid] = (float)(SN[tid] - (d == 0 ? cx : (d == 1 ? cy : cz)));
          }
          // V operand: 10 columns per source node, split into TF32 hi (rows 0..9) and lo (rows 16..25)
          for (int b = tid; b < NN; b += 128) {
            const int bi = b % M, bj = (b / M) % M, bk = b / (M * M);
            const float xb = (float)(SN[bi] - cx), yb = (float)(SN[M + bj] - cy), zb = (float)(SN[2 * M + bk] - cz);
            const float gm = G[b], m0 = G[NN + b], m1 = G[2 * NN + b], m2 = G[3 * NN + b];
            const float v[10] = {gm, gm * xb, gm * yb, gm * zb, m0, m1, m2,
                                 m1 * zb - m2 * yb, m2 * xb - m0 * zb, m0 * yb - m1 * xb};
            const int k = S::col(b);
            unsigned char *colp = sV + (k / 4) * LBO + (k % 4) * 4;
#pragma unroll
            for (int c = 0; c < 10; ++c) {
              const float h = tf32_hi(v[c]);
              *(float *)(colp + (c / 8) * SBO + (c % 8) * 16) = h;
              *(float *)(colp + ((16 + c) / 8) * SBO + ((16 + c) % 8) * 16) = v[c] - h;
            }
          }
        }
        fence_proxy_async_smem();
        // V and the node offsets written, raw buffer rb consumed
        if (bar_or(kEvalBar, 128, fail)) {
          fail = true;
          break;
        }
        if (tid == 0 && issued < np) {
          fence_proxy_async_smem();
          issue(issued, issued & 1);
          ++issued;
        }
        // the x-parts of the denominator per bi (both lanes), the y/z offsets per row
        float2 prx[M], rx2[M];
        float ryv[M], rzv[M];
#pragma unroll
        for (int b = 0; b < M; ++b) {
          const float rx = xa - sn[b];
          prx[b] = dup2(px * rx);
          rx2[b] = dup2(rx * rx);
          ryv[b] = ya - sn[M + b];
          rzv[b] = za - sn[2 * M + b];
        }
        const float2 py2 = dup2(py), pz2 = dup2(pz), eps2 = dup2(eps);
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
          const int bsel = g % NBUF;
          if (g >= NBUF && !fail) {
            fail |= !mbar_wait_bounded(&bar_empty[bsel], (uint32_t)(((g / NBUF) - 1) & 1), status);
            tc_fence_after();
          }
          uint32_t kh[CH], kl[CH];
#pragma unroll
          for (int m = 0; m < CH / 2; ++m) {
            const int q = (CH / 2) * c + m;  // column pair: rows 2 rp, 2 rp + 1 at bi
            if (q < NQ) {
              const int rp = q / M, bi = q % M;
              const int r0 = 2 * rp, r1 = 2 * rp + 1 < NR ? 2 * rp + 1 : 2 * rp;  // a missing row repeats r0
              const float2 ry = make_float2(ryv[r0 % M], ryv[r1 % M]), rz = make_float2(rzv[r0 / M], rzv[r1 / M]);
              const float2 P = fma2(py2, ry, mul2(pz2, rz));
              const float2 A = fma2(ry, ry, fma2(rz, rz, eps2));
              const float2 tt = add2(P, prx[bi]);
              const float2 d = fma2(tt, tt, add2(A, rx2[bi]));
              const float2 sv = rsqrt2(d);
              const float2 kv = mul2(mul2(sv, sv), sv);
              const float2 h = make_float2(tf32_hi(kv.x), tf32_hi(kv.y));
              const float2 lo = sub2(kv, h);
              kh[2 * m] = __float_as_uint(h.x);
              kh[2 * m + 1] = __float_as_uint(h.y);
              kl[2 * m] = __float_as_uint(lo.x);
              kl[2 * m + 1] = __float_as_uint(lo.y);
            } else {
              kh[2 * m] = kh[2 * m + 1] = kl[2 * m] = kl[2 * m + 1] = 0u;
            }
          }
          // the previous source's D, before this source's first chunk lets the MMAs overwrite it
          if (c == 0 && i > 0) readout(g - 1);
          const uint32_t acol = 32 + 32 * (uint32_t)bsel;
          tmem_st16(tbase + lane + acol, kh);
          tmem_st16(tbase + lane + acol + 16, kl);
          tmem_wait_st();
          tc_fence_before();
          __syncwarp();
          if ((tid & 31) == 0) mbar_arrive(&bar_full[bsel]);
          ++g;
        }
      }
      if (g > 0) readout(g - 1);  // the last source
      if (tid == 0)
        for (int k = consumed; k < issued; ++k) mbar_wait_bounded(&bar_tma[k & 1], (uint32_t)((k >> 1) & 1), status);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
      tc_fence_after();
      tmem_dealloc(tbase, S::TMEM_COLS);
    }
  }
  if (tid < NN) {
    float *out = loc + (int64_t)t * 6 * NN;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      float o = (float)((double)ks[c] - (double)kc[c]);
      if (accumulate) o += out[c * NN + tid];
      out[c * NN + tid] = o;
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
        ctx->get<int>(ctx->m2l_ptr_key), ctx->get<int>(ctx->m2l_src_key), ctx->get<double>("nodes"), ctx->get<double>("bbox"),
        ctx->get<double>("mom64"), ctx->get<double>("loc64"), ctx->get<double>("consts"), accumulate ? 1 : 0,
        ctx->d_status);
  return ctx->check_launch("m2l_kernel");
}

// The tensor-core kernel evaluates the factored sums only, so each target's row of the
// M2L lists is split by factored_ok: [0] the pairs for the tensor cores, [1] the pairs
// whose boxes nearly touch, which the CUDA-core kernel then adds with its direct sums.
// cnt holds 2 (nc + 1) entries, the last of each half 0.
template <int M>
__global__ void m2l_split_count_kernel(int64_t nc, const int *__restrict__ ptr, const int *__restrict__ src,
                                       const double *__restrict__ nodes, const double *__restrict__ bbox,
                                       int *__restrict__ cnt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > nc) return;
  int a = 0, b = 0;
  if (t < nc) {
    const double *tb = bbox + 6 * t;
    const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);
    for (int k = ptr[t]; k < ptr[t + 1]; ++k) {
      if (factored_ok(bbox + 6 * (int64_t)src[k], tb, cx, cy, cz))
        ++a;
      else
        ++b;
    }
  }
  cnt[t] = a;
  cnt[nc + 1 + t] = b;
}

template <int M>
__global__ void m2l_split_write_kernel(int64_t nc, const int *__restrict__ ptr, const int *__restrict__ src,
                                       const double *__restrict__ nodes, const double *__restrict__ bbox,
                                       const int *__restrict__ ptr2, int *__restrict__ src_a, int *__restrict__ src_b) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nc) return;
  const double *tb = bbox + 6 * t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);
  int oa = ptr2[t], ob = ptr2[nc + 1 + t];
  for (int k = ptr[t]; k < ptr[t + 1]; ++k) {
    const int s = src[k];
    if (factored_ok(bbox + 6 * (int64_t)s, tb, cx, cy, cz))
      src_a[oa++] = s;
    else
      src_b[ob++] = s;
  }
}

template <int NDEG>
int launch_m2l_tc(Ctx *ctx, bool accumulate) {
  using S = M2LShapeTC<NDEG>;
  constexpr int M = NDEG + 1;
  const int64_t nc = ctx->nc;
  if (nc <= 0) return FMMB200_OK;
  const int *ptr = ctx->get<int>(ctx->m2l_ptr_key), *src = ctx->get<int>(ctx->m2l_src_key);
  const double *nodes = ctx->get<double>("nodes"), *bbox = ctx->get<double>("bbox");
  int *cnt, *ptr2, *src_a, *src_b;
  FMM_TRY(ctx->ensure("tc_split_cnt", 2 * (nc + 1), &cnt));
  FMM_TRY(ctx->ensure("tc_split_ptr", 2 * (nc + 1), &ptr2));
  m2l_split_count_kernel<M><<<ceil_div(nc + 1, 256), 256, 0, ctx->stream>>>(nc, ptr, src, nodes, bbox, cnt);
  FMM_TRY(ctx->check_launch("m2l_split_count_kernel"));
  int64_t na = 0, nb = 0;
  FMM_TRY(exclusive_scan_i32(ctx, cnt, ptr2, nc + 1, &na));
  FMM_TRY(exclusive_scan_i32(ctx, cnt + nc + 1, ptr2 + nc + 1, nc + 1, &nb));
  FMM_TRY(ctx->ensure("tc_split_src_a", na > 0 ? na : 1, &src_a));
  FMM_TRY(ctx->ensure("tc_split_src_b", nb > 0 ? nb : 1, &src_b));
  m2l_split_write_kernel<M><<<ceil_div(nc, 256), 256, 0, ctx->stream>>>(nc, ptr, src, nodes, bbox, ptr2, src_a,
                                                                          src_b);
  FMM_TRY(ctx->check_launch("m2l_split_write_kernel"));
  auto kern = m2l_tc_kernel<NDEG>;
  FMM_TRY(opt_in_smem(ctx, kern, S::SMEM));
  kern<<<(unsigned)nc, kTcThreads, S::SMEM, ctx->stream>>>(ptr2, src_a, nodes, bbox, ctx->get<float>("mom32"),
                                                            ctx->get<float>("loc32"), ctx->get<double>("consts"),
                                                            accumulate ? 1 : 0, ctx->d_status);
  FMM_TRY(ctx->check_launch("m2l_tc_kernel"));
  if (nb == 0) return FMMB200_OK;
  using S2 = M2LShape2<NDEG>;
  auto k2 = m2l_x2_kernel<NDEG, false>;
  FMM_TRY(opt_in_smem(ctx, k2, S2::SMEM));
  k2<<<(unsigned)nc, S2::BT, S2::SMEM, ctx->stream>>>(ptr2 + nc + 1, src_b, nodes, bbox, ctx->get<float>("mom32"),
                                                      ctx->get<float>("loc32"), ctx->get<double>("consts"), 1,
                                                      ctx->d_status, nullptr);
  return ctx->check_launch("m2l_x2_kernel");
}

template <int NDEG, bool MASK>
int launch_m2l_mixed(Ctx *ctx, bool accumulate) {
  if constexpr (NDEG <= 4 && !MASK) {
    // the tensor-core form is factored (E = x'G - Q): only where nodes cannot coincide,
    // and the pairs whose boxes nearly touch still go to the CUDA cores
    if (ctx->m2l_engine == FMMB200_M2L_TENSOR_CORES) return launch_m2l_tc<NDEG>(ctx, accumulate);
  }
  using S = M2LShape2<NDEG>;
  auto kern = m2l_x2_kernel<NDEG, MASK>;
  FMM_TRY(opt_in_smem(ctx, kern, S::SMEM));
  const int *ptr = ctx->get<int>(ctx->m2l_ptr_key), *src = ctx->get<int>(ctx->m2l_src_key);
  uint32_t *srcf = nullptr;
  if (!MASK && ctx->nc > 0 && ctx->nm2l > 0) {  // every pair's factored / direct decision, up front
    FMM_TRY(ctx->ensure("m2l_srcf", ctx->nm2l, &srcf));
    m2l_dirflag_kernel<<<ceil_div(ctx->nc, 128), 128, 0, ctx->stream>>>(ctx->nc, ptr, src, ctx->get<double>("bbox"), srcf);
    FMM_TRY(ctx->check_launch("m2l_dirflag_kernel"));
  }
  if (ctx->nc > 0)
    kern<<<(unsigned)ctx->nc, S::BT, S::SMEM, ctx->stream>>>(
        ptr, src, ctx->get<double>("nodes"), ctx->get<double>("bbox"), ctx->get<float>("mom32"), ctx->get<float>("loc32"),
        ctx->get<double>("consts"), accumulate ? 1 : 0, ctx->d_status, srcf);
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
