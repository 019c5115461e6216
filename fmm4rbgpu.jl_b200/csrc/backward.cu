// backward.cu -- hand-written adjoint of the whole field map (E, B) = F(x, u)
// with the tree and the interaction lists held fixed (no counterpart in the
// reference; the map is piecewise smooth in x through the bounding boxes).
//
// Reverse of the forward pipeline, all FP64:
//   L2P^T   leaf local adjoints  += sum_p a_p w(x_p);   x_p and leaf boxes get
//           the derivative of the interpolant
//   L2L^T   parent local adjoints += transferred child adjoints; child/parent
//           boxes through the node positions (levels ml .. 1)
//   M2L^T   per target cluster over the union of its list and its transpose:
//           node-position gradients, source-role moment adjoints, d/dp_avg
//   M2M^T   child moment adjoints += transferred parent adjoints; boxes (top-down)
//   P2M^T   x_p, u_p from the leaf moment adjoints; leaf boxes
//   P2P^T   per target leaf over the union list (near field recomputed)
//   boxes   bounding-box adjoints flow down the tree to the extremal particles,
//           p_avg's adjoint to every momentum, then the scatter to caller order.
//
// Box geometry: node i of [a, b] is a + t_i (b - a) and a Lagrange weight only
// depends on xi = (x - a)/(b - a), so for an evaluation point x with partial G:
// dL/da += (xi - 1) G, dL/db += -xi G; for a node of the cluster itself:
// dL/da += (1 - t_i) G_i, dL/db += t_i G_i.
#include <cmath>
#include <type_traits>

#include "device_util.cuh"
#include "interp_util.cuh"
#include "kernels.cuh"
#include "packed.cuh"

namespace fmmb200 {

namespace {

template <int NDEG>
struct BShape {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int BT = NN <= 64 ? 64 : (NN <= 512 ? ((NN + 31) / 32) * 32 : 512);
  static constexpr int NPT = (NN + BT - 1) / BT;
};

// block-wide sum of V doubles per thread into out (all threads get the result)
template <int V>
__device__ __forceinline__ void block_sum(double (&v)[V], double *s_red /* [32][V] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < V; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < V; ++k) s_red[wid * V + k] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < V; ++k) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += s_red[w * V + k];
    v[k] = s;
  }
  __syncthreads();
}

// ---------------------------------------------------------------- gather / init
// adj: a = amp * (dL/dE, dL/dB) in tree order (SoA); rec16: the particle record
// (x,y,z,gamma,ux,uy,uz,0) followed by (aE, aB, 0, 0) and two doubles of padding --
// kRecB = 18 doubles (144 bytes) per particle, so that the records that the lanes
// of a warp read at once in P2P^T fall on distinct shared-memory banks.
constexpr int kRecB = 18;
__global__ void adj_gather_kernel(int N, const uint32_t *__restrict__ perm, const double *__restrict__ ge,
                                  const double *__restrict__ gb, double amp, const double *__restrict__ prec,
                                  double *__restrict__ adj, double *__restrict__ rec16, double *__restrict__ gxu) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int64_t o = 3 * (int64_t)perm[p];
  double v[6];
  for (int q = 0; q < 3; ++q) {
    v[q] = amp * ge[o + q];
    v[3 + q] = amp * gb[o + q];
  }
  double *r = rec16 + kRecB * (int64_t)p;
  for (int q = 0; q < 8; ++q) r[q] = prec[8 * (int64_t)p + q];
  for (int q = 0; q < 6; ++q) {
    adj[(int64_t)q * N + p] = v[q];
    r[8 + q] = v[q];
    gxu[(int64_t)q * N + p] = 0.0;
  }
  for (int q = 14; q < kRecB; ++q) r[q] = 0.0;
}

// ---------------------------------------------------------------- L2P^T / P2M^T (per leaf)
// MODE 0 (L2P^T): fields F = leaf locals (6), adjoint a_p (6): gx_p += sum_q a_q dF_q/dx;
//   also gloc[leaf] += sum_p a_p w(x_p).
// MODE 1 (P2M^T): fields F = leaf moment adjoints (4): gu_p += I_M + I_G u/gamma,
//   gx_p += gamma dI_G/dx + u . dI_M/dx.
constexpr int kBwdChunk = 64;

template <int NDEG, int MODE>
__global__ void __launch_bounds__(128)
    leaf_bwd_kernel(int leaf0, const int *__restrict__ lohi, const double *__restrict__ nodes,
                    const double *__restrict__ bbox, const double *__restrict__ prec,
                    const double *__restrict__ field, const double *__restrict__ adj, int N,
                    double *__restrict__ gxu, double *__restrict__ gloc, double *__restrict__ gbox) {
  using S = BShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS;
  constexpr int Q = MODE == 0 ? 6 : 4;
  extern __shared__ __align__(16) unsigned char smem[];
  double *s_f = (double *)smem;  // Q*NN
  __shared__ double s_n[3 * M];
  __shared__ double s_red[32 * 6];
  __shared__ double s_w[kBwdChunk][3][M];
  __shared__ double s_a[kBwdChunk][6];
  const int tid = threadIdx.x;
  const int c = leaf0 + blockIdx.x;
  const int lo = lohi[2 * c], hi = lohi[2 * c + 1];
  const double *bb = bbox + 6 * (int64_t)c;
  const double *fc = field + (int64_t)c * Q * NN;
  for (int e = tid; e < Q * NN; e += blockDim.x) s_f[e] = fc[e];
  for (int i = tid; i < 3 * M; i += blockDim.x) s_n[i] = nodes[(int64_t)c * NS + i];
  __syncthreads();
  double gbx[6] = {0, 0, 0, 0, 0, 0};
  // Two threads per particle (h = tid & 1), each over half of the Q quantities.  The
  // position gradient is linear in the fields, so each thread folds its quantities
  // into one field first (by the particle's adjoint a_q, or by (gamma, u) for P2M^T)
  // and contracts that once with the weights and their derivatives; a shuffle adds the
  // two halves.
  constexpr int QH = Q / 2;
  const int h = tid & 1;
  for (int base = lo; base <= hi; base += (int)blockDim.x / 2) {
    const int p = base + (tid >> 1);
    const bool act = p <= hi;
    const double *r = prec + 8 * (int64_t)(act ? p : lo);
    double w[3][M], dw[3][M];
    weights_d64<M>(r[0], s_n, w[0], dw[0]);
    weights_d64<M>(r[1], s_n + M, w[1], dw[1]);
    weights_d64<M>(r[2], s_n + 2 * M, w[2], dw[2]);
    // this thread's fold coefficients and, for P2M^T, the values of its quantities
    double cq[QH];
    if (MODE == 0) {
#pragma unroll
      for (int u = 0; u < QH; ++u) cq[u] = act ? adj[(int64_t)(QH * h + u) * N + p] : 0.0;
    } else {
      const double cf[4] = {r[3], r[4], r[5], r[6]};  // gamma, u
#pragma unroll
      for (int u = 0; u < QH; ++u) cq[u] = act ? cf[QH * h + u] : 0.0;
    }
    double Iv[QH];
#pragma unroll
    for (int u = 0; u < QH; ++u) Iv[u] = 0.0;
    double dx = 0, dy = 0, dz = 0;
#pragma unroll
    for (int k = 0; k < M; ++k) {
      double ay = 0, ady = 0, axd = 0, iy[QH];
#pragma unroll
      for (int u = 0; u < QH; ++u) iy[u] = 0.0;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const double *row = s_f + (QH * h) * NN + M * (j + M * k);
        double vx = 0, vdx = 0, ix[QH];
#pragma unroll
        for (int u = 0; u < QH; ++u) ix[u] = 0.0;
#pragma unroll
        for (int i = 0; i < M; ++i) {
          double hv = 0;
#pragma unroll
          for (int u = 0; u < QH; ++u) {
            const double f = row[u * NN + i];
            hv += cq[u] * f;
            if (MODE == 1) ix[u] += w[0][i] * f;
          }
          vx += w[0][i] * hv;
          vdx += dw[0][i] * hv;
        }
        ay += w[1][j] * vx;
        ady += dw[1][j] * vx;
        axd += w[1][j] * vdx;
        if (MODE == 1)
#pragma unroll
          for (int u = 0; u < QH; ++u) iy[u] += w[1][j] * ix[u];
      }
      dx += w[2][k] * axd;
      dy += w[2][k] * ady;
      dz += dw[2][k] * ay;
      if (MODE == 1)
#pragma unroll
        for (int u = 0; u < QH; ++u) Iv[u] += w[2][k] * iy[u];
    }
    double G[3] = {dx, dy, dz};
#pragma unroll
    for (int d = 0; d < 3; ++d) G[d] += __shfl_xor_sync(0xffffffffu, G[d], 1);
    if (MODE == 1) {
      // gu += I_M + (I_Gamma / gamma) u: thread 0 holds I_Gamma, I_M0; thread 1 I_M1, I_M2
      const double ig = __shfl_sync(0xffffffffu, Iv[0], (tid & 31) & ~1) / r[3];
      if (act) {
        if (h == 0) {
          gxu[(int64_t)3 * N + p] += Iv[1] + ig * r[4];
        } else {
          gxu[(int64_t)4 * N + p] += Iv[0] + ig * r[5];
          gxu[(int64_t)5 * N + p] += Iv[1] + ig * r[6];
        }
      }
    }
    if (act && h == 0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        gxu[(int64_t)d * N + p] += G[d];
        const double a = bb[d], b = bb[3 + d], wd = b - a;
        if (wd > 0.0) {
          const double xi = (r[d] - a) / wd;
          gbx[d] += (xi - 1.0) * G[d];
          gbx[3 + d] += -xi * G[d];
        }
      }
    }
  }
  block_sum<6>(gbx, s_red);
  if (tid < 6) gbox[6 * (int64_t)c + tid] += gbx[tid];
  if (MODE == 0) {
    // gloc[leaf][q][a] += sum_p a_p[q] w_a(x_p)
    double acc[(NN + 127) / 128][6];
#pragma unroll
    for (int r = 0; r < (NN + 127) / 128; ++r)
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[r][q] = 0.0;
    for (int c0 = lo; c0 <= hi; c0 += kBwdChunk) {
      const int cnt = (hi - c0 + 1) < kBwdChunk ? (hi - c0 + 1) : kBwdChunk;
      __syncthreads();
      for (int task = tid; task < 3 * cnt; task += blockDim.x) {
        const int p = task / 3, d = task % 3;
        weights64<M>(prec[8 * (int64_t)(c0 + p) + d], s_n + d * M, s_w[p][d]);
      }
      for (int task = tid; task < 6 * cnt; task += blockDim.x) {
        const int p = task / 6, q = task % 6;
        s_a[p][q] = adj[(int64_t)q * N + c0 + p];
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < (NN + 127) / 128; ++r) {
        const int a = tid + 128 * r;
        if (a < NN) {
          const int ai = a % M, aj = (a / M) % M, ak = a / (M * M);
          for (int p = 0; p < cnt; ++p) {
            const double wt = s_w[p][0][ai] * s_w[p][1][aj] * s_w[p][2][ak];
#pragma unroll
            for (int q = 0; q < 6; ++q) acc[r][q] += s_a[p][q] * wt;
          }
        }
      }
    }
    double *gl = gloc + (int64_t)c * 6 * NN;
#pragma unroll
    for (int r = 0; r < (NN + 127) / 128; ++r) {
      const int a = tid + 128 * r;
      if (a < NN)
#pragma unroll
        for (int q = 0; q < 6; ++q) gl[q * NN + a] += acc[r][q];
    }
  }
}

// ---------------------------------------------------------------- L2L^T / M2M^T (per parent)
// The transfer T_c: child[i] = sum_I parent[I] W_c[i][I], W_c = Lx (x) Ly (x) Lz with
// L[d][i][I] = w_I^{parent}(x^{child}_{d,i}).
// MODE 0 (L2L^T, children at clevel): gP += T_c^T gC over both children; geometry with
//   X_c = gC (child local adjoint), Y_P = the parent's final locals.
// MODE 1 (M2M^T, parents at plevel): gC += T_c gP; geometry with X_c = the child's
//   moments, Y_P = gP (the parent's moment adjoint).
// Geometry: G_d[i] = sum_q sum_{(i,j,k): i_d = i} X_c[q][ijk] (T_c^{(d)} Y_P)[q][ijk] where
// T^{(d)} uses the derivative weights on axis d.
template <int NDEG, int MODE>
__global__ void __launch_bounds__(BShape<NDEG>::BT)
    transfer_bwd_kernel(int plevel, const double *__restrict__ nodes, const double *__restrict__ bbox, ChebT ct,
                        const double *__restrict__ Xfield, const double *__restrict__ Yfield,
                        double *__restrict__ gfield, double *__restrict__ gbox) {
  using S = BShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, BT = S::BT, NPT = S::NPT;
  constexpr int Q = MODE == 0 ? 6 : 4;
  constexpr int QN = Q * NN;
  extern __shared__ __align__(16) unsigned char smem[];
  double *s_x = (double *)smem;  // [Q][NN]
  double *s_y = s_x + QN;        // [Q][NN]
  double *s_t1 = s_y + QN;       // [Q][NN]
  double *s_t2 = s_t1 + QN;      // [Q][NN]
  double *s_e = s_t2 + QN;       // 3*NN products for the three axes
  __shared__ double L[2][3][M][M], D[2][3][M][M];
  __shared__ double s_G[2][3][M];
  const int tid = threadIdx.x;
  const int p = (1 << plevel) - 1 + blockIdx.x;
  const int c1 = 2 * p + 1;
  for (int task = tid; task < 2 * 3 * M; task += BT) {
    const int ch = task / (3 * M), r = task % (3 * M), d = r / M, i = r % M;
    const double x = nodes[(int64_t)(c1 + ch) * NS + d * M + i];
    weights_d64<M>(x, nodes + (int64_t)p * NS + d * M, L[ch][d][i], D[ch][d][i]);
  }
  double accP[NPT][Q];  // MODE 0: parent adjoint accumulation
#pragma unroll
  for (int r = 0; r < NPT; ++r)
#pragma unroll
    for (int q = 0; q < Q; ++q) accP[r][q] = 0.0;
  for (int e = tid; e < 2 * 3 * M; e += BT) (&s_G[0][0][0])[e] = 0.0;
  // All Q quantities go through each contraction stage together.  A stage reads the
  // buffer the previous one wrote and the barrier after it orders the two; the last
  // (z) stage of a contraction reads only s_t2, which the next contraction's y stage
  // rewrites after the barrier that follows its x stage.
  // x stage: t1[q][i + M(J + MK)] = sum_I Wx[i][I] src[q][I + M(J + MK)]
  auto stage_x = [&](const double(*Wx)[M], const double *src) {
    for (int e = tid; e < QN; e += BT) {
      const int i = e % M, qJK = e / M;
      const double *sp = src + M * qJK;
      double v = 0;
#pragma unroll
      for (int I = 0; I < M; ++I) v += Wx[i][I] * sp[I];
      s_t1[e] = v;
    }
  };
  // y stage: t2[q][i + M(j + MK)] = sum_J Wy[j][J] t1[q][i + M(J + MK)]
  auto stage_y = [&](const double(*Wy)[M]) {
    for (int e = tid; e < QN; e += BT) {
      const int i = e % M, j = (e / M) % M, qK = e / (M * M);
      const double *sp = s_t1 + i + M * M * qK;
      double v = 0;
#pragma unroll
      for (int J = 0; J < M; ++J) v += Wy[j][J] * sp[M * J];
      s_t2[e] = v;
    }
  };
  // transposed x and y stages (contraction over the child index, MODE 0)
  auto stage_xT = [&](const double(*Wx)[M], const double *src) {
    for (int e = tid; e < QN; e += BT) {
      const int I = e % M, qjk = e / M;
      const double *sp = src + M * qjk;
      double v = 0;
#pragma unroll
      for (int i = 0; i < M; ++i) v += Wx[i][I] * sp[i];
      s_t1[e] = v;
    }
  };
  auto stage_yT = [&](const double(*Wy)[M]) {
    for (int e = tid; e < QN; e += BT) {
      const int I = e % M, J = (e / M) % M, qk = e / (M * M);
      const double *sp = s_t1 + I + M * M * qk;
      double v = 0;
#pragma unroll
      for (int j = 0; j < M; ++j) v += Wy[j][J] * sp[M * j];
      s_t2[e] = v;
    }
  };
  __syncthreads();

  for (int ch = 0; ch < 2; ++ch) {
    const int c = c1 + ch;
    double eacc[NPT][3];
#pragma unroll
    for (int r = 0; r < NPT; ++r) eacc[r][0] = eacc[r][1] = eacc[r][2] = 0.0;
    {
      const double *X = Xfield + (int64_t)c * QN;
      const double *Y = Yfield + (int64_t)p * QN;
      for (int e = tid; e < QN; e += BT) {
        s_x[e] = X[e];
        s_y[e] = Y[e];
      }
    }
    __syncthreads();
    // adjoint propagation
    if (MODE == 0) {
      // parent[I] += sum_i W[i][I] gC[i] (contract x, y, z over the child index)
      stage_xT(L[ch][0], s_x);
      __syncthreads();
      stage_yT(L[ch][1]);
      __syncthreads();
#pragma unroll
      for (int r = 0; r < NPT; ++r) {
        const int a = tid + r * BT;
        if (a < NN) {
          const int IJ = a % (M * M), K = a / (M * M);
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            double v = 0;
#pragma unroll
            for (int k = 0; k < M; ++k) v += L[ch][2][k][K] * s_t2[q * NN + IJ + M * M * k];
            accP[r][q] += v;
          }
        }
      }
    } else {
      // child[i] += sum_I W[i][I] gP[I]
      stage_x(L[ch][0], s_y);
      __syncthreads();
      stage_y(L[ch][1]);
      __syncthreads();
      double *gc = gfield + (int64_t)c * QN;
      for (int e = tid; e < QN; e += BT) {
        const int ij = e % (M * M), qk = e / (M * M), q = qk / M, k = qk - q * M;
        const double *sp = s_t2 + q * NN + ij;
        double v = 0;
#pragma unroll
        for (int K = 0; K < M; ++K) v += L[ch][2][k][K] * sp[M * M * K];
        gc[e] += v;
      }
    }
    // geometry: e_d[a] += sum_q X[q][a] * (T^{(d)} Y)[q][a] for d = x, y, z.  Axes z and y
    // share the x stage Lx Y, and for M2M^T the propagation above already left Lx Y in s_t1
    // and Ly Lx Y in s_t2 (the z axis needs exactly those), so the three contractions take
    // 6 stages after M2M^T's propagation and 8 after L2L^T's instead of 9.
    auto stage_ze = [&](int d, const double(*Wz)[M]) {
#pragma unroll
      for (int r = 0; r < NPT; ++r) {
        const int a = tid + r * BT;
        if (a < NN) {
          const int ij = a % (M * M), k = a / (M * M);
          double sum = 0;
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            double v = 0;
#pragma unroll
            for (int K = 0; K < M; ++K) v += Wz[k][K] * s_t2[q * NN + ij + M * M * K];
            sum += s_x[q * NN + a] * v;
          }
          eacc[r][d] += sum;
        }
      }
    };
    if (MODE == 0) {
      stage_x(L[ch][0], s_y);
      __syncthreads();
      stage_y(L[ch][1]);
      __syncthreads();
    }
    stage_ze(2, D[ch][2]);  // z: Dz Ly Lx Y
    __syncthreads();
    stage_y(D[ch][1]);      // y: Lz Dy Lx Y, from the Lx Y still in s_t1
    __syncthreads();
    stage_ze(1, L[ch][2]);
    __syncthreads();
    stage_x(D[ch][0], s_y);  // x: Lz Ly Dx Y
    __syncthreads();
    stage_y(L[ch][1]);
    __syncthreads();
    stage_ze(0, L[ch][2]);
    // G_d[i] = sum over the nodes with index i on axis d
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int a = tid + r * BT;
      if (a < NN) {
        s_e[a] = eacc[r][0];
        s_e[NN + a] = eacc[r][1];
        s_e[2 * NN + a] = eacc[r][2];
      }
    }
    __syncthreads();
    if (tid < 3 * M) {
      const int d = tid / M, i = tid % M;
      double g = 0;
      for (int u = 0; u < M; ++u)
        for (int v = 0; v < M; ++v) {
          const int a = d == 0 ? i + M * (u + M * v) : (d == 1 ? u + M * (i + M * v) : u + M * (v + M * i));
          g += s_e[d * NN + a];
        }
      s_G[ch][d][i] = g;
    }
    __syncthreads();
  }
  // boxes: the child's nodes move with its box; the parent's weights with the parent's box
  if (tid < 6 * 3) {
    const int who = tid / 6, k = tid % 6, d = k % 3, side = k / 3;  // who: 0,1 children, 2 parent
    double g = 0;
    if (who < 2) {
      for (int i = 0; i < M; ++i) g += (side == 0 ? 1.0 - ct.t[i] : ct.t[i]) * s_G[who][d][i];
      gbox[6 * (int64_t)(c1 + who) + k] += g;
    } else {
      const double a = bbox[6 * (int64_t)p + d], b = bbox[6 * (int64_t)p + 3 + d], wd = b - a;
      if (wd > 0.0)
        for (int ch = 0; ch < 2; ++ch)
          for (int i = 0; i < M; ++i) {
            const double xi = (nodes[(int64_t)(c1 + ch) * NS + d * M + i] - a) / wd;
            g += (side == 0 ? xi - 1.0 : -xi) * s_G[ch][d][i];
          }
      gbox[6 * (int64_t)p + k] += g;
    }
  }
  if (MODE == 0) {
    double *gp = gfield + (int64_t)p * Q * NN;
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int a = tid + r * BT;
      if (a < NN)
#pragma unroll
        for (int q = 0; q < Q; ++q) gp[q * NN + a] += accP[r][q];
    }
  }
}

// ---------------------------------------------------------------- M2L^T (per target cluster)
// Over the union U(t) of {s : (t,s) in list} (flag 1) and {s : (s,t) in list}
// (flag 2), with R = x_a - x_b, f = d^{-3/2}, K = f R:
//   c1 = Gamma_s[b] gE_t[a] + gB_t[a] x M_s[b]      (t is the target)
//   c2 = Gamma_t[a] gE_s[b] + gB_s[b] x M_t[a]      (t is the source)
//   gx_a     += f c - 3 d^{-5/2} (R.c)(R + (p.R) p),  c = [f1] c1 - [f2] c2
//   gGamma_a -= [f2] f gE_s[b].R,   gM_a -= [f2] f R x gB_s[b]
//   gp       += [f1] -3 d^{-5/2} (p.R)(R.c1) R
// MASK (eta > 1/2): coincident nodes contribute nothing, as in the forward.
template <int NDEG, bool MASK>
__global__ void __launch_bounds__(BShape<NDEG>::BT)
    m2l_bwd_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const uint8_t *__restrict__ flg,
                   const double *__restrict__ nodes, ChebT ct, const double *__restrict__ mom,
                   const double *__restrict__ gloc, const double *__restrict__ consts, double *__restrict__ gmom,
                   double *__restrict__ gbox, double *__restrict__ gp_part, int *__restrict__ status) {
  using S = BShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, BT = S::BT, NPT = S::NPT;
  constexpr int REC = 10 * NN + NS;  // Gamma, M(3), gE(3), gB(3) | nodes
  extern __shared__ __align__(16) unsigned char smem[];
  double *buf = (double *)smem;  // 2 * REC
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_red[32 * 6];
  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double px = consts[0], py = consts[1], pz = consts[2];
  double gx[NPT][3], gG[NPT], gM[NPT][3], gp[3] = {0, 0, 0};
  double own[NPT][10];  // Gamma_a, M_a(3), gE_a(3), gB_a(3)
#pragma unroll
  for (int r = 0; r < NPT; ++r) {
    gx[r][0] = gx[r][1] = gx[r][2] = gG[r] = gM[r][0] = gM[r][1] = gM[r][2] = 0.0;
    const int a = tid + r * BT;
#pragma unroll
    for (int q = 0; q < 10; ++q) own[r][q] = 0.0;
    if (a < NN) {
      const double *ma = mom + (int64_t)t * 4 * NN, *la = gloc + (int64_t)t * 6 * NN;
#pragma unroll
      for (int q = 0; q < 4; ++q) own[r][q] = ma[q * NN + a];
#pragma unroll
      for (int q = 0; q < 6; ++q) own[r][4 + q] = la[q * NN + a];
    }
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
      double *dst = buf + bb * REC;
      mbar_arrive_expect_tx(&bar[bb], REC * 8);
      bulk_g2s(dst, mom + (int64_t)s * 4 * NN, 4 * NN * 8, &bar[bb]);
      bulk_g2s(dst + 4 * NN, gloc + (int64_t)s * 6 * NN, 6 * NN * 8, &bar[bb]);
      bulk_g2s(dst + 10 * NN, nodes + (int64_t)s * NS, NS * 8, &bar[bb]);
    };
    if (tid == 0) issue(0, 0);
    for (int it = 0; it < np; ++it) {
      const int bb = it & 1;
      const int fl = flg[p0 + it];
      if (tid == 0 && it + 1 < np) {
        fence_proxy_async_smem();
        issue(it + 1, bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((it >> 1) & 1), status);
      if (ok) {
        const double *B = buf + bb * REC;
        const double *SN = B + 10 * NN;
        const bool f1 = fl & 1, f2 = fl & 2;
#pragma unroll
        for (int r = 0; r < NPT; ++r) {
          const int a = tid + r * BT;
          if (a >= NN) continue;
          const int ai = a % M, aj = (a / M) % M, ak = a / (M * M);
          const double tx = tn[ai], ty = tn[M + aj], tz = tn[2 * M + ak];
          const double Ga = own[r][0], Ma0 = own[r][1], Ma1 = own[r][2], Ma2 = own[r][3];
          const double gEa0 = own[r][4], gEa1 = own[r][5], gEa2 = own[r][6];
          const double gBa0 = own[r][7], gBa1 = own[r][8], gBa2 = own[r][9];
          double rxv[M], prx[M], rx2[M];
#pragma unroll
          for (int bi = 0; bi < M; ++bi) {
            rxv[bi] = tx - SN[bi];
            prx[bi] = px * rxv[bi];
            rx2[bi] = rxv[bi] * rxv[bi];
          }
          double ax0 = 0, ax1 = 0, ax2 = 0, aG = 0, aM0 = 0, aM1 = 0, aM2 = 0, ap0 = 0, ap1 = 0, ap2 = 0;
#pragma unroll 1
          for (int bk = 0; bk < M; ++bk) {
            const double rz = tz - SN[2 * M + bk];
            const double prz = pz * rz, rz2 = rz * rz + kEps64;
            for (int bj = 0; bj < M; ++bj) {
              const double ry = ty - SN[M + bj];
              const double P = py * ry + prz, A = ry * ry + rz2;
              const int b0 = M * (bj + M * bk);
#pragma unroll
              for (int bi = 0; bi < M; ++bi) {
                const int b = b0 + bi;
                const double rx = rxv[bi];
                const double pr = P + prx[bi];
                const double d = pr * pr + (A + rx2[bi]);
                const double s = MASK && !(d > kEps64) ? 0.0 : rsqrt(d);
                const double f = s * s * s, f5 = f * s * s;
                double c0 = 0, c1 = 0, c2 = 0;
                if (f1) {
                  const double gs = B[b], m0 = B[NN + b], m1 = B[2 * NN + b], m2 = B[3 * NN + b];
                  c0 = gs * gEa0 + (gBa1 * m2 - gBa2 * m1);
                  c1 = gs * gEa1 + (gBa2 * m0 - gBa0 * m2);
                  c2 = gs * gEa2 + (gBa0 * m1 - gBa1 * m0);
                  const double w = -3.0 * f5 * pr * (rx * c0 + ry * c1 + rz * c2);
                  ap0 += w * rx;
                  ap1 += w * ry;
                  ap2 += w * rz;
                }
                if (f2) {
                  const double e0 = B[4 * NN + b], e1 = B[5 * NN + b], e2 = B[6 * NN + b];
                  const double h0 = B[7 * NN + b], h1 = B[8 * NN + b], h2 = B[9 * NN + b];
                  c0 -= Ga * e0 + (h1 * Ma2 - h2 * Ma1);
                  c1 -= Ga * e1 + (h2 * Ma0 - h0 * Ma2);
                  c2 -= Ga * e2 + (h0 * Ma1 - h1 * Ma0);
                  aG -= f * (e0 * rx + e1 * ry + e2 * rz);
                  aM0 -= f * (ry * h2 - rz * h1);
                  aM1 -= f * (rz * h0 - rx * h2);
                  aM2 -= f * (rx * h1 - ry * h0);
                }
                const double w3 = 3.0 * f5 * (rx * c0 + ry * c1 + rz * c2);
                ax0 += f * c0 - w3 * (rx + pr * px);
                ax1 += f * c1 - w3 * (ry + pr * py);
                ax2 += f * c2 - w3 * (rz + pr * pz);
              }
            }
          }
          gx[r][0] += ax0;
          gx[r][1] += ax1;
          gx[r][2] += ax2;
          gG[r] += aG;
          gM[r][0] += aM0;
          gM[r][1] += aM1;
          gM[r][2] += aM2;
          gp[0] += ap0;
          gp[1] += ap1;
          gp[2] += ap2;
        }
      }
      __syncthreads();
    }
  }
  // moment adjoints (source role) and the target box from the node-position gradients
  double gbx[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int r = 0; r < NPT; ++r) {
    const int a = tid + r * BT;
    if (a >= NN) continue;
    double *gm = gmom + (int64_t)t * 4 * NN;
    gm[a] += gG[r];
    gm[NN + a] += gM[r][0];
    gm[2 * NN + a] += gM[r][1];
    gm[3 * NN + a] += gM[r][2];
    const int idx[3] = {a % M, (a / M) % M, a / (M * M)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      gbx[d] += (1.0 - ct.t[idx[d]]) * gx[r][d];
      gbx[3 + d] += ct.t[idx[d]] * gx[r][d];
    }
  }
  block_sum<6>(gbx, s_red);
  if (tid < 6) gbox[6 * (int64_t)t + tid] += gbx[tid];
  double g3[6] = {gp[0], gp[1], gp[2], 0, 0, 0};
  block_sum<6>(g3, s_red);
  if (tid < 3) gp_part[3 * (int64_t)t + tid] = g3[tid];
}

// ---------------------------------------------------------------- M2L^T, mixed form
// The adjoint of the mixed forward evaluates M2L^T in FP32: the saved FP32 moments
// and the local adjoints (rounded from FP64) of every cluster are packed into one
// record [Gamma | M(3) | gE(3) | gB(3)] x NN, RECF floats per cluster.
template <int NDEG>
struct MBShape2 {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int NP = (NN + 1) / 2;           // target-node pairs, one per thread
  static constexpr int BT = ((NP + 31) / 32) * 32;
  static constexpr int RECF = ((10 * NN + 3) / 4) * 4;
  static constexpr int RAWB = RECF * 4;              // bytes of the FP32 part of a staged record
  static constexpr int REC = RAWB + NS * 8;          // ... followed by the node coordinates
  static constexpr int NACC = 14;                    // per target: axf(3) axw(3) ap(3) aG aM(3) sp
  static constexpr int SMEM = 2 * REC + 5 * NN * 16 + 2 * NACC * BT * 8;
};

template <int NDEG>
__global__ void adj_rec32_kernel(int64_t nc, const float *__restrict__ mom32, const double *__restrict__ gloc,
                                 float *__restrict__ rec) {
  using S = MBShape2<NDEG>;
  constexpr int NN = S::NN, RECF = S::RECF;
  const int64_t total = nc * RECF;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / RECF;
    const int e = (int)(i - c * RECF);
    float v = 0.f;
    if (e < 4 * NN)
      v = mom32[c * 4 * NN + e];
    else if (e < 10 * NN)
      v = (float)gloc[c * 6 * NN + (e - 4 * NN)];
    rec[i] = v;
  }
}

// Per target cluster over its union list, two target nodes per thread in the two
// lanes of packed FP32x2 instructions; the quantities are those of m2l_bwd_kernel:
//   c = [f1] (Gamma_b gE_a + gB_a x M_b) - [f2] (Gamma_a gE_b + gB_b x M_a)
//   gx_a += f c - 3 f5 (R.c)(R + (p.R) p)            (accumulated as axf - 3 (axw + sp p))
//   gp   += [f1] -3 f5 (p.R)(R.c1) R                  (accumulated as -3 ap)
//   gGamma_a -= [f2] f gE_b.R,  gM_a -= [f2] f R x gB_b
// Per source the FP32 partial sums are added into per-thread FP64 sums in shared memory.
template <int NDEG, bool MASK>
__global__ void __launch_bounds__(MBShape2<NDEG>::BT)
    m2l_bwd_x2_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const uint8_t *__restrict__ flg,
                      const double *__restrict__ nodes, const double *__restrict__ bbox, ChebT ct,
                      const float *__restrict__ rec32, const double *__restrict__ consts, double *__restrict__ gmom,
                      double *__restrict__ gbox, double *__restrict__ gp_part, int *__restrict__ status) {
  using S = MBShape2<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, NP = S::NP, BT = S::BT, RECF = S::RECF, RAWB = S::RAWB;
  constexpr int REC = S::REC, NACC = S::NACC;
  extern __shared__ __align__(16) unsigned char smem[];
  float4 *pk = (float4 *)(smem + 2 * REC);                     // 5 NN duplicated per-node operands
  double *s_acc = (double *)(smem + 2 * REC + 5 * NN * 16);     // [2 NACC][BT] FP64 sums
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_sn[3 * M];  // source node offsets from the target centre
  __shared__ double s_red[32 * 6];

  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);
  const bool act = tid < NP;
  const bool two = act && tid + NP < NN;  // the second lane holds a real node
  const int a0 = act ? tid : 0, a1 = two ? tid + NP : a0;
  const double tx0 = tn[a0 % M] - cx, ty0 = tn[M + (a0 / M) % M] - cy, tz0 = tn[2 * M + a0 / (M * M)] - cz;
  const double tx1 = tn[a1 % M] - cx, ty1 = tn[M + (a1 / M) % M] - cy, tz1 = tn[2 * M + a1 / (M * M)] - cz;
  const float *own = rec32 + (int64_t)t * RECF;
  auto pair = [&](int q) { return make_float2(own[q * NN + a0], own[q * NN + a1]); };
  const float2 Ga = pair(0), Ma0 = pair(1), Ma1 = pair(2), Ma2 = pair(3);
  const float2 gE0 = pair(4), gE1 = pair(5), gE2 = pair(6), gB0 = pair(7), gB1 = pair(8), gB2 = pair(9);
  const float2 nGa = make_float2(-Ga.x, -Ga.y), nMa0 = make_float2(-Ma0.x, -Ma0.y),
               nMa1 = make_float2(-Ma1.x, -Ma1.y), nMa2 = make_float2(-Ma2.x, -Ma2.y);
  const float2 ngB0 = make_float2(-gB0.x, -gB0.y), ngB1 = make_float2(-gB1.x, -gB1.y),
               ngB2 = make_float2(-gB2.x, -gB2.y);
  for (int q = 0; q < 2 * NACC; ++q) s_acc[q * BT + tid] = 0.0;
  const float2 px = dup2((float)consts[0]), py = dup2((float)consts[1]), pz = dup2((float)consts[2]);
  const float2 eps = dup2((float)kEps64);
  const float epsf = (float)kEps64;

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
      bulk_g2s(dst, rec32 + (int64_t)s * RECF, RAWB, &bar[bb]);
      bulk_g2s(dst + RAWB, nodes + (int64_t)s * NS, NS * 8, &bar[bb]);
    };
    if (tid == 0) issue(0, 0);
    for (int i = 0; i < np; ++i) {
      const int bb = i & 1;
      const int fl = flg[p0 + i];
      if (tid == 0 && i + 1 < np) {
        fence_proxy_async_smem();
        issue(i + 1, bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((i >> 1) & 1), status);
      const float *G = (const float *)(smem + bb * REC);
      const double *SN = (const double *)(smem + bb * REC + RAWB);
      if (ok) {
        for (int e = tid; e < 3 * M; e += BT) {
          const int d = e / M;
          s_sn[e] = SN[e] - (d == 0 ? cx : (d == 1 ? cy : cz));
        }
        // A pair in only one role zeroes the other role's half of the source data:
        // that role's terms then vanish exactly, so one evaluation loop serves all pairs.
        const float k1 = (fl & 1) ? 1.f : 0.f, k2 = (fl & 2) ? 1.f : 0.f;
        for (int b = tid; b < NN; b += BT) {
          float v[10];
#pragma unroll
          for (int q = 0; q < 10; ++q) v[q] = G[q * NN + b] * (q < 4 ? k1 : k2);
          float4 *o = pk + 5 * b;
          o[0] = make_float4(v[0], v[0], v[1], v[1]);  // Gamma, M0
          o[1] = make_float4(v[2], v[2], v[3], v[3]);  // M1, M2
          o[2] = make_float4(v[4], v[4], v[5], v[5]);  // gE0, gE1
          o[3] = make_float4(v[6], v[6], v[7], v[7]);  // gE2, gB0
          o[4] = make_float4(v[8], v[8], v[9], v[9]);  // gB1, gB2
        }
      }
      __syncthreads();
      if (ok && act) {
        float2 rxv[M], nrxv[M], prx[M], rx2[M], ryv[M];
#pragma unroll
        for (int b = 0; b < M; ++b) {
          const float2 rx = make_float2((float)(tx0 - s_sn[b]), (float)(tx1 - s_sn[b]));
          rxv[b] = rx;
          nrxv[b] = make_float2(-rx.x, -rx.y);
          prx[b] = mul2(px, rx);
          rx2[b] = mul2(rx, rx);
          ryv[b] = make_float2((float)(ty0 - s_sn[M + b]), (float)(ty1 - s_sn[M + b]));
        }
        const float2 z = make_float2(0.f, 0.f);
        float2 axf0 = z, axf1 = z, axf2 = z, axw0 = z, axw1 = z, axw2 = z, ap0 = z, ap1 = z, ap2 = z;
        float2 aG = z, aM0 = z, aM1 = z, aM2 = z, sp = z;
        auto sweep = [&](auto FL) {
          constexpr int F = decltype(FL)::value;
#pragma unroll 1
          for (int bk = 0; bk < M; ++bk) {
            const float2 rz = make_float2((float)(tz0 - s_sn[2 * M + bk]), (float)(tz1 - s_sn[2 * M + bk]));
            const float2 nrz = make_float2(-rz.x, -rz.y);
            const float2 prz = mul2(pz, rz);
            const float2 rzz = fma2(rz, rz, eps);
#pragma unroll
            for (int bj = 0; bj < M; ++bj) {
              const float2 ry = ryv[bj], nry = make_float2(-ry.x, -ry.y);
              const float2 P = fma2(py, ry, prz);
              const float2 A = fma2(ry, ry, rzz);
              const float4 *pb = pk + 5 * M * (bj + M * bk);
#pragma unroll
              for (int bi = 0; bi < M; ++bi) {
                const float2 rx = rxv[bi];
                const float2 tt = add2(P, prx[bi]);  // p.R
                const float2 d = fma2(tt, tt, add2(A, rx2[bi]));
                float2 sv = rsqrt2(d);
                if constexpr (MASK) {
                  sv.x = d.x > epsf ? sv.x : 0.f;
                  sv.y = d.y > epsf ? sv.y : 0.f;
                }
                const float2 s2 = mul2(sv, sv);
                const float2 f = mul2(s2, sv);  // the s^5 terms are formed as f (s^2 ...): no FP32 overflow
                float2 c0 = z, c1 = z, c2 = z, rc = z;
                if constexpr ((F & 1) != 0) {
                  const float4 q0 = pb[5 * bi], q1 = pb[5 * bi + 1];
                  const float2 Gb = lo2(q0), Mb0 = hi2(q0), Mb1 = lo2(q1), Mb2 = hi2(q1);
                  c0 = fma2(Gb, gE0, fma2(gB1, Mb2, mul2(ngB2, Mb1)));
                  c1 = fma2(Gb, gE1, fma2(gB2, Mb0, mul2(ngB0, Mb2)));
                  c2 = fma2(Gb, gE2, fma2(gB0, Mb1, mul2(ngB1, Mb0)));
                  rc = fma2(rz, c2, fma2(ry, c1, mul2(rx, c0)));
                  const float2 w1 = mul2(f, mul2(mul2(s2, tt), rc));
                  ap0 = fma2(w1, rx, ap0);
                  ap1 = fma2(w1, ry, ap1);
                  ap2 = fma2(w1, rz, ap2);
                }
                if constexpr ((F & 2) != 0) {
                  const float4 q2 = pb[5 * bi + 2], q3 = pb[5 * bi + 3], q4 = pb[5 * bi + 4];
                  const float2 E0 = lo2(q2), E1 = hi2(q2), E2 = lo2(q3), H0 = hi2(q3), H1 = lo2(q4), H2 = hi2(q4);
                  c0 = fma2(nGa, E0, fma2(Ma1, H2, fma2(nMa2, H1, c0)));
                  c1 = fma2(nGa, E1, fma2(Ma2, H0, fma2(nMa0, H2, c1)));
                  c2 = fma2(nGa, E2, fma2(Ma0, H1, fma2(nMa1, H0, c2)));
                  rc = fma2(rz, c2, fma2(ry, c1, mul2(rx, c0)));
                  const float2 er = fma2(rz, E2, fma2(ry, E1, mul2(rx, E0)));
                  aG = fma2(f, er, aG);
                  aM0 = fma2(f, fma2(ry, H2, mul2(nrz, H1)), aM0);
                  aM1 = fma2(f, fma2(rz, H0, mul2(nrxv[bi], H2)), aM1);
                  aM2 = fma2(f, fma2(rx, H1, mul2(nry, H0)), aM2);
                }
                const float2 fr = mul2(f, mul2(s2, rc));
                axf0 = fma2(f, c0, axf0);
                axf1 = fma2(f, c1, axf1);
                axf2 = fma2(f, c2, axf2);
                axw0 = fma2(fr, rx, axw0);
                axw1 = fma2(fr, ry, axw1);
                axw2 = fma2(fr, rz, axw2);
                sp = fma2(fr, tt, sp);  // the (p.R) p part: p is the same for every evaluation
              }
            }
          }
        };
        if (fl != 0) sweep(std::integral_constant<int, 3>{});
        const float2 part[NACC] = {axf0, axf1, axf2, axw0, axw1, axw2, ap0, ap1, ap2, aG, aM0, aM1, aM2, sp};
#pragma unroll
        for (int q = 0; q < NACC; ++q) {
          s_acc[(2 * q) * BT + tid] += (double)part[q].x;
          s_acc[(2 * q + 1) * BT + tid] += (double)part[q].y;
        }
      }
      __syncthreads();  // the packed data and buffer bb are rewritten later
    }
  }
  // moment adjoints (source role), the box from the node-position gradients, d/dp_avg
  double gbx[6] = {0, 0, 0, 0, 0, 0};
  double gpv[6] = {0, 0, 0, 0, 0, 0};
  if (act) {
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (u == 1 && !two) break;
      const int a = u == 0 ? a0 : a1;
      double v[NACC];
#pragma unroll
      for (int q = 0; q < NACC; ++q) v[q] = s_acc[(2 * q + u) * BT + tid];
      double *gm = gmom + (int64_t)t * 4 * NN;
      gm[a] -= v[9];
      gm[NN + a] -= v[10];
      gm[2 * NN + a] -= v[11];
      gm[3 * NN + a] -= v[12];
      const int idx[3] = {a % M, (a / M) % M, a / (M * M)};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double gx = v[d] - 3.0 * (v[3 + d] + v[13] * consts[d]);
        gbx[d] += (1.0 - ct.t[idx[d]]) * gx;
        gbx[3 + d] += ct.t[idx[d]] * gx;
        gpv[d] += -3.0 * v[6 + d];
      }
    }
  }
  block_sum<6>(gbx, s_red);
  if (tid < 6) gbox[6 * (int64_t)t + tid] += gbx[tid];
  block_sum<6>(gpv, s_red);
  if (tid < 3) gp_part[3 * (int64_t)t + tid] = gpv[tid];
}

// M2L^T, mixed form, eta <= 1/2 (no two nodes of a pair coincide): one own node per
// thread in scalar FP32, the sums over the source nodes b factored so that every term
// linear in the source data costs one FMA per evaluation.  With R = x_a - y_b (both
// relative to the cluster's own centre) and f = s^3, f5 = s^5, s = d^{-1/2}:
//   sum f c          = gE_a SfG + gB_a x SfM - Gamma_a SfE + M_a x SfH
//   sum f R.gE_b     = x_a . SfE - Sfe,     sum f R x gB_b = x_a x SfH - Sfh
// where SfG = sum f Gamma_b, SfM = sum f M_b, SfE = sum f gE_b, SfH = sum f gB_b,
// Sfe = sum f (y_b . gE_b) and Sfh = sum f (y_b x gB_b); the last two are packed with
// the source data.  The scalar
//   R.c = Gamma_b (R.gE_a) + M_b.(R x gB_a) - Gamma_a (R.gE_b) + gB_b.(R x M_a)
// takes the parts of R.gE_a, R x gB_a and R x M_a that do not depend on the source
// column from the row and plane loops.  Per source pair the FP32 sums are combined
// into ten per-node values (node gradient, Gamma and M adjoints, p_avg partial) and
// added into FP64 sums in shared memory.  Scalar rather than packed FP32x2: the 21
// running sums of two nodes per thread would not fit the register file.
template <int NDEG>
struct MBShape1F {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int BT = ((NN + 31) / 32) * 32;
  static constexpr int RECF = MBShape2<NDEG>::RECF;  // the staged records of m2l_bwd_x2_kernel
  static constexpr int RAWB = RECF * 4;
  static constexpr int REC = RAWB + NS * 8;
  static constexpr int PKV = 4;   // float4 per packed source node
  static constexpr int NF = 10;   // FP64 sums per node: gx(3) gGamma gM(3) gp(3)
  static constexpr int SMEM = 2 * REC + PKV * NN * 16 + NF * BT * 8;
  // resident CTAs asked of the register allocator: 512 threads per SM, i.e. at most
  // 128 registers per thread (n = 4: four CTAs of 128 threads; measured 5 % faster
  // than the unbounded 167-register build)
  static constexpr int MINB = BT >= 512 ? 1 : 512 / BT;
};

template <int NDEG>
__global__ void __launch_bounds__(MBShape1F<NDEG>::BT, MBShape1F<NDEG>::MINB)
    m2l_bwd_x1f_kernel(const int *__restrict__ ptr, const int *__restrict__ src, const uint8_t *__restrict__ flg,
                       const double *__restrict__ nodes, const double *__restrict__ bbox, ChebT ct,
                       const float *__restrict__ rec32, const double *__restrict__ consts, double *__restrict__ gmom,
                       double *__restrict__ gbox, double *__restrict__ gp_part, int *__restrict__ status) {
  using S = MBShape1F<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS, BT = S::BT, RECF = S::RECF, RAWB = S::RAWB;
  constexpr int REC = S::REC, NF = S::NF, PKV = S::PKV;
  extern __shared__ __align__(16) unsigned char smem[];
  float4 *pk = (float4 *)(smem + 2 * REC);                      // PKV NN packed per-node operands
  double *s_acc = (double *)(smem + 2 * REC + PKV * NN * 16);    // [NF][BT] FP64 sums
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double s_sn[3 * M];  // source node offsets from the own centre
  __shared__ double s_red[32 * 6];
  __shared__ double s_ct[M];
  __shared__ int s_dir[2];  // per staged source: the boxes nearly touch (factored_ok fails)

  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  if (tid == 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) s_ct[i] = ct.t[i];
  }
  const int p0 = ptr[t], np = ptr[t + 1] - p0;
  const double *tn = nodes + (int64_t)t * NS;
  const double *tb = bbox + 6 * (int64_t)t;
  const double cx = 0.5 * (tb[0] + tb[3]), cy = 0.5 * (tb[1] + tb[4]), cz = 0.5 * (tb[2] + tb[5]);
  const bool act = tid < NN;
  const int a = act ? tid : 0;
  const double tx = tn[a % M] - cx, ty = tn[M + (a / M) % M] - cy, tz = tn[2 * M + a / (M * M)] - cz;
  const float *own = rec32 + (int64_t)t * RECF;
  const float Ga = own[a], Ma0 = own[NN + a], Ma1 = own[2 * NN + a], Ma2 = own[3 * NN + a];
  const float gE0 = own[4 * NN + a], gE1 = own[5 * NN + a], gE2 = own[6 * NN + a];
  const float gB0 = own[7 * NN + a], gB1 = own[8 * NN + a], gB2 = own[9 * NN + a];
  for (int q = 0; q < NF; ++q) s_acc[q * BT + tid] = 0.0;
  const float py = (float)consts[1], pz = (float)consts[2];
  const float eps = (float)kEps64;

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
      // written before the arrive, whose release orders it for the waiting threads
      s_dir[bb] = !factored_ok(bbox + 6 * (int64_t)s, tb, cx, cy, cz);
      mbar_arrive_expect_tx(&bar[bb], REC);
      bulk_g2s(dst, rec32 + (int64_t)s * RECF, RAWB, &bar[bb]);
      bulk_g2s(dst + RAWB, nodes + (int64_t)s * NS, NS * 8, &bar[bb]);
    };
    if (tid == 0) issue(0, 0);
    for (int i = 0; i < np; ++i) {
      const int bb = i & 1;
      const int fl = flg[p0 + i];
      if (tid == 0 && i + 1 < np) {
        fence_proxy_async_smem();
        issue(i + 1, bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((i >> 1) & 1), status);
      const float *G = (const float *)(smem + bb * REC);
      const double *SN = (const double *)(smem + bb * REC + RAWB);
      if (ok) {
        for (int e = tid; e < 3 * M; e += BT) {
          const int d = e / M;
          s_sn[e] = SN[e] - (d == 0 ? cx : (d == 1 ? cy : cz));
        }
        // A pair in only one role zeroes the other role's half of the source data.
        const float k1 = (fl & 1) ? 1.f : 0.f, k2 = (fl & 2) ? 1.f : 0.f;
        for (int b = tid; b < NN; b += BT) {
          float v[10];
#pragma unroll
          for (int q = 0; q < 10; ++q) v[q] = G[q * NN + b] * (q < 4 ? k1 : k2);
          const double yx = SN[b % M] - cx, yy = SN[M + (b / M) % M] - cy, yz = SN[2 * M + b / (M * M)] - cz;
          const float e = (float)(yx * v[4] + yy * v[5] + yz * v[6]);
          const float h0 = (float)(yy * v[9] - yz * v[8]), h1 = (float)(yz * v[7] - yx * v[9]),
                      h2 = (float)(yx * v[8] - yy * v[7]);
          float4 *o = pk + PKV * b;
          o[0] = make_float4(v[0], v[1], v[2], v[3]);  // Gamma, M
          o[1] = make_float4(v[4], v[5], v[6], v[7]);  // gE, gB0
          o[2] = make_float4(v[8], v[9], e, h0);       // gB1, gB2, y.gE, (y x gB)0
          o[3] = make_float4(h1, h2, 0.f, 0.f);        // (y x gB)1, (y x gB)2
        }
      }
      __syncthreads();
      if (ok && act && fl != 0) {
        float rxv[M], prx[M], rx2[M], ryv[M];
        {
          const float px = (float)consts[0];
#pragma unroll
          for (int b = 0; b < M; ++b) {
            const float rx = (float)(tx - s_sn[b]);
            rxv[b] = rx;
            prx[b] = px * rx;
            rx2[b] = rx * rx;
            ryv[b] = (float)(ty - s_sn[M + b]);
          }
        }
        float part[NF];
        if (s_dir[bb]) {
          // Boxes that nearly touch: the factored form of the moment adjoints, x_a . SfE - Sfe
          // and x_a x SfH - Sfh, would cancel, so those two sums are accumulated directly
          // (f R.gE_b, f R x gB_b); the other sums have no position difference and stay
          // factored.  Rows one at a time: with the factored branch's 25 unrolled evaluations
          // the two loop bodies would not fit the instruction cache together.
          float SfG = 0.f, SfM0 = 0.f, SfM1 = 0.f, SfM2 = 0.f, SfE0 = 0.f, SfE1 = 0.f, SfE2 = 0.f;
          float SfH0 = 0.f, SfH1 = 0.f, SfH2 = 0.f, aG = 0.f, aM0 = 0.f, aM1 = 0.f, aM2 = 0.f;
          float aw0 = 0.f, aw1 = 0.f, aw2 = 0.f, sp = 0.f, ap0 = 0.f, ap1 = 0.f, ap2 = 0.f;
#pragma unroll 1
          for (int bk = 0; bk < M; ++bk) {
            const float rz = (float)(tz - s_sn[2 * M + bk]);
            const float prz = pz * rz;
            const float rzz = fmaf(rz, rz, eps);
            const float ek = rz * gE2;
            const float w1k = rz * gB0;
            const float v1k = rz * Ma0;
#pragma unroll 1
            for (int bj = 0; bj < M; ++bj) {
              const float ry = (float)(ty - s_sn[M + bj]);
              const float P = fmaf(py, ry, prz);
              const float A = fmaf(ry, ry, rzz);
              const float ejk = fmaf(ry, gE1, ek);
              const float w0 = fmaf(ry, gB2, -(rz * gB1));
              const float w2j = -(ry * gB0);
              const float v0 = fmaf(ry, Ma2, -(rz * Ma1));
              const float v2j = -(ry * Ma0);
              const float4 *pb = pk + PKV * M * (bj + M * bk);
#pragma unroll
              for (int bi = 0; bi < M; ++bi) {
                const float rx = rxv[bi];
                const float tt = P + prx[bi];
                const float d = fmaf(tt, tt, A + rx2[bi]);
                const float sv = rsqrt_approx_f32(d);
                const float s2 = sv * sv;
                const float f = s2 * sv;  // the s^5 terms are formed as f (s^2 ...): no FP32 overflow
                const float4 q0 = pb[PKV * bi], q1 = pb[PKV * bi + 1];
                const float2 q2 = *(const float2 *)(pb + PKV * bi + 2);
                const float Gb = q0.x, Mb0 = q0.y, Mb1 = q0.z, Mb2 = q0.w;
                const float E0 = q1.x, E1 = q1.y, E2 = q1.z, H0 = q1.w, H1 = q2.x, H2 = q2.y;
                const float rge = fmaf(rx, gE0, ejk);
                const float w1 = fmaf(rx, -gB2, w1k);
                const float w2 = fmaf(rx, gB1, w2j);
                const float rc1 = fmaf(Gb, rge, fmaf(Mb2, w2, fmaf(Mb1, w1, Mb0 * w0)));
                const float er = fmaf(rz, E2, fmaf(ry, E1, rx * E0));
                const float v1 = fmaf(rx, -Ma2, v1k);
                const float v2 = fmaf(rx, Ma1, v2j);
                const float rc = fmaf(H2, v2, fmaf(H1, v1, fmaf(H0, v0, fmaf(-Ga, er, rc1))));
                const float wp = f * ((s2 * tt) * rc1);
                ap0 = fmaf(wp, rx, ap0);
                ap1 = fmaf(wp, ry, ap1);
                ap2 = fmaf(wp, rz, ap2);
                const float fr = f * (s2 * rc);
                aw0 = fmaf(fr, rx, aw0);
                aw1 = fmaf(fr, ry, aw1);
                aw2 = fmaf(fr, rz, aw2);
                sp = fmaf(fr, tt, sp);
                SfG = fmaf(f, Gb, SfG);
                SfM0 = fmaf(f, Mb0, SfM0);
                SfM1 = fmaf(f, Mb1, SfM1);
                SfM2 = fmaf(f, Mb2, SfM2);
                SfE0 = fmaf(f, E0, SfE0);
                SfE1 = fmaf(f, E1, SfE1);
                SfE2 = fmaf(f, E2, SfE2);
                SfH0 = fmaf(f, H0, SfH0);
                SfH1 = fmaf(f, H1, SfH1);
                SfH2 = fmaf(f, H2, SfH2);
                aG = fmaf(f, er, aG);
                aM0 = fmaf(f, fmaf(ry, H2, -(rz * H1)), aM0);
                aM1 = fmaf(f, fmaf(rz, H0, -(rx * H2)), aM1);
                aM2 = fmaf(f, fmaf(rx, H1, -(ry * H0)), aM2);
              }
            }
          }
          const float px = (float)consts[0];
          part[0] = fmaf(-3.f, fmaf(sp, px, aw0), gE0 * SfG + (gB1 * SfM2 - gB2 * SfM1) +
                                                      (Ma1 * SfH2 - Ma2 * SfH1) - Ga * SfE0);
          part[1] = fmaf(-3.f, fmaf(sp, py, aw1), gE1 * SfG + (gB2 * SfM0 - gB0 * SfM2) +
                                                      (Ma2 * SfH0 - Ma0 * SfH2) - Ga * SfE1);
          part[2] = fmaf(-3.f, fmaf(sp, pz, aw2), gE2 * SfG + (gB0 * SfM1 - gB1 * SfM0) +
                                                      (Ma0 * SfH1 - Ma1 * SfH0) - Ga * SfE2);
          part[3] = aG;
          part[4] = aM0;
          part[5] = aM1;
          part[6] = aM2;
          part[7] = ap0;
          part[8] = ap1;
          part[9] = ap2;
        } else {
        float SfG = 0.f, SfM0 = 0.f, SfM1 = 0.f, SfM2 = 0.f, SfE0 = 0.f, SfE1 = 0.f, SfE2 = 0.f;
        float SfH0 = 0.f, SfH1 = 0.f, SfH2 = 0.f, Sfe = 0.f, Sfh0 = 0.f, Sfh1 = 0.f, Sfh2 = 0.f;
        float aw0 = 0.f, aw1 = 0.f, aw2 = 0.f, sp = 0.f, ap0 = 0.f, ap1 = 0.f, ap2 = 0.f;
#pragma unroll 1
        for (int bk = 0; bk < M; ++bk) {
          const float rz = (float)(tz - s_sn[2 * M + bk]);
          const float prz = pz * rz;
          const float rzz = fmaf(rz, rz, eps);
          const float ek = rz * gE2;   // (R.gE_a): z part
          const float w1k = rz * gB0;  // (R x gB_a)_1 = rz gB0 - rx gB2
          const float v1k = rz * Ma0;  // (R x M_a)_1 = rz Ma0 - rx Ma2
#pragma unroll
          for (int bj = 0; bj < M; ++bj) {
            const float ry = ryv[bj];
            const float P = fmaf(py, ry, prz);
            const float A = fmaf(ry, ry, rzz);
            const float ejk = fmaf(ry, gE1, ek);
            const float w0 = fmaf(ry, gB2, -(rz * gB1));  // (R x gB_a)_0
            const float w2j = -(ry * gB0);                // (R x gB_a)_2 = rx gB1 - ry gB0
            const float v0 = fmaf(ry, Ma2, -(rz * Ma1));  // (R x M_a)_0
            const float v2j = -(ry * Ma0);                // (R x M_a)_2 = rx Ma1 - ry Ma0
            const float4 *pb = pk + PKV * M * (bj + M * bk);
#pragma unroll
            for (int bi = 0; bi < M; ++bi) {
              const float rx = rxv[bi];
              const float tt = P + prx[bi];  // p.R
              const float d = fmaf(tt, tt, A + rx2[bi]);
              const float sv = rsqrt_approx_f32(d);
              const float s2 = sv * sv;
              const float f = s2 * sv;  // the s^5 terms are formed as f (s^2 ...): no FP32 overflow
              const float4 q0 = pb[PKV * bi], q1 = pb[PKV * bi + 1], q2 = pb[PKV * bi + 2];
              const float2 q3 = *(const float2 *)(pb + PKV * bi + 3);
              const float Gb = q0.x, Mb0 = q0.y, Mb1 = q0.z, Mb2 = q0.w;
              const float E0 = q1.x, E1 = q1.y, E2 = q1.z, H0 = q1.w, H1 = q2.x, H2 = q2.y;
              const float rge = fmaf(rx, gE0, ejk);
              const float w1 = fmaf(rx, -gB2, w1k);
              const float w2 = fmaf(rx, gB1, w2j);
              const float rc1 = fmaf(Gb, rge, fmaf(Mb2, w2, fmaf(Mb1, w1, Mb0 * w0)));
              const float er = fmaf(rz, E2, fmaf(ry, E1, rx * E0));
              const float v1 = fmaf(rx, -Ma2, v1k);
              const float v2 = fmaf(rx, Ma1, v2j);
              const float rc = fmaf(H2, v2, fmaf(H1, v1, fmaf(H0, v0, fmaf(-Ga, er, rc1))));
              const float wp = f * ((s2 * tt) * rc1);
              ap0 = fmaf(wp, rx, ap0);
              ap1 = fmaf(wp, ry, ap1);
              ap2 = fmaf(wp, rz, ap2);
              const float fr = f * (s2 * rc);
              aw0 = fmaf(fr, rx, aw0);
              aw1 = fmaf(fr, ry, aw1);
              aw2 = fmaf(fr, rz, aw2);
              sp = fmaf(fr, tt, sp);  // the (p.R) p part: p is the same for every evaluation
              SfG = fmaf(f, Gb, SfG);
              SfM0 = fmaf(f, Mb0, SfM0);
              SfM1 = fmaf(f, Mb1, SfM1);
              SfM2 = fmaf(f, Mb2, SfM2);
              SfE0 = fmaf(f, E0, SfE0);
              SfE1 = fmaf(f, E1, SfE1);
              SfE2 = fmaf(f, E2, SfE2);
              SfH0 = fmaf(f, H0, SfH0);
              SfH1 = fmaf(f, H1, SfH1);
              SfH2 = fmaf(f, H2, SfH2);
              Sfe = fmaf(f, q2.z, Sfe);
              Sfh0 = fmaf(f, q2.w, Sfh0);
              Sfh1 = fmaf(f, q3.x, Sfh1);
              Sfh2 = fmaf(f, q3.y, Sfh2);
            }
          }
        }
        // this source pair's contributions, combined in FP32
        const float xa = (float)tx, ya = (float)ty, za = (float)tz;
        const float px = (float)consts[0];
        // gx = gE_a SfG + gB_a x SfM - Gamma_a SfE + M_a x SfH - 3 (aw + sp p)
        part[0] = fmaf(-3.f, fmaf(sp, px, aw0), gE0 * SfG + (gB1 * SfM2 - gB2 * SfM1) +
                                                    (Ma1 * SfH2 - Ma2 * SfH1) - Ga * SfE0);
        part[1] = fmaf(-3.f, fmaf(sp, py, aw1), gE1 * SfG + (gB2 * SfM0 - gB0 * SfM2) +
                                                    (Ma2 * SfH0 - Ma0 * SfH2) - Ga * SfE1);
        part[2] = fmaf(-3.f, fmaf(sp, pz, aw2), gE2 * SfG + (gB0 * SfM1 - gB1 * SfM0) +
                                                    (Ma0 * SfH1 - Ma1 * SfH0) - Ga * SfE2);
        // sum f R.gE_b and sum f R x gB_b (subtracted from the moment adjoints)
        part[3] = fmaf(za, SfE2, fmaf(ya, SfE1, xa * SfE0)) - Sfe;
        part[4] = (ya * SfH2 - za * SfH1) - Sfh0;
        part[5] = (za * SfH0 - xa * SfH2) - Sfh1;
        part[6] = (xa * SfH1 - ya * SfH0) - Sfh2;
        part[7] = ap0;
        part[8] = ap1;
        part[9] = ap2;
        }
#pragma unroll
        for (int q = 0; q < NF; ++q) s_acc[q * BT + tid] += (double)part[q];
      }
      __syncthreads();  // the packed data and buffer bb are rewritten later
    }
  }
  __syncthreads();  // s_ct
  // moment adjoints (source role), the box from the node-position gradients, d/dp_avg
  double gbx[6] = {0, 0, 0, 0, 0, 0};
  double gpv[6] = {0, 0, 0, 0, 0, 0};
  if (act) {
    double v[NF];
#pragma unroll
    for (int q = 0; q < NF; ++q) v[q] = s_acc[q * BT + tid];
    double *gm = gmom + (int64_t)t * 4 * NN;
    gm[a] -= v[3];
    gm[NN + a] -= v[4];
    gm[2 * NN + a] -= v[5];
    gm[3 * NN + a] -= v[6];
    const int idx[3] = {a % M, (a / M) % M, a / (M * M)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      gbx[d] += (1.0 - s_ct[idx[d]]) * v[d];
      gbx[3 + d] += s_ct[idx[d]] * v[d];
      gpv[d] += -3.0 * v[7 + d];
    }
  }
  block_sum<6>(gbx, s_red);
  if (tid < 6) gbox[6 * (int64_t)t + tid] += gbx[tid];
  block_sum<6>(gpv, s_red);
  if (tid < 3) gp_part[3 * (int64_t)t + tid] = gpv[tid];
}

// ---------------------------------------------------------------- P2P^T (per target leaf)
// Per target particle p over the particles j of every source leaf in the union list:
//   (t <- s), flag 1: K1 = K(R; u_j), c1 = gamma_j a_E,p + a_B,p x u_j:
//        gx_p += J1^T c1 = f1 c1 - 3 d1^{-5/2} (R.c1)(R + (u_j.R) u_j)
//   (s <- t), flag 2: K2 = K(-R; u_p), c2 = gamma_p a_E,j + a_B,j x u_p:
//        gx_p -= J2^T c2;  gu_p += 3 d2^{-5/2}(R.c2)(u_p.R) R - f2 (a_E,j.R) u_p/gamma_p - f2 R x a_B,j
// with R = x_p - x_j; the self pair j = p is skipped.
constexpr int kPbTile = 64;

template <int G>
__global__ void __launch_bounds__(128)
    p2p_bwd_kernel(int leaf0, const int *__restrict__ lohi, const int *__restrict__ ptr, const int *__restrict__ src,
                   const uint8_t *__restrict__ flg, const double *__restrict__ rec16, int N,
                   double *__restrict__ gxu, int *__restrict__ status) {
  __shared__ __align__(16) double buf[2][kPbTile * kRecB];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int meta[2][3];  // cnt, flag, first tree index
  __shared__ int s_warp[33];
  const int tid = threadIdx.x, TP = blockDim.x / G, tl = tid / G, g = tid % G;
  const int c = leaf0 + blockIdx.x;
  const int tlo = lohi[2 * c], thi = lohi[2 * c + 1], tcnt = thi - tlo + 1;
  const int p0 = ptr[c], np = ptr[c + 1] - p0;
  int w = 0;
  for (int k = tid; k < np; k += blockDim.x) {
    const int s = src[p0 + k];
    w += (lohi[2 * s + 1] - lohi[2 * s] + kPbTile) / kPbTile;
  }
  int W;
  block_excl_scan(w, s_warp, &W);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int wk = 0, woff = 0;
  auto issue = [&](int bb) {
    const int s = src[p0 + wk];
    const int slo = lohi[2 * s], scnt = lohi[2 * s + 1] - slo + 1;
    const int cnt = scnt - woff < kPbTile ? scnt - woff : kPbTile;
    meta[bb][0] = cnt;
    meta[bb][1] = flg[p0 + wk];
    meta[bb][2] = slo + woff;
    mbar_arrive_expect_tx(&bar[bb], (uint32_t)(cnt * kRecB * 8));
    bulk_g2s(&buf[bb][0], rec16 + kRecB * (int64_t)(slo + woff), (uint32_t)(cnt * kRecB * 8), &bar[bb]);
    woff += kPbTile;
    if (woff >= scnt) {
      woff = 0;
      ++wk;
    }
  };
  int it = 0;
  for (int tc = 0; tc < tcnt; tc += TP) {
    const int ti = tc + tl;
    const bool active = ti < tcnt;
    const int pi = tlo + (active ? ti : 0);
    const double *rp = rec16 + kRecB * (int64_t)pi;
    const double xp = rp[0], yp = rp[1], zp = rp[2], gp_ = rp[3], up0 = rp[4], up1 = rp[5], up2 = rp[6];
    const double aE0 = rp[8], aE1 = rp[9], aE2 = rp[10], aB0 = rp[11], aB1 = rp[12], aB2 = rp[13];
    double acc[6] = {0, 0, 0, 0, 0, 0};  // gx(3), gu(3)
    if (tid == 0) {
      wk = 0;
      woff = 0;
      if (W > 0) {
        fence_proxy_async_smem();
        issue(it & 1);
      }
    }
    for (int i = 0; i < W; ++i, ++it) {
      const int bb = it & 1;
      if (tid == 0 && i + 1 < W) {
        fence_proxy_async_smem();
        issue(bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((it >> 1) & 1), status);
      if (ok && active) {
        const int cnt = meta[bb][0], fl = meta[bb][1], first = meta[bb][2];
        for (int j = g; j < cnt; j += G) {
          if (first + j == pi) continue;
          const double *r = &buf[bb][kRecB * j];
          const double rx = xp - r[0], ry = yp - r[1], rz = zp - r[2];
          const double rr = rx * rx + ry * ry + rz * rz;
          if (fl & 1) {
            const double gj = r[3], u0 = r[4], u1 = r[5], u2 = r[6];
            const double ur = u0 * rx + u1 * ry + u2 * rz;
            const double s = rsqrt(rr + ur * ur + kEps64);
            const double f = s * s * s, f5 = f * s * s;
            const double k0 = gj * aE0 + (aB1 * u2 - aB2 * u1);
            const double k1 = gj * aE1 + (aB2 * u0 - aB0 * u2);
            const double k2 = gj * aE2 + (aB0 * u1 - aB1 * u0);
            const double w3 = 3.0 * f5 * (rx * k0 + ry * k1 + rz * k2);
            acc[0] += f * k0 - w3 * (rx + ur * u0);
            acc[1] += f * k1 - w3 * (ry + ur * u1);
            acc[2] += f * k2 - w3 * (rz + ur * u2);
          }
          if (fl & 2) {
            const double e0 = r[8], e1 = r[9], e2 = r[10], h0 = r[11], h1 = r[12], h2 = r[13];
            const double ur = up0 * rx + up1 * ry + up2 * rz;
            const double s = rsqrt(rr + ur * ur + kEps64);
            const double f = s * s * s, f5 = f * s * s;
            const double k0 = gp_ * e0 + (h1 * up2 - h2 * up1);
            const double k1 = gp_ * e1 + (h2 * up0 - h0 * up2);
            const double k2 = gp_ * e2 + (h0 * up1 - h1 * up0);
            const double w3 = 3.0 * f5 * (rx * k0 + ry * k1 + rz * k2);
            acc[0] -= f * k0 - w3 * (rx + ur * up0);
            acc[1] -= f * k1 - w3 * (ry + ur * up1);
            acc[2] -= f * k2 - w3 * (rz + ur * up2);
            const double er = (e0 * rx + e1 * ry + e2 * rz) * f / gp_;
            const double wu = w3 * ur;
            acc[3] += wu * rx - er * up0 - f * (ry * h2 - rz * h1);
            acc[4] += wu * ry - er * up1 - f * (rz * h0 - rx * h2);
            acc[5] += wu * rz - er * up2 - f * (rx * h1 - ry * h0);
          }
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
      for (int o = 1; o < G; o <<= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    if (active && g == 0)
#pragma unroll
      for (int q = 0; q < 6; ++q) gxu[(int64_t)q * N + pi] += acc[q];
  }
}

// ---------------------------------------------------------------- P2P^T, mixed form
// Source records of the mixed adjoint (9 float4, every value duplicated): the
// forward's P2P record (negated hi/lo leaf-local coordinates, gamma, u), the
// particle's field adjoint a_E, a_B and one float4 of padding -- a 144-byte stride
// puts the records that the lane groups of a warp read at once on distinct
// shared-memory banks (a 128-byte stride maps them all to the same four).
__global__ void adj_p2p_rec_kernel(int N, const float4 *__restrict__ prec32x2, const double *__restrict__ adj,
                                   float4 *__restrict__ rec) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  float4 *o = rec + 9 * (int64_t)p;
#pragma unroll
  for (int q = 0; q < 5; ++q) o[q] = prec32x2[5 * (int64_t)p + q];
  float a[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) a[q] = (float)adj[(int64_t)q * N + p];
  o[5] = make_float4(a[0], a[0], a[1], a[1]);
  o[6] = make_float4(a[2], a[2], a[3], a[3]);
  o[7] = make_float4(a[4], a[4], a[5], a[5]);
  o[8] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Per target leaf over its union list, G lanes per pair of target particles, the
// two targets in the two lanes of packed FP32x2 instructions (quantities as in
// p2p_bwd_kernel).  R = x_p - x_j is formed in the source leaf's frame from hi + lo
// parts as in the mixed forward.  The particle itself is skipped, as in the FP64
// adjoint; a distinct particle at the same position keeps the regularised
// kernel's finite derivative (f = eps^-3/2 times c; the f5 term is formed as
// f (s^2 (R.c)) and vanishes without overflowing).  The FP32 partial sums of
// kPbFold tiles at a time are added into FP64 sums in shared memory.  Tiles whose
// boxes are apart by more than 1/kHiOnlyGap of the larger extent form R from the hi
// parts alone, as in the forward.
constexpr int kPbFold = 8;

template <int G>
__global__ void __launch_bounds__(128)
    p2p_bwd_x2_kernel(int leaf0, const int *__restrict__ lohi, const int *__restrict__ ptr,
                      const int *__restrict__ src, const uint8_t *__restrict__ flg, const double *__restrict__ bbox,
                      const float4 *__restrict__ recb, const double *__restrict__ rec16, int N,
                      double *__restrict__ gxu, int *__restrict__ status) {
  constexpr int REC = 9;  // float4 per source record (the last one padding)
  __shared__ __align__(16) float4 buf[2][kPbTile * REC];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_cnt[2], s_flag[2], s_first[2], s_near[2];
  __shared__ double s_centre[2][3];
  __shared__ int s_warp[33];
  __shared__ double s_acc[14][128];  // per thread: gx(3), gu(3), sw of both targets, FP64
  const int tid = threadIdx.x, TG = blockDim.x / G, tl = tid / G, g = tid % G;
  const int c = leaf0 + blockIdx.x;
  const double *tbox = bbox + 6 * (int64_t)c;
  const int tlo = lohi[2 * c], thi = lohi[2 * c + 1], tcnt = thi - tlo + 1;
  const int p0 = ptr[c], np = ptr[c + 1] - p0;
  int w = 0;
  for (int k = tid; k < np; k += blockDim.x) {
    const int s = src[p0 + k];
    w += (lohi[2 * s + 1] - lohi[2 * s] + kPbTile) / kPbTile;
  }
  int W;
  block_excl_scan(w, s_warp, &W);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int wk = 0, woff = 0;
  auto issue = [&](int bb) {
    const int s = src[p0 + wk];
    const int slo = lohi[2 * s], scnt = lohi[2 * s + 1] - slo + 1;
    const int cnt = scnt - woff < kPbTile ? scnt - woff : kPbTile;
    s_cnt[bb] = cnt;
    s_flag[bb] = flg[p0 + wk];
    s_first[bb] = slo + woff;
    const double *sb = bbox + 6 * (int64_t)s;
    s_centre[bb][0] = 0.5 * (sb[0] + sb[3]);
    s_centre[bb][1] = 0.5 * (sb[1] + sb[4]);
    s_centre[bb][2] = 0.5 * (sb[2] + sb[5]);
    s_near[bb] = p2p_tile_needs_lo(sb, tbox);
    const uint32_t bytes = (uint32_t)(cnt * REC * sizeof(float4));
    mbar_arrive_expect_tx(&bar[bb], bytes);
    bulk_g2s(&buf[bb][0], recb + (int64_t)(slo + woff) * REC, bytes, &bar[bb]);
    woff += kPbTile;
    if (woff >= scnt) {
      woff = 0;
      ++wk;
    }
  };
  const float2 z = make_float2(0.f, 0.f), eps = dup2((float)kEps64), three = dup2(3.f);
  int it = 0;
  for (int tc = 0; tc < tcnt; tc += 2 * TG) {
    const int ti0 = tc + tl, ti1 = tc + tl + TG;
    const bool act0 = ti0 < tcnt, act1 = ti1 < tcnt;
    const int64_t pj0 = tlo + (act0 ? ti0 : 0), pj1 = tlo + (act1 ? ti1 : 0);
    const double *r0 = rec16 + kRecB * pj0, *r1 = rec16 + kRecB * pj1;
    auto pr = [&](int q) { return make_float2((float)r0[q], (float)r1[q]); };
    const float2 gp = pr(3), up0 = pr(4), up1 = pr(5), up2 = pr(6);
    const float2 aE0 = pr(8), aE1 = pr(9), aE2 = pr(10), aB0 = pr(11), aB1 = pr(12), aB2 = pr(13);
    const float2 nup0 = make_float2(-up0.x, -up0.y), nup1 = make_float2(-up1.x, -up1.y),
                 nup2 = make_float2(-up2.x, -up2.y);
    const float2 naB0 = make_float2(-aB0.x, -aB0.y), naB1 = make_float2(-aB1.x, -aB1.y),
                 naB2 = make_float2(-aB2.x, -aB2.y);
    const float2 igp = make_float2(1.f / gp.x, 1.f / gp.y);
#pragma unroll
    for (int q = 0; q < 14; ++q) s_acc[q][tid] = 0.0;
    if (tid == 0) {
      wk = 0;
      woff = 0;
      if (W > 0) {
        fence_proxy_async_smem();
        issue(it & 1);
      }
    }
    float2 gx0 = z, gx1 = z, gx2 = z, gu0 = z, gu1 = z, gu2 = z, sw = z, ser = z;
    for (int i = 0; i < W; ++i, ++it) {
      const int bb = it & 1;
      if (tid == 0 && i + 1 < W) {
        fence_proxy_async_smem();
        issue(bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((it >> 1) & 1), status);
      if (ok && act0) {
        const int cnt = s_cnt[bb], fl = s_flag[bb];
        const int self0 = (int)pj0 - s_first[bb], self1 = (int)pj1 - s_first[bb];  // j of the targets themselves
        const double scx = s_centre[bb][0], scy = s_centre[bb][1], scz = s_centre[bb][2];
        // the targets' FP64 coordinates (re-read per tile: L1-resident, saves registers)
        const double dx0 = r0[0] - scx, dy0 = r0[1] - scy, dz0 = r0[2] - scz;
        const double dx1 = r1[0] - scx, dy1 = r1[1] - scy, dz1 = r1[2] - scz;
        const float2 xh = make_float2((float)dx0, (float)dx1), yh = make_float2((float)dy0, (float)dy1),
                     zh = make_float2((float)dz0, (float)dz1);
        const float2 xl = make_float2((float)(dx0 - (double)xh.x), (float)(dx1 - (double)xh.y));
        const float2 yl = make_float2((float)(dy0 - (double)yh.x), (float)(dy1 - (double)yh.y));
        const float2 zl = make_float2((float)(dz0 - (double)zh.x), (float)(dz1 - (double)zh.y));
        const float4 *S = &buf[bb][0];
        auto sweep = [&](auto FL, auto NEARC) {
          constexpr int F = decltype(FL)::value;
          constexpr bool NEAR = decltype(NEARC)::value;
#pragma unroll 2
          for (int j = g; j < cnt; j += G) {
            const float4 *q = S + j * REC;
            const float4 q0 = q[0], q1 = q[1];
            float2 rx, ry, rz;
            if constexpr (NEAR) {
              const float4 q2 = q[2];
              rx = add2(add2(xh, lo2(q0)), add2(xl, hi2(q1)));
              ry = add2(add2(yh, hi2(q0)), add2(yl, lo2(q2)));
              rz = add2(add2(zh, lo2(q1)), add2(zl, hi2(q2)));
            } else {
              rx = add2(xh, lo2(q0));
              ry = add2(yh, hi2(q0));
              rz = add2(zh, lo2(q1));
            }
            const float2 rr = fma2(rx, rx, fma2(ry, ry, mul2(rz, rz)));
            if constexpr ((F & 1) != 0) {  // j's field at the target: uses u_j, gamma_j and the target's a_E, a_B
              const float4 q3 = q[3], q4 = q[4];
              const float2 gj = lo2(q3), uj0 = hi2(q3), uj1 = lo2(q4), uj2 = hi2(q4);
              const float2 ur = fma2(uj2, rz, fma2(uj1, ry, mul2(uj0, rx)));
              const float2 d = fma2(ur, ur, add2(rr, eps));
              float2 sv = rsqrt2(d);
              sv.x = j != self0 ? sv.x : 0.f;
              sv.y = j != self1 ? sv.y : 0.f;
              const float2 s2 = mul2(sv, sv), f = mul2(s2, sv);
              const float2 k0 = fma2(gj, aE0, fma2(aB1, uj2, mul2(naB2, uj1)));
              const float2 k1 = fma2(gj, aE1, fma2(aB2, uj0, mul2(naB0, uj2)));
              const float2 k2 = fma2(gj, aE2, fma2(aB0, uj1, mul2(naB1, uj0)));
              const float2 rk = fma2(rz, k2, fma2(ry, k1, mul2(rx, k0)));
              const float2 nw = mul2(mul2(f, mul2(s2, rk)), dup2(-3.f));  // -3 f5 (R.k), no FP32 overflow
              gx0 = fma2(nw, fma2(ur, uj0, rx), fma2(f, k0, gx0));
              gx1 = fma2(nw, fma2(ur, uj1, ry), fma2(f, k1, gx1));
              gx2 = fma2(nw, fma2(ur, uj2, rz), fma2(f, k2, gx2));
            }
            if constexpr ((F & 2) != 0) {  // the target's field at j: uses u_p, gamma_p and j's a_E, a_B
              const float4 q5 = q[5], q6 = q[6], q7 = q[7];
              const float2 e0 = lo2(q5), e1 = hi2(q5), e2 = lo2(q6), h0 = hi2(q6), h1 = lo2(q7), h2 = hi2(q7);
              const float2 ur = fma2(up2, rz, fma2(up1, ry, mul2(up0, rx)));
              const float2 d = fma2(ur, ur, add2(rr, eps));
              float2 sv = rsqrt2(d);
              sv.x = j != self0 ? sv.x : 0.f;
              sv.y = j != self1 ? sv.y : 0.f;
              const float2 s2 = mul2(sv, sv), f = mul2(s2, sv), nf = make_float2(-f.x, -f.y);
              const float2 k0 = fma2(gp, e0, fma2(h1, up2, mul2(h2, nup1)));
              const float2 k1 = fma2(gp, e1, fma2(h2, up0, mul2(h0, nup2)));
              const float2 k2 = fma2(gp, e2, fma2(h0, up1, mul2(h1, nup0)));
              const float2 rk = fma2(rz, k2, fma2(ry, k1, mul2(rx, k0)));
              const float2 w = mul2(mul2(f, mul2(s2, rk)), three);  // 3 f5 (R.k)
              const float2 wu = mul2(w, ur);
              gx0 = fma2(w, rx, fma2(nf, k0, gx0));  // + w (R + (u_p.R) u_p): the u_p part as sum(wu) u_p
              gx1 = fma2(w, ry, fma2(nf, k1, gx1));
              gx2 = fma2(w, rz, fma2(nf, k2, gx2));
              sw = add2(sw, wu);
              // the gamma_p = sqrt(1 + u_p.u_p) term, (u_p / gamma_p) sum -f (R.e_j), is
              // multiplied out once per tile
              ser = fma2(fma2(rz, e2, fma2(ry, e1, mul2(rx, e0))), nf, ser);
              gu0 = fma2(nf, sub2(mul2(ry, h2), mul2(rz, h1)), fma2(wu, rx, gu0));
              gu1 = fma2(nf, sub2(mul2(rz, h0), mul2(rx, h2)), fma2(wu, ry, gu1));
              gu2 = fma2(nf, sub2(mul2(rx, h1), mul2(ry, h0)), fma2(wu, rz, gu2));
            }
          }
        };
        const std::true_type near_tile{};
        const std::false_type far_tile{};
        if (s_near[bb]) {
          if (fl == 3)
            sweep(std::integral_constant<int, 3>{}, near_tile);
          else if (fl == 1)
            sweep(std::integral_constant<int, 1>{}, near_tile);
          else if (fl == 2)
            sweep(std::integral_constant<int, 2>{}, near_tile);
        } else {
          if (fl == 3)
            sweep(std::integral_constant<int, 3>{}, far_tile);
          else if (fl == 1)
            sweep(std::integral_constant<int, 1>{}, far_tile);
          else if (fl == 2)
            sweep(std::integral_constant<int, 2>{}, far_tile);
        }
      }
      if ((i + 1) % kPbFold == 0 || i + 1 == W) {
        const float2 sg = mul2(ser, igp);
        const float2 part[7] = {gx0, gx1, gx2, fma2(sg, up0, gu0), fma2(sg, up1, gu1), fma2(sg, up2, gu2), sw};
#pragma unroll
        for (int q = 0; q < 7; ++q) {
          s_acc[q][tid] += (double)part[q].x;
          s_acc[7 + q][tid] += (double)part[q].y;
        }
        gx0 = gx1 = gx2 = gu0 = gu1 = gu2 = sw = ser = z;
      }
      __syncthreads();  // buffer bb is refilled two iterations later
    }
    double acc0[6], acc1[6];
    const double sw0 = s_acc[6][tid], sw1 = s_acc[13][tid];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      acc0[q] = s_acc[q][tid] + (q < 3 ? sw0 * r0[4 + q] : 0.0);
      acc1[q] = s_acc[7 + q][tid] + (q < 3 ? sw1 * r1[4 + q] : 0.0);
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        acc0[q] += __shfl_xor_sync(0xffffffffu, acc0[q], o);
        acc1[q] += __shfl_xor_sync(0xffffffffu, acc1[q], o);
      }
    }
    if (g == 0) {
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        if (act0) gxu[(int64_t)q * N + pj0] += acc0[q];
        if (act1) gxu[(int64_t)q * N + pj1] += acc1[q];
      }
    }
  }
}

// ---------------------------------------------------------------- boxes, p_avg, scatter
// A box side of cluster c is attained by argext[c]: pass its adjoint to the child
// holding that particle (levels top-down).
__global__ void box_down_kernel(int l, const int *__restrict__ argext, double *__restrict__ gbox) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (1 << l)) return;
  const int c = (1 << l) - 1 + idx, c1 = 2 * c + 1;
  for (int k = 0; k < 6; ++k) {
    const int who = argext[6 * (int64_t)c1 + k] == argext[6 * (int64_t)c + k] ? c1 : c1 + 1;
    gbox[6 * (int64_t)who + k] += gbox[6 * (int64_t)c + k];
  }
}

__global__ void box_leaf_kernel(int leaf0, int nleaf, const int *__restrict__ argext, const int *__restrict__ invperm,
                                const double *__restrict__ gbox, int N, double *__restrict__ gxu) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nleaf) return;
  const int c = leaf0 + l;
  for (int k = 0; k < 6; ++k) {
    const int d = k % 3;
    const int pos = invperm[argext[6 * (int64_t)c + k]];
    gxu[(int64_t)d * N + pos] += gbox[6 * (int64_t)c + k];
  }
}

__global__ void invperm_kernel(int N, const uint32_t *__restrict__ perm, int *__restrict__ inv) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) inv[perm[p]] = p;
}

// deterministic sum of the per-target p_avg adjoints (single block)
__global__ void pbar_reduce_kernel(int64_t nc, const double *__restrict__ part, double *__restrict__ out) {
  __shared__ double s[3][1024];
  double v[3] = {0, 0, 0};
  for (int64_t c = threadIdx.x; c < nc; c += blockDim.x)
    for (int k = 0; k < 3; ++k) v[k] += part[3 * c + k];
  for (int k = 0; k < 3; ++k) s[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) out[threadIdx.x] = s[threadIdx.x][0];
}

__global__ void grad_scatter_kernel(int N, const uint32_t *__restrict__ perm, const double *__restrict__ gxu,
                                    const double *__restrict__ gpbar, int use_pbar, double *__restrict__ gx,
                                    double *__restrict__ gu) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int64_t o = 3 * (int64_t)perm[p];
  for (int d = 0; d < 3; ++d) {
    gx[o + d] = gxu[(int64_t)d * N + p];
    gu[o + d] = gxu[(int64_t)(3 + d) * N + p] + (use_pbar ? gpbar[d] / (double)N : 0.0);
  }
}

template <int NDEG>
int run_backward_t(Ctx *ctx, const double *d_ge, const double *d_gb, double *d_gx, double *d_gu) {
  using S = BShape<NDEG>;
  constexpr int M = S::M, NN = S::NN, NS = S::NS;
  const int N = (int)ctx->N, ml = ctx->ml;
  const int64_t nc = ctx->nc, nleaf = ctx->nleaf;
  double *adj, *rec16, *gxu, *gloc, *gmom, *gbox, *gpp, *gpbar;
  int *invp;
  FMM_TRY(ctx->ensure("bwd_adj", 6 * (int64_t)N, &adj));
  FMM_TRY(ctx->ensure("bwd_rec16", kRecB * (int64_t)N, &rec16));
  FMM_TRY(ctx->ensure("bwd_gxu", 6 * (int64_t)N, &gxu));
  FMM_TRY(ctx->ensure("bwd_gloc", 6 * NN * nc, &gloc));
  FMM_TRY(ctx->ensure("bwd_gmom", 4 * NN * nc, &gmom));
  FMM_TRY(ctx->ensure("bwd_gbox", 6 * nc, &gbox));
  FMM_TRY(ctx->ensure("bwd_gp_part", 3 * nc, &gpp));
  FMM_TRY(ctx->ensure("bwd_gpbar", 4, &gpbar));
  FMM_TRY(ctx->ensure("bwd_invperm", N, &invp));
  cudaStream_t st = ctx->stream;
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(gloc, 0, sizeof(double) * 6 * NN * nc, st));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(gmom, 0, sizeof(double) * 4 * NN * nc, st));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(gbox, 0, sizeof(double) * 6 * nc, st));
  const uint32_t *perm = ctx->get<uint32_t>("perm");
  const double amp = kRe * ctx->charge / ctx->lambda;
  adj_gather_kernel<<<ceil_div(N, 256), 256, 0, st>>>(N, perm, d_ge, d_gb, amp, ctx->get<double>("prec64"), adj,
                                                      rec16, gxu);
  FMM_TRY(ctx->check_launch("adj_gather_kernel"));
  ChebT ct;
  for (int i = 0; i < kMaxNodes1D; ++i) ct.t[i] = 0.0;
  for (int i = 0; i < M; ++i) ct.t[i] = (std::cos(M_PI * (double)i / (double)NDEG) + 1.0) / 2.0;
  const int *lohi = ctx->get<int>("lohi");
  const double *nodes = ctx->get<double>("nodes"), *bbox = ctx->get<double>("bbox");
  const double *prec = ctx->get<double>("prec64");
  const double *loc = ctx->get<double>("loc64"), *mom = ctx->get<double>("mom64");
  // L2P^T
  {
    auto k = leaf_bwd_kernel<NDEG, 0>;
    const int sm = 6 * NN * 8;
    FMM_TRY(opt_in_smem(ctx, k, sm));
    k<<<(unsigned)nleaf, 128, sm, st>>>((int)ctx->leaf0, lohi, nodes, bbox, prec, loc, adj, N, gxu, gloc, gbox);
    FMM_TRY(ctx->check_launch("leaf_bwd_kernel<L2P>"));
  }
  // L2L^T, children at levels ml .. 1
  {
    auto k = transfer_bwd_kernel<NDEG, 0>;
    const int sm = (4 * 6 + 3) * NN * 8;
    FMM_TRY(opt_in_smem(ctx, k, sm));
    for (int l = ml; l >= 1; --l) {
      k<<<1u << (l - 1), S::BT, sm, st>>>(l - 1, nodes, bbox, ct, gloc, loc, gloc, gbox);
      FMM_TRY(ctx->check_launch("transfer_bwd_kernel<L2L>"));
    }
  }
  // M2L^T over the union lists (coincident nodes are possible only for eta > 1/2)
  const bool mask = !(ctx->eta <= 0.5);
  if (ctx->precision == FMMB200_PRECISION_MIXED) {
    using S2 = MBShape2<NDEG>;
    float *rec32;
    FMM_TRY(ctx->ensure("bwd_rec32", (int64_t)S2::RECF * nc, &rec32));
    adj_rec32_kernel<NDEG><<<592, 256, 0, st>>>(nc, ctx->get<float>("mom32"), gloc, rec32);
    FMM_TRY(ctx->check_launch("adj_rec32_kernel"));
    // n = 8 keeps the packed kernel: one node per thread would need 736 threads per CTA
    if (mask || NDEG >= 8) {
      auto k = mask ? m2l_bwd_x2_kernel<NDEG, true> : m2l_bwd_x2_kernel<NDEG, false>;
      FMM_TRY(opt_in_smem(ctx, k, S2::SMEM));
      k<<<(unsigned)nc, S2::BT, S2::SMEM, st>>>(ctx->get<int>("m2lu_ptr"), ctx->get<int>("m2lu_src"),
                                                ctx->get<uint8_t>("m2lu_flag"), nodes, bbox, ct, rec32,
                                                ctx->get<double>("consts"), gmom, gbox, gpp, ctx->d_status);
      FMM_TRY(ctx->check_launch("m2l_bwd_x2_kernel"));
    } else if constexpr (NDEG < 8) {
      using SF = MBShape1F<NDEG>;
      auto k = m2l_bwd_x1f_kernel<NDEG>;
      FMM_TRY(opt_in_smem(ctx, k, SF::SMEM));
      k<<<(unsigned)nc, SF::BT, SF::SMEM, st>>>(ctx->get<int>("m2lu_ptr"), ctx->get<int>("m2lu_src"),
                                                ctx->get<uint8_t>("m2lu_flag"), nodes, bbox, ct, rec32,
                                                ctx->get<double>("consts"), gmom, gbox, gpp, ctx->d_status);
      FMM_TRY(ctx->check_launch("m2l_bwd_x1f_kernel"));
    }
  } else {
    auto k = mask ? m2l_bwd_kernel<NDEG, true> : m2l_bwd_kernel<NDEG, false>;
    const int sm = 2 * (10 * NN + NS) * 8;
    FMM_TRY(opt_in_smem(ctx, k, sm));
    k<<<(unsigned)nc, S::BT, sm, st>>>(ctx->get<int>("m2lu_ptr"), ctx->get<int>("m2lu_src"),
                                        ctx->get<uint8_t>("m2lu_flag"), nodes, ct, mom, gloc, ctx->get<double>("consts"),
                                        gmom, gbox, gpp, ctx->d_status);
    FMM_TRY(ctx->check_launch("m2l_bwd_kernel"));
  }
  // M2M^T, parents at levels 0 .. ml-1 (top-down)
  {
    auto k = transfer_bwd_kernel<NDEG, 1>;
    const int sm = (4 * 4 + 3) * NN * 8;
    FMM_TRY(opt_in_smem(ctx, k, sm));
    for (int l = 0; l < ml; ++l) {
      k<<<1u << l, S::BT, sm, st>>>(l, nodes, bbox, ct, mom, gmom, gmom, gbox);
      FMM_TRY(ctx->check_launch("transfer_bwd_kernel<M2M>"));
    }
  }
  // P2M^T
  {
    auto k = leaf_bwd_kernel<NDEG, 1>;
    const int sm = 4 * NN * 8;
    FMM_TRY(opt_in_smem(ctx, k, sm));
    k<<<(unsigned)nleaf, 128, sm, st>>>((int)ctx->leaf0, lohi, nodes, bbox, prec, gmom, adj, N, gxu, gloc, gbox);
    FMM_TRY(ctx->check_launch("leaf_bwd_kernel<P2M>"));
  }
  // P2P^T (G lanes per target particle as in the forward)
  if (ctx->precision == FMMB200_PRECISION_MIXED) {
    float4 *recb;
    FMM_TRY(ctx->ensure("bwd_p2p_rec", 9 * (int64_t)N, &recb));
    adj_p2p_rec_kernel<<<ceil_div(N, 256), 256, 0, st>>>(N, ctx->get<float4>("prec32x2"), adj, recb);
    FMM_TRY(ctx->check_launch("adj_p2p_rec_kernel"));
    const int *pp = ctx->get<int>("p2pu_ptr"), *ps = ctx->get<int>("p2pu_src");
    const uint8_t *pf = ctx->get<uint8_t>("p2pu_flag");
    // two targets per lane group: G lanes share them (as in the mixed forward)
    if (ctx->max_leaf <= 32)
      p2p_bwd_x2_kernel<8><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, bbox, recb, rec16, N,
                                                            gxu, ctx->d_status);
    else if (ctx->max_leaf <= 64)
      p2p_bwd_x2_kernel<4><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, bbox, recb, rec16, N,
                                                            gxu, ctx->d_status);
    else if (ctx->max_leaf <= 128)
      p2p_bwd_x2_kernel<2><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, bbox, recb, rec16, N,
                                                            gxu, ctx->d_status);
    else
      p2p_bwd_x2_kernel<1><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, bbox, recb, rec16, N,
                                                            gxu, ctx->d_status);
    FMM_TRY(ctx->check_launch("p2p_bwd_x2_kernel"));
  } else {
    const int *pp = ctx->get<int>("p2pu_ptr"), *ps = ctx->get<int>("p2pu_src");
    const uint8_t *pf = ctx->get<uint8_t>("p2pu_flag");
    if (ctx->max_leaf <= 32)
      p2p_bwd_kernel<4><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, rec16, N, gxu, ctx->d_status);
    else if (ctx->max_leaf <= 64)
      p2p_bwd_kernel<2><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, rec16, N, gxu, ctx->d_status);
    else
      p2p_bwd_kernel<1><<<(unsigned)nleaf, 128, 0, st>>>((int)ctx->leaf0, lohi, pp, ps, pf, rec16, N, gxu, ctx->d_status);
    FMM_TRY(ctx->check_launch("p2p_bwd_kernel"));
  }
  // boxes -> extremal particles; p_avg -> every momentum; scatter to caller order
  const int *argext = ctx->get<int>("argext");
  for (int l = 0; l < ml; ++l) {
    box_down_kernel<<<ceil_div(1 << l, 256), 256, 0, st>>>(l, argext, gbox);
    FMM_TRY(ctx->check_launch("box_down_kernel"));
  }
  invperm_kernel<<<ceil_div(N, 256), 256, 0, st>>>(N, perm, invp);
  box_leaf_kernel<<<ceil_div(nleaf, 256), 256, 0, st>>>((int)ctx->leaf0, (int)nleaf, argext, invp, gbox, N, gxu);
  pbar_reduce_kernel<<<1, 1024, 0, st>>>(nc, gpp, gpbar);
  grad_scatter_kernel<<<ceil_div(N, 256), 256, 0, st>>>(N, perm, gxu, gpbar, ctx->pavg_from_momenta ? 1 : 0, d_gx,
                                                        d_gu);
  FMM_TRY(ctx->check_launch("box/pbar/scatter kernels", 4));
  return FMMB200_OK;
}

}  // namespace

int run_backward(Ctx *ctx, const double *d_ge, const double *d_gb, double *d_gx, double *d_gu) {
  switch (ctx->n) {
    case 1: return run_backward_t<1>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 2: return run_backward_t<2>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 3: return run_backward_t<3>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 4: return run_backward_t<4>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 5: return run_backward_t<5>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 6: return run_backward_t<6>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 7: return run_backward_t<7>(ctx, d_ge, d_gb, d_gx, d_gu);
    case 8: return run_backward_t<8>(ctx, d_ge, d_gb, d_gx, d_gu);
    default:
      return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "the adjoint supports degrees n = 1..8");
  }
}

}  // namespace fmmb200
