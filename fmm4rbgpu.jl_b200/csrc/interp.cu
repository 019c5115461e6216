// interp.cu -- the Lagrange-interpolation passes on tensor grids of Chebyshev
// points of the second kind:
//   P2M  leaf moments            (gpu_P2M!, src/gpu_fmm/gpu_upwardpass.jl:3-85)
//   M2M  parent moments          (gpu_M2M!, src/gpu_fmm/gpu_upwardpass.jl:87-163)
//   L2L  child local fields      (gpu_L2L!, src/gpu_fmm/gpu_downwardpass.jl:4-74)
//   L2P  particle far fields     (gpu_L2P!, src/gpu_fmm/gpu_downwardpass.jl:76-145)
// with barycentric weights w_i(x) = (ws_i/(x - x_i)) / sum_j ws_j/(x - x_j) and
// the exact-node rule |x - x_i| < eps(Float64) -> indicator of the last such node.
//
// B200 design: moments and locals are stored per cluster as contiguous SoA
// records ([Gamma|Mx|My|Mz], [Ex|Ey|Ez|Bx|By|Bz], node index i fastest), so
// every CTA streams one record.  M2M and L2L use the tensor structure: the
// weight of parent node I at child node i factorises per axis, so the (n+1)^6
// dense transfer of the reference becomes three (n+1)x(n+1) contractions per
// quantity, O((n+1)^4), staged in shared memory.  L2P fuses the far field with
// the P2P near field, the amp normalisation and the scatter back to the
// caller's particle order.
#include "device_util.cuh"
#include "interp_util.cuh"
#include "kernels.cuh"

namespace fmmb200 {

namespace {

template <int NDEG>
struct Grid {
  static constexpr int M = NDEG + 1;
  static constexpr int NN = M * M * M;
  static constexpr int NS = ((3 * M) + 1) & ~1;
  static constexpr int BT = NN <= 64 ? 64 : (NN <= 512 ? ((NN + 31) / 32) * 32 : 512);
  static constexpr int NPT = (NN + BT - 1) / BT;
};

constexpr int kP2MChunk = 64;

// ---------------------------------------------------------------- P2M
template <int NDEG, bool MIXED>
__global__ void __launch_bounds__(Grid<NDEG>::BT)
    p2m_kernel(const int *__restrict__ leaf_ids, int leaf0, const int *__restrict__ lohi,
               const double *__restrict__ nodes, const double *__restrict__ bbox, const void *__restrict__ prec_v,
               void *__restrict__ mom_v, int accumulate) {
  using Gd = Grid<NDEG>;
  constexpr int M = Gd::M, NN = Gd::NN, NS = Gd::NS, BT = Gd::BT, NPT = Gd::NPT;
  using T = typename std::conditional<MIXED, float, double>::type;
  __shared__ T s_w[kP2MChunk][3][M];
  __shared__ T s_q[kP2MChunk][4];
  __shared__ double s_n64[3 * M];
  __shared__ float s_n32[3 * M];
  const int tid = threadIdx.x;
  const int c = leaf_ids ? leaf_ids[blockIdx.x] : leaf0 + blockIdx.x;
  const int lo = lohi[2 * c], hi = lohi[2 * c + 1];
  const double *bb = bbox + 6 * (int64_t)c;
  for (int i = tid; i < 3 * M; i += BT) {
    const double v = nodes[(int64_t)c * NS + i];
    s_n64[i] = v;
    const int d = i / M;
    s_n32[i] = (float)(v - 0.5 * (bb[d] + bb[3 + d]));
  }
  T acc[NPT][4];
#pragma unroll
  for (int r = 0; r < NPT; ++r) acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = (T)0;
  __syncthreads();
  for (int c0 = lo; c0 <= hi; c0 += kP2MChunk) {
    const int cnt = (hi - c0 + 1) < kP2MChunk ? (hi - c0 + 1) : kP2MChunk;
    for (int task = tid; task < 3 * cnt; task += BT) {
      const int p = task / 3, d = task % 3;
      if constexpr (MIXED) {
        const float x = ((const float *)prec_v)[(int64_t)(c0 + p) * 8 + d];
        weights32<M>(x, s_n32 + d * M, s_w[p][d]);
      } else {
        const double x = ((const double *)prec_v)[(int64_t)(c0 + p) * 8 + d];
        weights64<M>(x, s_n64 + d * M, s_w[p][d]);
      }
    }
    for (int p = tid; p < cnt; p += BT) {
      const T *r = (const T *)prec_v + (int64_t)(c0 + p) * 8;
      s_q[p][0] = r[3];
      s_q[p][1] = r[4];
      s_q[p][2] = r[5];
      s_q[p][3] = r[6];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int a = tid + r * BT;
      if (a < NN) {
        const int ai = a % M, aj = (a / M) % M, ak = a / (M * M);
        for (int p = 0; p < cnt; ++p) {
          const T w = s_w[p][0][ai] * s_w[p][1][aj] * s_w[p][2][ak];
          acc[r][0] += s_q[p][0] * w;
          acc[r][1] += s_q[p][1] * w;
          acc[r][2] += s_q[p][2] * w;
          acc[r][3] += s_q[p][3] * w;
        }
      }
    }
    __syncthreads();
  }
  T *out = (T *)mom_v + (int64_t)c * 4 * NN;
#pragma unroll
  for (int r = 0; r < NPT; ++r) {
    const int a = tid + r * BT;
    if (a < NN) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        T v = acc[r][q];
        if (accumulate) v += out[q * NN + a];
        out[q * NN + a] = v;
      }
    }
  }
}

// L[c][d][i][I]: weight of parent node I at coordinate d of child node i, for the nch
// children c1, c1 + 1 (nch = 1: c1 only)
template <int M, typename T>
__device__ __forceinline__ void transfer_weights(const double *__restrict__ nodes, int NS, int p, int c1,
                                                 T (*L)[3][M][M], int nch = 2) {
  for (int task = threadIdx.x; task < nch * 3 * M; task += blockDim.x) {
    const int ch = task / (3 * M), r = task % (3 * M), d = r / M, i = r % M;
    const int c = c1 + ch;
    const double x = nodes[(int64_t)c * NS + d * M + i];
    weights64<M>(x, nodes + (int64_t)p * NS + d * M, L[ch][d][i]);
  }
}

// ---------------------------------------------------------------- M2M
// The tree is a heap stored from cluster `off` on (off = 0: the whole tree; a sharded
// rank keeps the top levels of the beam's tree at an offset).
template <int NDEG, bool MIXED>
__global__ void __launch_bounds__(Grid<NDEG>::BT)
    m2m_kernel(int plevel, int off, const double *__restrict__ nodes, void *__restrict__ mom_v, int accumulate) {
  using Gd = Grid<NDEG>;
  constexpr int M = Gd::M, NN = Gd::NN, NS = Gd::NS, BT = Gd::BT, NPT = Gd::NPT;
  using T = typename std::conditional<MIXED, float, double>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ T L[2][3][M][M];
  T *s_in = (T *)smem;      // 4*NN
  T *s_t1 = s_in + 4 * NN;  // 4*NN
  T *s_t2 = s_t1 + 4 * NN;  // 4*NN
  T *mom = (T *)mom_v;
  const int tid = threadIdx.x;
  const int p = off + (1 << plevel) - 1 + blockIdx.x;
  const int c1 = off + 2 * (p - off) + 1;
  transfer_weights<M, T>(nodes, NS, p, c1, L);
  T acc[NPT][4];
#pragma unroll
  for (int r = 0; r < NPT; ++r) acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = (T)0;
  for (int ch = 0; ch < 2; ++ch) {
    const T *cm = mom + (int64_t)(c1 + ch) * 4 * NN;
    for (int e = tid; e < 4 * NN; e += BT) s_in[e] = cm[e];
    __syncthreads();
    // x: t1[q][I + M(j + Mk)] = sum_i L[x][i][I] in[q][i + M(j + Mk)]
    for (int e = tid; e < 4 * NN; e += BT) {
      const int q = e / NN, o = e % NN, I = o % M, jk = o / M;
      const T *src = s_in + q * NN + M * jk;
      T v = 0;
#pragma unroll
      for (int i = 0; i < M; ++i) v += L[ch][0][i][I] * src[i];
      s_t1[e] = v;
    }
    __syncthreads();
    // y: t2[q][I + M(J + Mk)] = sum_j L[y][j][J] t1[q][I + M(j + Mk)]
    for (int e = tid; e < 4 * NN; e += BT) {
      const int q = e / NN, o = e % NN, I = o % M, J = (o / M) % M, k = o / (M * M);
      const T *src = s_t1 + q * NN + I + M * M * k;
      T v = 0;
#pragma unroll
      for (int j = 0; j < M; ++j) v += L[ch][1][j][J] * src[M * j];
      s_t2[e] = v;
    }
    __syncthreads();
    // z: parent[q][I + M(J + MK)] += sum_k L[z][k][K] t2[q][I + M(J + Mk)]
#pragma unroll
    for (int r = 0; r < NPT; ++r) {
      const int a = tid + r * BT;
      if (a < NN) {
        const int IJ = a % (M * M), K = a / (M * M);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const T *src = s_t2 + q * NN + IJ;
          T v = 0;
#pragma unroll
          for (int k = 0; k < M; ++k) v += L[ch][2][k][K] * src[M * M * k];
          acc[r][q] += v;
        }
      }
    }
    __syncthreads();
  }
  T *out = mom + (int64_t)p * 4 * NN;
#pragma unroll
  for (int r = 0; r < NPT; ++r) {
    const int a = tid + r * BT;
    if (a < NN) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        T v = acc[r][q];
        if (accumulate) v += out[q * NN + a];
        out[q * NN + a] = v;
      }
    }
  }
}

// ---------------------------------------------------------------- L2L
// One CTA per parent at level clevel-1 of the heap stored from cluster `off`; both
// children receive
// child[q][i + M(j + Mk)] += sum_{IJK} parent[q][I + M(J + MK)] Lx[i][I] Ly[j][J] Lz[k][K].
// With pc given, CTA b instead transfers parent pc[b].x into the one child pc[b].y.
template <int NDEG, bool MIXED>
__global__ void __launch_bounds__(Grid<NDEG>::BT)
    l2l_kernel(int clevel, int off, const int2 *__restrict__ pc, const double *__restrict__ nodes,
               void *__restrict__ loc_v) {
  using Gd = Grid<NDEG>;
  constexpr int M = Gd::M, NN = Gd::NN, NS = Gd::NS, BT = Gd::BT;
  using T = typename std::conditional<MIXED, float, double>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ T L[2][3][M][M];
  T *s_par = (T *)smem;       // 6*NN
  T *s_t1 = s_par + 6 * NN;   // 6*NN
  T *s_t2 = s_t1 + 6 * NN;    // 6*NN
  T *loc = (T *)loc_v;
  const int tid = threadIdx.x;
  const int p = pc ? pc[blockIdx.x].x : off + (1 << (clevel - 1)) - 1 + blockIdx.x;
  const int c1 = pc ? pc[blockIdx.x].y : off + 2 * (p - off) + 1;
  const int nch = pc ? 1 : 2;
  transfer_weights<M, T>(nodes, NS, p, c1, L, nch);
  const T *pl = loc + (int64_t)p * 6 * NN;
  for (int e = tid; e < 6 * NN; e += BT) s_par[e] = pl[e];
  __syncthreads();
  // all six quantities per stage; the z stage of one child reads only t2, which the
  // next child's y stage rewrites after the barrier that follows its x stage
  for (int ch = 0; ch < nch; ++ch) {
    T *cl = loc + (int64_t)(c1 + ch) * 6 * NN;
    // x: t1[q][i + M(J + MK)] = sum_I Lx[i][I] par[q][I + M(J + MK)]
    for (int e = tid; e < 6 * NN; e += BT) {
      const int i = e % M, qJK = e / M;
      const T *src = s_par + M * qJK;
      T v = 0;
#pragma unroll
      for (int I = 0; I < M; ++I) v += L[ch][0][i][I] * src[I];
      s_t1[e] = v;
    }
    __syncthreads();
    // y: t2[q][i + M(j + MK)] = sum_J Ly[j][J] t1[q][i + M(J + MK)]
    for (int e = tid; e < 6 * NN; e += BT) {
      const int i = e % M, j = (e / M) % M, qK = e / (M * M);
      const T *src = s_t1 + i + M * M * qK;
      T v = 0;
#pragma unroll
      for (int J = 0; J < M; ++J) v += L[ch][1][j][J] * src[M * J];
      s_t2[e] = v;
    }
    __syncthreads();
    // z: child[q][i + M(j + Mk)] += sum_K Lz[k][K] t2[q][i + M(j + MK)]
    for (int e = tid; e < 6 * NN; e += BT) {
      const int q = e / NN, o = e - q * NN, ij = o % (M * M), k = o / (M * M);
      const T *src = s_t2 + q * NN + ij;
      T v = 0;
#pragma unroll
      for (int K = 0; K < M; ++K) v += L[ch][2][k][K] * src[M * M * K];
      cl[e] += v;
    }
  }
}

// ---------------------------------------------------------------- L2P
// mode 0: near[q][p] += far (tree order); mode 1: out[perm[p]] = amp*(near + far).
// Two threads per particle: h = 0 evaluates the E components, h = 1 the B
// components of the leaf's local expansion, as three independent accumulation
// chains over the tensor-product grid.  The leaf's locals sit in shared memory
// with each x-row padded to a whole number of 16-byte vectors, so a row of M
// values costs ceil(M / 4) (FP32) or ceil(M / 2) (FP64) shared loads instead of M.
__device__ __forceinline__ void unpack_vec(float4 v, float *a) {
  a[0] = v.x;
  a[1] = v.y;
  a[2] = v.z;
  a[3] = v.w;
}
__device__ __forceinline__ void unpack_vec(double2 v, double *a) {
  a[0] = v.x;
  a[1] = v.y;
}

template <typename T, int M>
struct L2PRows {
  static constexpr int VE = 16 / (int)sizeof(T);          // values per 16-byte load
  static constexpr int NV = (M + VE - 1) / VE;            // loads per row
  static constexpr int RS = NV * VE;                      // padded row stride
  static constexpr int SMEM = 6 * M * M * RS * (int)sizeof(T);
};

template <int NDEG, bool MIXED>
__global__ void __launch_bounds__(128)
    l2p_kernel(const int *__restrict__ leaf_ids, int leaf0, const int *__restrict__ lohi,
               const double *__restrict__ nodes, const double *__restrict__ bbox, const void *__restrict__ prec_v,
               const void *__restrict__ loc_v, double *__restrict__ near, int N, int mode, double amp,
               const uint32_t *__restrict__ perm, double *__restrict__ out_e, double *__restrict__ out_b) {
  using Gd = Grid<NDEG>;
  constexpr int M = Gd::M, NN = Gd::NN, NS = Gd::NS;
  using T = typename std::conditional<MIXED, float, double>::type;
  using V = typename std::conditional<MIXED, float4, double2>::type;
  using Rw = L2PRows<T, M>;
  constexpr int RS = Rw::RS, NV = Rw::NV, VE = Rw::VE;
  extern __shared__ __align__(16) unsigned char smem[];
  T *s_loc = (T *)smem;  // [6 M M][RS]
  __shared__ double s_n64[3 * M];
  __shared__ float s_n32[3 * M];
  const int tid = threadIdx.x;
  const int h = tid & 1;
  const int c = leaf_ids ? leaf_ids[blockIdx.x] : leaf0 + blockIdx.x;
  const int lo = lohi[2 * c], hi = lohi[2 * c + 1];
  const double *bb = bbox + 6 * (int64_t)c;
  const T *lc = (const T *)loc_v + (int64_t)c * 6 * NN;
  for (int e = tid; e < 6 * M * M * RS; e += blockDim.x) {
    const int row = e / RS, i = e - row * RS;
    s_loc[e] = i < M ? lc[row * M + i] : T(0);
  }
  for (int i = tid; i < 3 * M; i += blockDim.x) {
    const double v = nodes[(int64_t)c * NS + i];
    s_n64[i] = v;
    const int d = i / M;
    s_n32[i] = (float)(v - 0.5 * (bb[d] + bb[3 + d]));
  }
  __syncthreads();
  const T *L0 = s_loc + (3 * h) * M * M * RS, *L1 = L0 + M * M * RS, *L2 = L1 + M * M * RS;
  for (int p = lo + (tid >> 1); p <= hi; p += blockDim.x >> 1) {
    T wx[M], wy[M], wz[M];
    if constexpr (MIXED) {
      const float *r = (const float *)prec_v + (int64_t)p * 8;
      weights32_fast<M>(r[0], s_n32, wx);
      weights32_fast<M>(r[1], s_n32 + M, wy);
      weights32_fast<M>(r[2], s_n32 + 2 * M, wz);
    } else {
      const double *r = (const double *)prec_v + (int64_t)p * 8;
      weights64<M>(r[0], s_n64, wx);
      weights64<M>(r[1], s_n64 + M, wy);
      weights64<M>(r[2], s_n64 + 2 * M, wz);
    }
    T f0 = 0, f1 = 0, f2 = 0;
#pragma unroll 1
    for (int k = 0; k < M; ++k) {
      T y0 = 0, y1 = 0, y2 = 0;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const int o = RS * (j + M * k);
        T x0 = 0, x1 = 0, x2 = 0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          T a0[VE], a1[VE], a2[VE];
          unpack_vec(*(const V *)(L0 + o + v * VE), a0);
          unpack_vec(*(const V *)(L1 + o + v * VE), a1);
          unpack_vec(*(const V *)(L2 + o + v * VE), a2);
#pragma unroll
          for (int u = 0; u < VE; ++u) {
            const int i = v * VE + u;
            if (i < M) {
              x0 += wx[i] * a0[u];
              x1 += wx[i] * a1[u];
              x2 += wx[i] * a2[u];
            }
          }
        }
        y0 += wy[j] * x0;
        y1 += wy[j] * x1;
        y2 += wy[j] * x2;
      }
      f0 += wz[k] * y0;
      f1 += wz[k] * y1;
      f2 += wz[k] * y2;
    }
    const double f[3] = {(double)f0, (double)f1, (double)f2};
    if (mode == 0) {
#pragma unroll
      for (int q = 0; q < 3; ++q) near[(int64_t)(3 * h + q) * N + p] += f[q];
    } else {
      const int64_t o = 3 * (int64_t)perm[p];
      double *out = h == 0 ? out_e : out_b;
#pragma unroll
      for (int q = 0; q < 3; ++q) out[o + q] = amp * (near[(int64_t)(3 * h + q) * N + p] + f[q]);
    }
  }
}

template <int NDEG, bool MIXED>
struct Launch {
  using Gd = Grid<NDEG>;
  using T = typename std::conditional<MIXED, float, double>::type;
  static int p2m(Ctx *ctx, const int *ids, int64_t nleaf, bool accumulate) {
    if (nleaf <= 0) return FMMB200_OK;
    p2m_kernel<NDEG, MIXED><<<(unsigned)nleaf, Gd::BT, 0, ctx->stream>>>(
        ids, (int)ctx->leaf0, ctx->get<int>("lohi"), ctx->get<double>("nodes"), ctx->get<double>("bbox"),
        MIXED ? (const void *)ctx->get<float>("prec32") : (const void *)ctx->get<double>("prec64"),
        MIXED ? (void *)ctx->get<float>("mom32") : (void *)ctx->get<double>("mom64"), accumulate ? 1 : 0);
    return ctx->check_launch("p2m_kernel");
  }
  static int m2m(Ctx *ctx, int plevel, bool accumulate, int off = 0) {
    const int smem = 3 * 4 * Gd::NN * (int)sizeof(T);
    auto k = m2m_kernel<NDEG, MIXED>;
    FMM_TRY(opt_in_smem(ctx, k, smem));
    k<<<1u << plevel, Gd::BT, smem, ctx->stream>>>(
        plevel, off, ctx->get<double>("nodes"),
        MIXED ? (void *)ctx->get<float>("mom32") : (void *)ctx->get<double>("mom64"), accumulate ? 1 : 0);
    return ctx->check_launch("m2m_kernel");
  }
  static int l2l(Ctx *ctx, int clevel, int off = 0, const int2 *pc = nullptr, int npc = 0) {
    const int smem = 18 * Gd::NN * (int)sizeof(T);
    auto k = l2l_kernel<NDEG, MIXED>;
    FMM_TRY(opt_in_smem(ctx, k, smem));
    const unsigned grid = pc ? (unsigned)npc : 1u << (clevel - 1);
    if (grid == 0) return FMMB200_OK;
    k<<<grid, Gd::BT, smem, ctx->stream>>>(
        clevel, off, pc, ctx->get<double>("nodes"),
        MIXED ? (void *)ctx->get<float>("loc32") : (void *)ctx->get<double>("loc64"));
    return ctx->check_launch("l2l_kernel");
  }
  static int l2p(Ctx *ctx, const int *ids, int64_t nleaf, int mode, double amp, double *oe, double *ob) {
    if (nleaf <= 0) return FMMB200_OK;
    const int smem = L2PRows<T, Gd::M>::SMEM;
    auto k = l2p_kernel<NDEG, MIXED>;
    FMM_TRY(opt_in_smem(ctx, k, smem));
    k<<<(unsigned)nleaf, 128, smem, ctx->stream>>>(
        ids, (int)ctx->leaf0, ctx->get<int>("lohi"), ctx->get<double>("nodes"), ctx->get<double>("bbox"),
        MIXED ? (const void *)ctx->get<float>("prec32") : (const void *)ctx->get<double>("prec64"),
        MIXED ? (const void *)ctx->get<float>("loc32") : (const void *)ctx->get<double>("loc64"),
        ctx->get<double>("near"), (int)ctx->N, mode, amp, ctx->get<uint32_t>("perm"), oe, ob);
    return ctx->check_launch("l2p_kernel");
  }
};

}  // namespace

#define FMM_DISPATCH(n, mixed, CALL)                                              \
  switch (n) {                                                                    \
    case 1: return mixed ? Launch<1, true>::CALL : Launch<1, false>::CALL;        \
    case 2: return mixed ? Launch<2, true>::CALL : Launch<2, false>::CALL;        \
    case 3: return mixed ? Launch<3, true>::CALL : Launch<3, false>::CALL;        \
    case 4: return mixed ? Launch<4, true>::CALL : Launch<4, false>::CALL;        \
    case 5: return mixed ? Launch<5, true>::CALL : Launch<5, false>::CALL;        \
    case 6: return mixed ? Launch<6, true>::CALL : Launch<6, false>::CALL;        \
    case 7: return mixed ? Launch<7, true>::CALL : Launch<7, false>::CALL;        \
    case 8: return mixed ? Launch<8, true>::CALL : Launch<8, false>::CALL;        \
    case 9: return mixed ? Launch<9, true>::CALL : Launch<9, false>::CALL;        \
    case 10: return mixed ? Launch<10, true>::CALL : Launch<10, false>::CALL;     \
    default: return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "degree n must be in 1..10"); \
  }

int launch_p2m(Ctx *ctx, int n, bool mixed, const int *ids, int64_t nleaf, bool accumulate) {
  FMM_DISPATCH(n, mixed, p2m(ctx, ids, nleaf, accumulate))
}
int launch_m2m(Ctx *ctx, int n, bool mixed, int plevel, bool accumulate) {
  FMM_DISPATCH(n, mixed, m2m(ctx, plevel, accumulate))
}
int launch_l2l(Ctx *ctx, int n, bool mixed, int clevel) { FMM_DISPATCH(n, mixed, l2l(ctx, clevel)) }
int launch_m2m_heap(Ctx *ctx, int n, bool mixed, int plevel, int off) {
  FMM_DISPATCH(n, mixed, m2m(ctx, plevel, false, off))
}
int launch_l2l_heap(Ctx *ctx, int n, bool mixed, int clevel, int off) {
  FMM_DISPATCH(n, mixed, l2l(ctx, clevel, off))
}
int launch_l2l_pairs(Ctx *ctx, int n, bool mixed, const int2 *d_pc, int npc) {
  FMM_DISPATCH(n, mixed, l2l(ctx, 1, 0, d_pc, npc))
}
int launch_l2p(Ctx *ctx, int n, bool mixed, const int *ids, int64_t nleaf, int mode, double amp, double *oe,
               double *ob) {
  FMM_DISPATCH(n, mixed, l2p(ctx, ids, nleaf, mode, amp, oe, ob))
}

}  // namespace fmmb200
