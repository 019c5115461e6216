// p2p.cu -- P2P near field (the reference's gpu_P2P!,
// src/gpu_fmm/gpu_interaction.jl:43-86, and P2P!, src/fmm/interaction.jl:49-75):
//   E_i += sum_j gamma_j K(x_i - x_j; u_j),  B_i += sum_j u_j x K(x_i - x_j; u_j)
// over the particles j of every source leaf in target leaf i's P2P list (j = i
// gives R = 0 and K = 0, as in the reference).
//
// Design: one CTA per target leaf.  Particles are stored in tree order as
// 64-byte (FP64) or 32-byte (FP32) records, so every source leaf is one
// contiguous range: tiles of up to 128 source records are bulk-copied (TMA)
// into a double buffer guarded by mbarriers.  G adjacent lanes share a target
// particles (each lane holds two targets, which share every staged source
// record) and split the sources; their partial fields are combined with warp
// shuffles.  G is chosen from the leaf size so that small leaves (64 particles
// at N0 = 125) still fill the CTA -- the reference launches N0 threads per
// leaf and leaves about half of them idle.
//
// Mixed form: FP32 arithmetic on coordinates relative to the source leaf's box
// centre, each stored as a hi + lo pair of floats.  Per tile the target is moved
// into the source's frame in FP64 once and split the same way; every pair
// difference R = (X_hi - x_hi) + (X_lo - x_lo) is then formed to ~1 ulp of |R|
// even for very close pairs (the hi difference is exact, Sterbenz), which a
// plain FP32 leaf-local coordinate cannot give.  Per-tile partial sums are
// folded into Kahan-compensated FP32 accumulators; the output is FP64.
#include "device_util.cuh"
#include "kernels.cuh"

namespace fmmb200 {

namespace {

constexpr int kP2PTile = 128;

__device__ __forceinline__ float rsqrt_approx_p(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct TileMeta {
  int cnt;
  double scx, scy, scz;  // mixed: the source leaf's box centre
};

// Two target particles per thread (TT = 2) share every staged source record.
constexpr int kTT = 2;

template <int G, bool MIXED>
__global__ void __launch_bounds__(128) p2p_kernel(const int *__restrict__ leaf_ids, int leaf0,
                                                  const int *__restrict__ lohi, const int *__restrict__ ptr,
                                                  const int *__restrict__ src, const double *__restrict__ bbox,
                                                  const void *__restrict__ prec_v, const float4 *__restrict__ lo32,
                                                  const double *__restrict__ prec64, double *__restrict__ near,
                                                  int N, int accumulate, int *__restrict__ status) {
  using T = typename std::conditional<MIXED, float, double>::type;
  constexpr int REC = 8;  // T values per particle record
  __shared__ __align__(16) T buf[2][kP2PTile * REC];
  __shared__ __align__(16) float4 blo[MIXED ? 2 : 1][MIXED ? kP2PTile : 1];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ TileMeta meta[2];
  __shared__ int s_warp[33];

  const T *prec = (const T *)prec_v;
  const int tid = threadIdx.x, BT = blockDim.x, TG = BT / G;
  const int tl = tid / G, g = tid % G;
  const int c = leaf_ids ? leaf_ids[blockIdx.x] : leaf0 + blockIdx.x;
  const int tlo = lohi[2 * c], thi = lohi[2 * c + 1], tcnt = thi - tlo + 1;
  const int p0 = ptr[c], np = ptr[c + 1] - p0;

  // number of staged tiles for this target leaf
  int w = 0;
  for (int k = tid; k < np; k += BT) {
    const int s = src[p0 + k];
    w += (lohi[2 * s + 1] - lohi[2 * s] + kP2PTile) / kP2PTile;
  }
  int W;
  block_excl_scan(w, s_warp, &W);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();

  // producer state (thread 0 only)
  int wk = 0, woff = 0;
  auto issue = [&](int bb) {
    const int s = src[p0 + wk];
    const int slo = lohi[2 * s], scnt = lohi[2 * s + 1] - slo + 1;
    const int cnt = scnt - woff < kP2PTile ? scnt - woff : kP2PTile;
    TileMeta m;
    m.cnt = cnt;
    if constexpr (MIXED) {
      const double *sb = bbox + 6 * (int64_t)s;
      m.scx = 0.5 * (sb[0] + sb[3]);
      m.scy = 0.5 * (sb[1] + sb[4]);
      m.scz = 0.5 * (sb[2] + sb[5]);
    } else {
      m.scx = m.scy = m.scz = 0.0;
    }
    meta[bb] = m;
    const uint32_t rec_bytes = (uint32_t)(cnt * REC * sizeof(T));
    mbar_arrive_expect_tx(&bar[bb], MIXED ? rec_bytes + (uint32_t)(cnt * sizeof(float4)) : rec_bytes);
    bulk_g2s(&buf[bb][0], prec + (int64_t)(slo + woff) * REC, rec_bytes, &bar[bb]);
    if constexpr (MIXED) bulk_g2s(&blo[bb][0], lo32 + (slo + woff), (uint32_t)(cnt * sizeof(float4)), &bar[bb]);
    woff += kP2PTile;
    if (woff >= scnt) {
      woff = 0;
      ++wk;
    }
  };

  int it = 0;  // global iteration count (mbarrier phase parity)
  for (int tc = 0; tc < tcnt; tc += kTT * TG) {
    int ti[kTT];
    bool active[kTT];
    T xi[kTT], yi[kTT], zi[kTT];
    double x64[kTT], y64[kTT], z64[kTT];
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      ti[u] = tc + tl + u * TG;
      active[u] = ti[u] < tcnt;
      const int pj = tlo + (active[u] ? ti[u] : 0);
      if constexpr (MIXED) {
        x64[u] = prec64[(int64_t)pj * 8 + 0];
        y64[u] = prec64[(int64_t)pj * 8 + 1];
        z64[u] = prec64[(int64_t)pj * 8 + 2];
        xi[u] = yi[u] = zi[u] = 0;
      } else {
        xi[u] = prec[(int64_t)pj * REC + 0];
        yi[u] = prec[(int64_t)pj * REC + 1];
        zi[u] = prec[(int64_t)pj * REC + 2];
        x64[u] = y64[u] = z64[u] = 0;
      }
    }
    const bool any = active[0];
    double a64[kTT][6];
    float ks[kTT][6], kc[kTT][6];
#pragma unroll
    for (int u = 0; u < kTT; ++u)
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        a64[u][q] = 0.0;
        ks[u][q] = kc[u][q] = 0.f;
      }
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
      if (ok && any) {
        const TileMeta m = meta[bb];
        T x0[kTT], y0[kTT], z0[kTT], xl[kTT], yl[kTT], zl[kTT];
#pragma unroll
        for (int u = 0; u < kTT; ++u) {
          if constexpr (MIXED) {  // the target in the source leaf's frame, as hi + lo
            const double X = x64[u] - m.scx, Y = y64[u] - m.scy, Z = z64[u] - m.scz;
            x0[u] = (float)X;
            y0[u] = (float)Y;
            z0[u] = (float)Z;
            xl[u] = (float)(X - (double)x0[u]);
            yl[u] = (float)(Y - (double)y0[u]);
            zl[u] = (float)(Z - (double)z0[u]);
          } else {
            x0[u] = xi[u];
            y0[u] = yi[u];
            z0[u] = zi[u];
            xl[u] = yl[u] = zl[u] = 0;
          }
        }
        T e[kTT][6];
#pragma unroll
        for (int u = 0; u < kTT; ++u)
#pragma unroll
          for (int q = 0; q < 6; ++q) e[u][q] = 0;
        const T *S = &buf[bb][0];
#pragma unroll 2
        for (int j = g; j < m.cnt; j += G) {
          const T *r = S + j * REC;
          const T sx = r[0], sy = r[1], sz = r[2], gam = r[3], ux = r[4], uy = r[5], uz = r[6];
          float4 l = make_float4(0.f, 0.f, 0.f, 0.f);
          if constexpr (MIXED) l = blo[bb][j];
#pragma unroll
          for (int u = 0; u < kTT; ++u) {
            T rx = x0[u] - sx, ry = y0[u] - sy, rz = z0[u] - sz;
            if constexpr (MIXED) {
              rx += xl[u] - l.x;
              ry += yl[u] - l.y;
              rz += zl[u] - l.z;
            }
            const T rre = rx * rx + (ry * ry + (rz * rz + (T)kEps64));
            const T pr = ux * rx + uy * ry + uz * rz;
            const T d = pr * pr + rre;
            T s;
            if constexpr (MIXED)
              s = rsqrt_approx_p(d);
            else
              s = rsqrt(d);
            const T s3 = s * s * s;
            const T gg = gam * s3;
            e[u][0] += gg * rx;
            e[u][1] += gg * ry;
            e[u][2] += gg * rz;
            const T hx = ux * s3, hy = uy * s3, hz = uz * s3;
            e[u][3] += hy * rz - hz * ry;
            e[u][4] += hz * rx - hx * rz;
            e[u][5] += hx * ry - hy * rx;
          }
        }
#pragma unroll
        for (int u = 0; u < kTT; ++u)
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            if constexpr (MIXED) {
              float y = e[u][q] - kc[u][q];
              float t = ks[u][q] + y;
              kc[u][q] = (t - ks[u][q]) - y;
              ks[u][q] = t;
            } else {
              a64[u][q] += e[u][q];
            }
          }
      }
      __syncthreads();  // buffer bb is refilled two iterations later
    }
    // combine the G lanes of each target group (warp shuffles), FP64 result
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      double v[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        if constexpr (MIXED)
          v[q] = (double)ks[u][q] - (double)kc[u][q];
        else
          v[q] = a64[u][q];
#pragma unroll
        for (int o = 1; o < G; o <<= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
      }
      if (active[u] && g == 0) {
        const int64_t pj = tlo + ti[u];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          double o = v[q];
          if (accumulate) o += near[(int64_t)q * N + pj];
          near[(int64_t)q * N + pj] = o;
        }
      }
    }
  }
}

template <int G, bool MIXED>
int launch_p2p_t(Ctx *ctx, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  if (nleaf <= 0) return FMMB200_OK;
  p2p_kernel<G, MIXED><<<(unsigned)nleaf, 128, 0, ctx->stream>>>(
      d_leaf_ids, (int)ctx->leaf0, ctx->get<int>("lohi"), ctx->get<int>("p2p_ptr"), ctx->get<int>("p2p_src"),
      ctx->get<double>("bbox"), MIXED ? (const void *)ctx->get<float>("prec32") : (const void *)ctx->get<double>("prec64"),
      MIXED ? ctx->get<float4>("prec32lo") : nullptr, ctx->get<double>("prec64"), ctx->get<double>("near"), (int)ctx->N,
      accumulate ? 1 : 0, ctx->d_status);
  return ctx->check_launch("p2p_kernel");
}

}  // namespace

// max_leaf: the largest target leaf (particles); selects lanes per target.
int launch_p2p(Ctx *ctx, bool mixed, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  // lanes per target group: 128 threads, two targets per lane group
  const int64_t max_leaf = ctx->max_leaf;
  if (max_leaf <= 32) return mixed ? launch_p2p_t<8, true>(ctx, d_leaf_ids, nleaf, accumulate)
                                   : launch_p2p_t<8, false>(ctx, d_leaf_ids, nleaf, accumulate);
  if (max_leaf <= 64) return mixed ? launch_p2p_t<4, true>(ctx, d_leaf_ids, nleaf, accumulate)
                                   : launch_p2p_t<4, false>(ctx, d_leaf_ids, nleaf, accumulate);
  if (max_leaf <= 128) return mixed ? launch_p2p_t<2, true>(ctx, d_leaf_ids, nleaf, accumulate)
                                    : launch_p2p_t<2, false>(ctx, d_leaf_ids, nleaf, accumulate);
  return mixed ? launch_p2p_t<1, true>(ctx, d_leaf_ids, nleaf, accumulate)
               : launch_p2p_t<1, false>(ctx, d_leaf_ids, nleaf, accumulate);
}

}  // namespace fmmb200
