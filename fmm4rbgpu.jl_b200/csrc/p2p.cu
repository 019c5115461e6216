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
// particle and split the sources; their partial fields are combined with warp
// shuffles.  G is chosen from the leaf size so that small leaves (64 particles
// at N0 = 125) still fill the CTA -- the reference launches N0 threads per
// leaf and leaves about half of them idle.
//
// Mixed form: FP32 leaf-local coordinates (the target's frame is shifted by the
// FP64 centre offset once per tile), FP32 arithmetic, per-tile partial sums
// folded into Kahan-compensated FP32 accumulators, FP64 output.
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
  float dcx, dcy, dcz;  // mixed: source-centre minus target-centre (target frame shift)
};

template <int G, bool MIXED>
__global__ void __launch_bounds__(128) p2p_kernel(const int *__restrict__ leaf_ids, int leaf0,
                                                  const int *__restrict__ lohi, const int *__restrict__ ptr,
                                                  const int *__restrict__ src, const double *__restrict__ bbox,
                                                  const void *__restrict__ prec_v, double *__restrict__ near,
                                                  int N, int accumulate, int *__restrict__ status) {
  using T = typename std::conditional<MIXED, float, double>::type;
  constexpr int REC = 8;  // T values per particle record
  __shared__ __align__(16) T buf[2][kP2PTile * REC];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ TileMeta meta[2];
  __shared__ int s_warp[33];
  __shared__ int s_work;

  const T *prec = (const T *)prec_v;
  const int tid = threadIdx.x, BT = blockDim.x, TP = BT / G;
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

  double tcx = 0, tcy = 0, tcz = 0;
  if constexpr (MIXED) {
    const double *bb = bbox + 6 * (int64_t)c;
    tcx = 0.5 * (bb[0] + bb[3]);
    tcy = 0.5 * (bb[1] + bb[4]);
    tcz = 0.5 * (bb[2] + bb[5]);
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    s_work = 0;
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
      m.dcx = (float)(0.5 * (sb[0] + sb[3]) - tcx);
      m.dcy = (float)(0.5 * (sb[1] + sb[4]) - tcy);
      m.dcz = (float)(0.5 * (sb[2] + sb[5]) - tcz);
    } else {
      m.dcx = m.dcy = m.dcz = 0.f;
    }
    meta[bb] = m;
    mbar_arrive_expect_tx(&bar[bb], (uint32_t)(cnt * REC * sizeof(T)));
    bulk_g2s(&buf[bb][0], prec + (int64_t)(slo + woff) * REC, (uint32_t)(cnt * REC * sizeof(T)), &bar[bb]);
    woff += kP2PTile;
    if (woff >= scnt) {
      woff = 0;
      ++wk;
    }
  };

  int it = 0;  // global iteration count (mbarrier phase parity)
  for (int tc = 0; tc < tcnt; tc += TP) {
    const int ti = tc + tl;
    const bool active = ti < tcnt;
    T xi = 0, yi = 0, zi = 0;
    if (active) {
      xi = prec[(int64_t)(tlo + ti) * REC + 0];
      yi = prec[(int64_t)(tlo + ti) * REC + 1];
      zi = prec[(int64_t)(tlo + ti) * REC + 2];
    }
    double a64[6] = {0, 0, 0, 0, 0, 0};
    float ks[6] = {0, 0, 0, 0, 0, 0}, kc[6] = {0, 0, 0, 0, 0, 0};
    if (tid == 0) {
      wk = 0;
      woff = 0;
      if (W > 0) issue(it & 1);
    }
    for (int i = 0; i < W; ++i, ++it) {
      const int bb = it & 1;
      if (tid == 0 && i + 1 < W) {
        fence_proxy_async_smem();
        issue(bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((it >> 1) & 1), status);
      if (ok && active) {
        const TileMeta m = meta[bb];
        T x0 = xi, y0 = yi, z0 = zi;
        if constexpr (MIXED) {
          x0 -= m.dcx;
          y0 -= m.dcy;
          z0 -= m.dcz;
        }
        T e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
        const T *S = &buf[bb][0];
#pragma unroll 4
        for (int j = g; j < m.cnt; j += G) {
          const T *r = S + j * REC;
          const T rx = x0 - r[0], ry = y0 - r[1], rz = z0 - r[2];
          const T gam = r[3], ux = r[4], uy = r[5], uz = r[6];
          const T rr = rx * rx + ry * ry + rz * rz;
          const T pr = ux * rx + uy * ry + uz * rz;
          const T d = pr * pr + rr + (T)kEps64;
          T s;
          if constexpr (MIXED)
            s = rsqrt_approx_p(d);
          else
            s = rsqrt(d);
          const T s3 = s * s * s;
          const T gg = gam * s3;
          e0 += gg * rx;
          e1 += gg * ry;
          e2 += gg * rz;
          const T hx = ux * s3, hy = uy * s3, hz = uz * s3;
          b0 += hy * rz - hz * ry;
          b1 += hz * rx - hx * rz;
          b2 += hx * ry - hy * rx;
        }
        if constexpr (MIXED) {
          const float v[6] = {e0, e1, e2, b0, b1, b2};
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            float y = v[q] - kc[q];
            float t = ks[q] + y;
            kc[q] = (t - ks[q]) - y;
            ks[q] = t;
          }
        } else {
          a64[0] += e0;
          a64[1] += e1;
          a64[2] += e2;
          a64[3] += b0;
          a64[4] += b1;
          a64[5] += b2;
        }
      }
      __syncthreads();  // buffer bb is refilled two iterations later
    }
    // combine the G lanes of each target (warp shuffles), FP64 result
    double v[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      if constexpr (MIXED)
        v[q] = (double)ks[q] - (double)kc[q];
      else
        v[q] = a64[q];
#pragma unroll
      for (int o = 1; o < G; o <<= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    if (active && g == 0) {
      const int64_t pj = tlo + ti;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        double o = v[q];
        if (accumulate) o += near[(int64_t)q * N + pj];
        near[(int64_t)q * N + pj] = o;
      }
    }
  }
  (void)s_work;
}

template <int G, bool MIXED>
int launch_p2p_t(Ctx *ctx, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  if (nleaf <= 0) return FMMB200_OK;
  p2p_kernel<G, MIXED><<<(unsigned)nleaf, 128, 0, ctx->stream>>>(
      d_leaf_ids, (int)ctx->leaf0, ctx->get<int>("lohi"), ctx->get<int>("p2p_ptr"), ctx->get<int>("p2p_src"),
      ctx->get<double>("bbox"), MIXED ? (const void *)ctx->get<float>("prec32") : (const void *)ctx->get<double>("prec64"),
      ctx->get<double>("near"), (int)ctx->N, accumulate ? 1 : 0, ctx->d_status);
  return ctx->check_launch("p2p_kernel");
}

}  // namespace

// max_leaf: the largest target leaf (particles); selects lanes per target.
int launch_p2p(Ctx *ctx, bool mixed, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  const int64_t max_leaf = ctx->max_leaf;
  if (max_leaf <= 32) return mixed ? launch_p2p_t<4, true>(ctx, d_leaf_ids, nleaf, accumulate)
                                   : launch_p2p_t<4, false>(ctx, d_leaf_ids, nleaf, accumulate);
  if (max_leaf <= 64) return mixed ? launch_p2p_t<2, true>(ctx, d_leaf_ids, nleaf, accumulate)
                                   : launch_p2p_t<2, false>(ctx, d_leaf_ids, nleaf, accumulate);
  return mixed ? launch_p2p_t<1, true>(ctx, d_leaf_ids, nleaf, accumulate)
               : launch_p2p_t<1, false>(ctx, d_leaf_ids, nleaf, accumulate);
}

}  // namespace fmmb200
