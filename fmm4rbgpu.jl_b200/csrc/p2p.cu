// p2p.cu -- P2P near field (the reference's gpu_P2P!,
// src/gpu_fmm/gpu_interaction.jl:43-86, and P2P!, src/fmm/interaction.jl:49-75):
//   E_i += sum_j gamma_j K(x_i - x_j; u_j),  B_i += sum_j u_j x K(x_i - x_j; u_j)
// over the particles j of every source leaf in target leaf i's P2P list (j = i
// gives R = 0 and K = 0, as in the reference).
//
// Design: one CTA per target leaf.  Particles are stored in tree order, so every
// source leaf is one contiguous range of records: tiles of up to 128 source
// records are bulk-copied (TMA) into a double buffer guarded by mbarriers.  G
// adjacent lanes share two target particles (both use every staged source
// record) and split the sources; their partial fields are combined with warp
// shuffles.  G is chosen from the leaf size so that small leaves (64 particles
// at N0 = 125) still fill the CTA -- the reference launches N0 threads per
// leaf and leaves about half of them idle.
//
// FP64 form (p2p_kernel): 64-byte records, double arithmetic.
// Mixed form (p2p_x2_kernel): each pair of targets of a lane group is evaluated in
// the two lanes of packed FP32x2 instructions on coordinates relative to the
// source leaf's box centre, each stored as a hi + lo pair of floats.  Per tile
// the targets are moved into the source's frame in FP64 once and split the same
// way; every pair difference R = (X_hi - x_hi) + (X_lo - x_lo) is then formed to
// ~1 ulp of |R| even for very close pairs (the hi difference is exact,
// Sterbenz), which a plain FP32 leaf-local coordinate cannot give.  Source
// records (80 bytes) hold every value duplicated, so that a 128-bit shared load
// yields two packed operands.  Per-tile FP32 partial sums are added into per-thread
// FP64 sums in shared memory; the output is FP64.
#include <type_traits>

#include "device_util.cuh"
#include "kernels.cuh"
#include "packed.cuh"

namespace fmmb200 {

namespace {

constexpr int kP2PTile = 128;

// Two target particles per lane group share every staged source record.
constexpr int kTT = 2;
// Staged source tiles whose FP32 partial sums the mixed kernel adds up before folding
// them into its FP64 sums (every tile: 61.6 ms at N = 2^24; every 8th: 57.0 ms, error
// vs FP64 2.12e-7 -> 2.23e-7).
constexpr int kP2PFold = 8;


// Number of staged tiles of target leaf c's source list (block-wide).
__device__ __forceinline__ int count_tiles(const int *__restrict__ lohi, const int *__restrict__ src, int p0, int np,
                                           int *s_warp) {
  int w = 0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    const int s = src[p0 + k];
    w += (lohi[2 * s + 1] - lohi[2 * s] + kP2PTile) / kP2PTile;
  }
  int W;
  block_excl_scan(w, s_warp, &W);
  return W;
}

// Producer position in the tile sequence (thread 0 only): source wk, offset woff.
struct TileCursor {
  int wk, woff;
  // Next tile: source leaf s, its first record slo + woff, cnt records; advances.
  __device__ __forceinline__ void next(const int *__restrict__ lohi, const int *__restrict__ src, int p0, int *s,
                                       int *first, int *cnt) {
    *s = src[p0 + wk];
    const int slo = lohi[2 * *s], scnt = lohi[2 * *s + 1] - slo + 1;
    *cnt = scnt - woff < kP2PTile ? scnt - woff : kP2PTile;
    *first = slo + woff;
    woff += kP2PTile;
    if (woff >= scnt) {
      woff = 0;
      ++wk;
    }
  }
};

template <int G>
__global__ void __launch_bounds__(128) p2p_kernel(const int *__restrict__ leaf_ids, int leaf0,
                                                  const int *__restrict__ lohi, const int *__restrict__ ptr,
                                                  const int *__restrict__ src, const double *__restrict__ prec,
                                                  double *__restrict__ near, int N, int accumulate,
                                                  int *__restrict__ status) {
  constexpr int REC = 8;  // doubles per particle record
  __shared__ __align__(16) double buf[2][kP2PTile * REC];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_cnt[2];
  __shared__ int s_warp[33];

  const int tid = threadIdx.x, BT = blockDim.x, TG = BT / G;
  const int tl = tid / G, g = tid % G;
  const int c = leaf_ids ? leaf_ids[blockIdx.x] : leaf0 + blockIdx.x;
  const int tlo = lohi[2 * c], thi = lohi[2 * c + 1], tcnt = thi - tlo + 1;
  const int p0 = ptr[c], np = ptr[c + 1] - p0;
  const int W = count_tiles(lohi, src, p0, np, s_warp);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();

  TileCursor cur{0, 0};
  auto issue = [&](int bb) {
    int s, first, cnt;
    cur.next(lohi, src, p0, &s, &first, &cnt);
    s_cnt[bb] = cnt;
    const uint32_t bytes = (uint32_t)(cnt * REC * sizeof(double));
    mbar_arrive_expect_tx(&bar[bb], bytes);
    bulk_g2s(&buf[bb][0], prec + (int64_t)first * REC, bytes, &bar[bb]);
  };

  int it = 0;  // global iteration count (mbarrier phase parity)
  for (int tc = 0; tc < tcnt; tc += kTT * TG) {
    int ti[kTT];
    bool active[kTT];
    double xi[kTT], yi[kTT], zi[kTT];
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      ti[u] = tc + tl + u * TG;
      active[u] = ti[u] < tcnt;
      const int pj = tlo + (active[u] ? ti[u] : 0);
      xi[u] = prec[(int64_t)pj * REC + 0];
      yi[u] = prec[(int64_t)pj * REC + 1];
      zi[u] = prec[(int64_t)pj * REC + 2];
    }
    const bool any = active[0];
    double acc[kTT][6];
#pragma unroll
    for (int u = 0; u < kTT; ++u)
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[u][q] = 0.0;
    if (tid == 0) {
      cur = TileCursor{0, 0};
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
        const int cnt = s_cnt[bb];
        const double *S = &buf[bb][0];
#pragma unroll 2
        for (int j = g; j < cnt; j += G) {
          const double *r = S + j * REC;
          const double sx = r[0], sy = r[1], sz = r[2], gam = r[3], ux = r[4], uy = r[5], uz = r[6];
#pragma unroll
          for (int u = 0; u < kTT; ++u) {
            const double rx = xi[u] - sx, ry = yi[u] - sy, rz = zi[u] - sz;
            const double rre = rx * rx + (ry * ry + (rz * rz + kEps64));
            const double pr = ux * rx + uy * ry + uz * rz;
            const double d = pr * pr + rre;
            const double s = rsqrt(d);
            const double s3 = s * s * s;
            const double gg = gam * s3;
            acc[u][0] += gg * rx;
            acc[u][1] += gg * ry;
            acc[u][2] += gg * rz;
            const double hx = ux * s3, hy = uy * s3, hz = uz * s3;
            acc[u][3] += hy * rz - hz * ry;
            acc[u][4] += hz * rx - hx * rz;
            acc[u][5] += hx * ry - hy * rx;
          }
        }
      }
      __syncthreads();  // buffer bb is refilled two iterations later
    }
    // combine the G lanes of each target group (warp shuffles)
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      double v[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        v[q] = acc[u][q];
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

template <int G, int TP>
__global__ void __launch_bounds__(128) p2p_x2_kernel(const int *__restrict__ leaf_ids, int leaf0,
                                                     const int *__restrict__ lohi, const int *__restrict__ ptr,
                                                     const int *__restrict__ src, const double *__restrict__ bbox,
                                                     const float4 *__restrict__ rec_x2,
                                                     const double *__restrict__ prec64, double *__restrict__ near,
                                                     int N, int accumulate, int *__restrict__ status) {
  constexpr int REC = 5;  // float4 per source record
  __shared__ __align__(16) float4 buf[2][kP2PTile * REC];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_cnt[2], s_near[2];
  __shared__ double s_centre[2][3];
  __shared__ int s_warp[33];
  __shared__ double s_acc[12 * TP][128];  // per thread: E, B of its 2 TP targets, FP64 sums over tiles

  const int tid = threadIdx.x, BT = blockDim.x, TG = BT / G;
  const int tl = tid / G, g = tid % G;
  const int c = leaf_ids ? leaf_ids[blockIdx.x] : leaf0 + blockIdx.x;
  const double *tbox = bbox + 6 * (int64_t)c;
  const int tlo = lohi[2 * c], thi = lohi[2 * c + 1], tcnt = thi - tlo + 1;
  const int p0 = ptr[c], np = ptr[c + 1] - p0;
  const int W = count_tiles(lohi, src, p0, np, s_warp);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();

  TileCursor cur{0, 0};
  auto issue = [&](int bb) {
    int s, first, cnt;
    cur.next(lohi, src, p0, &s, &first, &cnt);
    s_cnt[bb] = cnt;
    const double *sb = bbox + 6 * (int64_t)s;
    s_centre[bb][0] = 0.5 * (sb[0] + sb[3]);
    s_centre[bb][1] = 0.5 * (sb[1] + sb[4]);
    s_centre[bb][2] = 0.5 * (sb[2] + sb[5]);
    // boxes apart by more than 1/kHiOnlyGap of the larger extent: R from the hi parts alone
    s_near[bb] = p2p_tile_needs_lo(sb, tbox);
    const uint32_t bytes = (uint32_t)(cnt * REC * sizeof(float4));
    mbar_arrive_expect_tx(&bar[bb], bytes);
    bulk_g2s(&buf[bb][0], rec_x2 + (int64_t)first * REC, bytes, &bar[bb]);
  };

  int it = 0;  // global iteration count (mbarrier phase parity)
  // a lane group holds 2 TP targets: pair t = (ti[2t], ti[2t+1]) in the lanes of FP32x2
  for (int tc = 0; tc < tcnt; tc += 2 * TP * TG) {
    int ti[2 * TP];
    bool act[2 * TP];
    int64_t pj[2 * TP];
    double tX[2 * TP], tY[2 * TP], tZ[2 * TP];  // FP64 target coordinates
#pragma unroll
    for (int u = 0; u < 2 * TP; ++u) {
      ti[u] = tc + tl + u * TG;
      act[u] = ti[u] < tcnt;
      pj[u] = tlo + (act[u] ? ti[u] : 0);
      tX[u] = prec64[pj[u] * 8 + 0];
      tY[u] = prec64[pj[u] * 8 + 1];
      tZ[u] = prec64[pj[u] * 8 + 2];
    }
#pragma unroll
    for (int q = 0; q < 12 * TP; ++q) s_acc[q][tid] = 0.0;
    if (tid == 0) {
      cur = TileCursor{0, 0};
      if (W > 0) {
        fence_proxy_async_smem();
        issue(it & 1);
      }
    }
    // FP32 partial sums over kP2PFold tiles, then added into the FP64 sums
    const float2 z = make_float2(0.f, 0.f);
    float2 e0[TP], e1[TP], e2[TP], bp0[TP], bp1[TP], bp2[TP], bm0[TP], bm1[TP], bm2[TP];
#pragma unroll
    for (int t = 0; t < TP; ++t) e0[t] = e1[t] = e2[t] = bp0[t] = bp1[t] = bp2[t] = bm0[t] = bm1[t] = bm2[t] = z;
    for (int i = 0; i < W; ++i, ++it) {
      const int bb = it & 1;
      if (tid == 0 && i + 1 < W) {
        fence_proxy_async_smem();
        issue(bb ^ 1);
      }
      const bool ok = mbar_wait_bounded(&bar[bb], (uint32_t)((it >> 1) & 1), status);
      if (ok && act[0]) {
        const int cnt = s_cnt[bb];
        // the targets in the source leaf's frame, as hi + lo
        const double scx = s_centre[bb][0], scy = s_centre[bb][1], scz = s_centre[bb][2];
        float2 xh[TP], yh[TP], zh[TP], xl[TP], yl[TP], zl[TP];
#pragma unroll
        for (int t = 0; t < TP; ++t) {
          const double dx0 = tX[2 * t] - scx, dy0 = tY[2 * t] - scy, dz0 = tZ[2 * t] - scz;
          const double dx1 = tX[2 * t + 1] - scx, dy1 = tY[2 * t + 1] - scy, dz1 = tZ[2 * t + 1] - scz;
          xh[t] = make_float2((float)dx0, (float)dx1);
          yh[t] = make_float2((float)dy0, (float)dy1);
          zh[t] = make_float2((float)dz0, (float)dz1);
          xl[t] = make_float2((float)(dx0 - (double)xh[t].x), (float)(dx1 - (double)xh[t].y));
          yl[t] = make_float2((float)(dy0 - (double)yh[t].x), (float)(dy1 - (double)yh[t].y));
          zl[t] = make_float2((float)(dz0 - (double)zh[t].x), (float)(dz1 - (double)zh[t].y));
        }
        const float2 eps = dup2((float)kEps64);
        const float4 *S = &buf[bb][0];
        auto sweep = [&](auto NEARC) {
          constexpr bool NEAR = decltype(NEARC)::value;
#pragma unroll 2
          for (int j = g; j < cnt; j += G) {
            const float4 *r = S + j * REC;
            const float4 r0 = r[0], r1 = r[1], r3 = r[3], r4 = r[4];
            const float4 r2 = NEAR ? r[2] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float2 gam = lo2(r3), ux = hi2(r3), uy = lo2(r4), uz = hi2(r4);
#pragma unroll
            for (int t = 0; t < TP; ++t) {
              // R = (target hi - source hi) + (target lo - source lo); the record holds -hi, -lo
              float2 rx, ry, rz;
              if constexpr (NEAR) {
                rx = add2(add2(xh[t], lo2(r0)), add2(xl[t], hi2(r1)));
                ry = add2(add2(yh[t], hi2(r0)), add2(yl[t], lo2(r2)));
                rz = add2(add2(zh[t], lo2(r1)), add2(zl[t], hi2(r2)));
              } else {
                rx = add2(xh[t], lo2(r0));
                ry = add2(yh[t], hi2(r0));
                rz = add2(zh[t], lo2(r1));
              }
              const float2 rre = fma2(rx, rx, fma2(ry, ry, fma2(rz, rz, eps)));
              const float2 pr = fma2(uz, rz, fma2(uy, ry, mul2(ux, rx)));
              const float2 d = fma2(pr, pr, rre);
              const float2 s = rsqrt2(d);
              const float2 s3 = mul2(mul2(s, s), s);
              const float2 kx = mul2(s3, rx), ky = mul2(s3, ry), kz = mul2(s3, rz);  // K = s^3 R
              e0[t] = fma2(gam, kx, e0[t]);
              e1[t] = fma2(gam, ky, e1[t]);
              e2[t] = fma2(gam, kz, e2[t]);
              bp0[t] = fma2(uy, kz, bp0[t]);  // B = u x K as (bp - bm)
              bm0[t] = fma2(uz, ky, bm0[t]);
              bp1[t] = fma2(uz, kx, bp1[t]);
              bm1[t] = fma2(ux, kz, bm1[t]);
              bp2[t] = fma2(ux, ky, bp2[t]);
              bm2[t] = fma2(uy, kx, bm2[t]);
            }
          }
        };
        if (s_near[bb])
          sweep(std::integral_constant<bool, true>{});
        else
          sweep(std::integral_constant<bool, false>{});
      }
      if ((i + 1) % kP2PFold == 0 || i + 1 == W) {
#pragma unroll
        for (int t = 0; t < TP; ++t) {
          const float2 part[6] = {e0[t], e1[t], e2[t], sub2(bp0[t], bm0[t]), sub2(bp1[t], bm1[t]),
                                  sub2(bp2[t], bm2[t])};
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            s_acc[12 * t + q][tid] += (double)part[q].x;
            s_acc[12 * t + 6 + q][tid] += (double)part[q].y;
          }
          e0[t] = e1[t] = e2[t] = bp0[t] = bp1[t] = bp2[t] = bm0[t] = bm1[t] = bm2[t] = z;
        }
      }
      __syncthreads();  // buffer bb is refilled two iterations later
    }
    // combine the G lanes of each target group (warp shuffles), FP64 result
#pragma unroll
    for (int t = 0; t < TP; ++t) {
      double v0[6], v1[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        v0[q] = s_acc[12 * t + q][tid];
        v1[q] = s_acc[12 * t + 6 + q][tid];
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
          v0[q] += __shfl_xor_sync(0xffffffffu, v0[q], o);
          v1[q] += __shfl_xor_sync(0xffffffffu, v1[q], o);
        }
      }
      if (g == 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          if (act[2 * t]) {
            double o = v0[q];
            if (accumulate) o += near[(int64_t)q * N + pj[2 * t]];
            near[(int64_t)q * N + pj[2 * t]] = o;
          }
          if (act[2 * t + 1]) {
            double o = v1[q];
            if (accumulate) o += near[(int64_t)q * N + pj[2 * t + 1]];
            near[(int64_t)q * N + pj[2 * t + 1]] = o;
          }
        }
      }
    }
  }
}

template <int G>
int launch_p2p_fp64(Ctx *ctx, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  if (nleaf <= 0) return FMMB200_OK;
  p2p_kernel<G><<<(unsigned)nleaf, 128, 0, ctx->stream>>>(d_leaf_ids, (int)ctx->leaf0, ctx->get<int>("lohi"),
                                                         ctx->get<int>("p2p_ptr"), ctx->get<int>("p2p_src"),
                                                         ctx->get<double>("prec64"), ctx->get<double>("near"),
                                                         (int)ctx->N, accumulate ? 1 : 0, ctx->d_status);
  return ctx->check_launch("p2p_kernel");
}

// Leaves above 64 particles (G <= 2): two target pairs per lane group over 2 G lanes, which
// halves the shared loads per evaluation (beamlets, N0 = 200, leaves of 128: 44.1 -> 37.4 ms
// at 2^22); for smaller leaves one pair per group keeps the register count at 80 and is faster
// (Gaussian bunch, leaves of 64: 16.9 vs 18.0 ms).
template <int G>
int launch_p2p_mixed(Ctx *ctx, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  if (nleaf <= 0) return FMMB200_OK;
  constexpr int TP = G <= 2 ? 2 : 1;
  constexpr int GG = G * TP;
  p2p_x2_kernel<GG, TP><<<(unsigned)nleaf, 128, 0, ctx->stream>>>(
      d_leaf_ids, (int)ctx->leaf0, ctx->get<int>("lohi"), ctx->get<int>("p2p_ptr"), ctx->get<int>("p2p_src"),
      ctx->get<double>("bbox"), ctx->get<float4>("prec32x2"), ctx->get<double>("prec64"), ctx->get<double>("near"),
      (int)ctx->N, accumulate ? 1 : 0, ctx->d_status);
  return ctx->check_launch("p2p_x2_kernel");
}

template <int G>
int launch_p2p_g(Ctx *ctx, bool mixed, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  return mixed ? launch_p2p_mixed<G>(ctx, d_leaf_ids, nleaf, accumulate)
               : launch_p2p_fp64<G>(ctx, d_leaf_ids, nleaf, accumulate);
}

}  // namespace

// Lanes per target group from the largest target leaf (ctx->max_leaf): 128
// threads, two targets per lane group.
int launch_p2p(Ctx *ctx, bool mixed, const int *d_leaf_ids, int64_t nleaf, bool accumulate) {
  const int64_t max_leaf = ctx->max_leaf;
  if (max_leaf <= 32) return launch_p2p_g<8>(ctx, mixed, d_leaf_ids, nleaf, accumulate);
  if (max_leaf <= 64) return launch_p2p_g<4>(ctx, mixed, d_leaf_ids, nleaf, accumulate);
  if (max_leaf <= 128) return launch_p2p_g<2>(ctx, mixed, d_leaf_ids, nleaf, accumulate);
  return launch_p2p_g<1>(ctx, mixed, d_leaf_ids, nleaf, accumulate);
}

}  // namespace fmmb200
