// p2p.cu -- P2P near field (the reference's gpu_P2P!,
// src/gpu_fmm/gpu_interaction.jl:43-86, and P2P!, src/fmm/interaction.jl:49-75):
//   E_i += sum_j gamma_j K(x_i - x_j; u_j),  B_i += sum_j u_j x K(x_i - x_j; u_j)
// over the particles j of every source leaf in target leaf i's P2P list (j = i
// gives R = 0 and K = 0, as in the reference).
//
// Design: one CTA per target leaf.  Particles are stored in tree order, so every
// source leaf is one contiguous range of records: tiles of up to 128 source
// records are bulk-copied (TMA) into a double buffer guarded by mbarriers.  G
// source lanes share the targets (both use every staged source record) and split
// the sources.  A lane is TG = 128 / G threads, whole warps for G <= 4, so every
// record load is a shared-memory broadcast; the lanes' FP64 sums are combined
// through shared memory, pairwise in lane order.  G is chosen from the leaf size
// so that small leaves (64 particles at N0 = 125) still fill the CTA -- the
// reference launches N0 threads per leaf and leaves about half of them idle.
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

// Sum of G values v[0], v[stride], ..., pairwise in index order: ((v0 + v1) + (v2 + v3)) + ...
template <int G>
__device__ __forceinline__ double lane_tree_sum(const double *v, int stride) {
  if constexpr (G == 1)
    return v[0];
  else
    return lane_tree_sum<G / 2>(v, stride) + lane_tree_sum<G / 2>(v + (G / 2) * stride, stride);
}

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
  __shared__ double s_red[kTT * 6][128];  // per thread: E, B of its targets, for the lane sum

  const int tid = threadIdx.x, BT = blockDim.x, TG = BT / G;
  // source lane g = tid / TG: a warp's threads share one lane (TG >= 32), so every staged
  // record load is a broadcast
  const int tl = tid % TG, g = tid / TG;
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
    // combine the G lanes of each target group through shared memory, pairwise in lane
    // order (the order of an xor butterfly over adjacent lanes)
#pragma unroll
    for (int u = 0; u < kTT; ++u)
#pragma unroll
      for (int q = 0; q < 6; ++q) s_red[u * 6 + q][tid] = acc[u][q];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      if (active[u] && g == 0) {
        const int64_t pj = tlo + ti[u];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          double o = lane_tree_sum<G>(&s_red[u * 6 + q][tl], TG);
          if (accumulate) o += near[(int64_t)q * N + pj];
          near[(int64_t)q * N + pj] = o;
        }
      }
    }
    __syncthreads();  // s_red is rewritten by the next round
  }
}

// The evaluation body of the mixed kernels, shared with the probe of its attainable rate.
// A pair of targets (the two lanes of FP32x2) in a source leaf's frame, as hi + lo parts.
struct P2PTargets {
  float2 xh, yh, zh, xl, yl, zl;
};
// FP32 partial sums of a target pair: E, and B = bp - bm.
struct P2PAcc {
  float2 e0, e1, e2, bp0, bp1, bp2, bm0, bm1, bm2;
};
// One staged source record: -hi, -lo coordinates (lo only for NEAR), gamma, u.
struct P2PSource {
  float2 xh, yh, zh, xl, yl, zl, gam, ux, uy, uz;
};

template <bool NEAR>
__device__ __forceinline__ P2PSource p2p_x2_load(const float4 *__restrict__ r) {
  const float4 r0 = r[0], r1 = r[1], r3 = r[3], r4 = r[4];
  const float4 r2 = NEAR ? r[2] : make_float4(0.f, 0.f, 0.f, 0.f);
  return P2PSource{lo2(r0), hi2(r0), lo2(r1), hi2(r1), lo2(r2), hi2(r2), lo2(r3), hi2(r3), lo2(r4), hi2(r4)};
}

// E += gamma K, B += u x K with K = s^3 R, s = (R.R + (u.R)^2 + eps)^(-1/2), for one source and
// one target pair.  R = (target hi - source hi) + (target lo - source lo) when NEAR, else from
// the hi parts alone; the record holds -hi, -lo.
template <bool NEAR>
__device__ __forceinline__ void p2p_x2_eval(const P2PSource &q, const P2PTargets &t, float2 eps, P2PAcc &a) {
  float2 rx, ry, rz;
  if constexpr (NEAR) {
    rx = add2(add2(t.xh, q.xh), add2(t.xl, q.xl));
    ry = add2(add2(t.yh, q.yh), add2(t.yl, q.yl));
    rz = add2(add2(t.zh, q.zh), add2(t.zl, q.zl));
  } else {
    rx = add2(t.xh, q.xh);
    ry = add2(t.yh, q.yh);
    rz = add2(t.zh, q.zh);
  }
  const float2 rre = fma2(rx, rx, fma2(ry, ry, fma2(rz, rz, eps)));
  const float2 pr = fma2(q.uz, rz, fma2(q.uy, ry, mul2(q.ux, rx)));
  const float2 d = fma2(pr, pr, rre);
  const float2 sv = rsqrt2(d);
  const float2 s3 = mul2(mul2(sv, sv), sv);
  const float2 kx = mul2(s3, rx), ky = mul2(s3, ry), kz = mul2(s3, rz);  // K = s^3 R
  a.e0 = fma2(q.gam, kx, a.e0);
  a.e1 = fma2(q.gam, ky, a.e1);
  a.e2 = fma2(q.gam, kz, a.e2);
  a.bp0 = fma2(q.uy, kz, a.bp0);  // B = u x K as (bp - bm)
  a.bm0 = fma2(q.uz, ky, a.bm0);
  a.bp1 = fma2(q.uz, kx, a.bp1);
  a.bm1 = fma2(q.ux, kz, a.bm1);
  a.bp2 = fma2(q.ux, ky, a.bp2);
  a.bm2 = fma2(q.uy, kx, a.bm2);
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
  // source lane g = tid / TG: the TG threads of a lane, whole warps when TG >= 32, read
  // the same staged source record at once (one shared-memory broadcast per load)
  const int tl = tid % TG, g = tid / TG;
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
    P2PAcc acc[TP];
#pragma unroll
    for (int t = 0; t < TP; ++t) acc[t] = P2PAcc{z, z, z, z, z, z, z, z, z};
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
        P2PTargets tg[TP];
#pragma unroll
        for (int t = 0; t < TP; ++t) {
          const double dx0 = tX[2 * t] - scx, dy0 = tY[2 * t] - scy, dz0 = tZ[2 * t] - scz;
          const double dx1 = tX[2 * t + 1] - scx, dy1 = tY[2 * t + 1] - scy, dz1 = tZ[2 * t + 1] - scz;
          P2PTargets &o = tg[t];
          o.xh = make_float2((float)dx0, (float)dx1);
          o.yh = make_float2((float)dy0, (float)dy1);
          o.zh = make_float2((float)dz0, (float)dz1);
          o.xl = make_float2((float)(dx0 - (double)o.xh.x), (float)(dx1 - (double)o.xh.y));
          o.yl = make_float2((float)(dy0 - (double)o.yh.x), (float)(dy1 - (double)o.yh.y));
          o.zl = make_float2((float)(dz0 - (double)o.zh.x), (float)(dz1 - (double)o.zh.y));
        }
        const float2 eps = dup2((float)kEps64);
        const float4 *S = &buf[bb][0];
        auto sweep = [&](auto NEARC) {
          constexpr bool NEAR = decltype(NEARC)::value;
#pragma unroll 2
          for (int j = g; j < cnt; j += G) {
            const P2PSource q = p2p_x2_load<NEAR>(S + j * REC);
#pragma unroll
            for (int t = 0; t < TP; ++t) p2p_x2_eval<NEAR>(q, tg[t], eps, acc[t]);
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
          const P2PAcc &a = acc[t];
          const float2 part[6] = {a.e0, a.e1, a.e2, sub2(a.bp0, a.bm0), sub2(a.bp1, a.bm1), sub2(a.bp2, a.bm2)};
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            s_acc[12 * t + q][tid] += (double)part[q].x;
            s_acc[12 * t + 6 + q][tid] += (double)part[q].y;
          }
          acc[t] = P2PAcc{z, z, z, z, z, z, z, z, z};
        }
      }
      __syncthreads();  // buffer bb is refilled two iterations later
    }
    // combine the G lanes of each target group, FP64 result: pairwise in lane order, the
    // order of an xor butterfly over adjacent lanes
    __syncthreads();  // every lane's sums are in s_acc
#pragma unroll
    for (int t = 0; t < TP; ++t) {
      double v0[6], v1[6];
      if (g == 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          v0[q] = lane_tree_sum<G>(&s_acc[12 * t + q][tl], TG);
          v1[q] = lane_tree_sum<G>(&s_acc[12 * t + 6 + q][tl], TG);
        }
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
    __syncthreads();  // s_acc is reset by the next round
  }
}

// The attainable rate of the mixed evaluation body on this GPU: the kernel's own load and
// evaluation code (p2p_x2_load / p2p_x2_eval) over 64 synthetic source records held in
// shared memory, G = 4 source lanes (one per warp) as for leaves of 64, looped without staging,
// barriers or folds.  out: one value per thread, so that nothing is dead code.
template <bool NEAR>
__global__ void __launch_bounds__(128) p2p_body_probe_kernel(int reps, float *__restrict__ out) {
  constexpr int NS = 64, G = 4;
  __shared__ __align__(16) float4 S[NS * 5];
  for (int j = threadIdx.x; j < NS; j += blockDim.x) {
    const float x = 0.3f * __cosf((float)j), y = 0.3f * __sinf((float)j), zz = 0.01f * (float)j / NS;
    const float xl = 1e-9f * (float)(j % 3), yl = -1e-9f * (float)(j % 5), zl = 2e-9f;
    S[5 * j + 0] = make_float4(-x, -x, -y, -y);
    S[5 * j + 1] = make_float4(-zz, -zz, -xl, -xl);
    S[5 * j + 2] = make_float4(-yl, -yl, -zl, -zl);
    S[5 * j + 3] = make_float4(200.f, 200.f, 0.01f, 0.01f);
    S[5 * j + 4] = make_float4(-0.02f, -0.02f, 199.9f, 199.9f);
  }
  __syncthreads();
  const int g = threadIdx.x / (blockDim.x / G), w = threadIdx.x % (blockDim.x / G);  // the kernel's lanes
  const P2PTargets t{make_float2(0.5f + 0.001f * w, 0.52f + 0.001f * w), make_float2(-0.2f, -0.21f),
                     make_float2(0.05f, 0.04f), make_float2(1e-9f, -1e-9f), make_float2(0.f, 1e-9f),
                     make_float2(-2e-9f, 0.f)};
  const float2 z = make_float2(0.f, 0.f), eps = dup2((float)kEps64);
  P2PAcc a{z, z, z, z, z, z, z, z, z};
  for (int r = 0; r < reps; ++r) {
#pragma unroll 2
    for (int j = g; j < NS; j += G) p2p_x2_eval<NEAR>(p2p_x2_load<NEAR>(S + 5 * j), t, eps, a);
  }
  const float2 v = add2(add2(add2(a.e0, a.e1), add2(a.e2, a.bp0)),
                        add2(add2(a.bp1, a.bp2), add2(add2(a.bm0, a.bm1), a.bm2)));
  out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = v.x + v.y;
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

using namespace fmmb200;

extern "C" {

int fmmb200_measure_p2p_body(fmmb200_ctx *ctx, double *far_evals_per_s, double *near_evals_per_s) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  // six CTAs of 128 threads per SM: the residency of p2p_x2_kernel<4, 1> (80 registers)
  const int threads = 128, blocks = nsm * 6, reps = 256;
  float *out;
  FMM_TRY(ctx->ensure("p2p_probe_out", (int64_t)threads * blocks, &out));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  // evaluations per launch: every thread holds a target pair and sees 64 / 4 sources per rep
  const double evals = 2.0 * (64 / 4) * (double)reps * threads * blocks;
  double best[2] = {0.0, 0.0};
  for (int rep = 0; rep < 4; ++rep) {
    for (int k = 0; k < 2; ++k) {
      cudaEventRecord(a, ctx->stream);
      if (k == 0)
        p2p_body_probe_kernel<false><<<blocks, threads, 0, ctx->stream>>>(reps, out);
      else
        p2p_body_probe_kernel<true><<<blocks, threads, 0, ctx->stream>>>(reps, out);
      cudaEventRecord(b, ctx->stream);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0 && ms > 0.f && evals / (ms * 1e-3) > best[k]) best[k] = evals / (ms * 1e-3);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  FMM_TRY(ctx->check_launch("p2p_body_probe_kernel", 8));
  if (far_evals_per_s) *far_evals_per_s = best[0];
  if (near_evals_per_s) *near_evals_per_s = best[1];
  return FMMB200_OK;
}

}  // extern "C"
