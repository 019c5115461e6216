// direct.cu -- FP64 direct summation on the GPU (the reference's BruteForce,
// src/update_particles_field.jl:21-38, which is serial host code there) and an
// FMA-throughput microbenchmark that measures the CUDA-core FP64/FP32 peaks
// used as roofline denominators for the M2L and P2P kernels.
//
// Direct sum: targets are split over CTAs of 128 threads (one target each) and
// the sources over `splits` slices; each CTA streams its slice through shared
// memory tiles and writes one partial per target, and a second kernel adds the
// partials in slice order, so the result is deterministic.
#include <mutex>
#include <vector>

#include "device_util.cuh"
#include "kernels.cuh"

using namespace fmmb200;

namespace {

// Scratch of fmmb200_direct_noalloc: 6 partial sums per (target, source slice)
// slot, for at most kNoAllocSlots slots (3 MiB).  Every GPU that loads the
// library holds this array until the process exits.
constexpr int64_t kNoAllocSlots = 65536;
__device__ __align__(256) double g_noalloc_scratch[6 * kNoAllocSlots];

// Device address of g_noalloc_scratch per device (the host-side symbol is a
// stand-in, not a device address), filled once per device.
constexpr int kMaxDevices = 64;
double *g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

constexpr int kDirThreads = 128;
constexpr int kDirTile = 256;

// A target index outside [0, N) is never dereferenced: that target's partials are
// NaN, and `status` (when given) is raised to kDevBadIndex.
__global__ void __launch_bounds__(kDirThreads)
    direct_partial_kernel(int64_t N, const double *__restrict__ pos, const double *__restrict__ mom,
                          int64_t ntarget, const int64_t *__restrict__ targets, int splits,
                          double *__restrict__ part, int *__restrict__ status) {
  __shared__ double s[kDirTile][7];
  const int64_t q = (int64_t)blockIdx.x * kDirThreads + threadIdx.x;
  const int split = blockIdx.y;
  const int64_t per = (N + splits - 1) / splits;
  const int64_t j0 = split * per, j1 = j0 + per < N ? j0 + per : N;
  double xi = 0, yi = 0, zi = 0;
  bool bad = false;
  if (q < ntarget) {
    const int64_t i = targets ? targets[q] : q;
    bad = i < 0 || i >= N;
    if (bad) {
      if (status && split == 0) atomicCAS(status, kDevOk, kDevBadIndex);
    } else {
      xi = pos[3 * i];
      yi = pos[3 * i + 1];
      zi = pos[3 * i + 2];
    }
  }
  double e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
  for (int64_t t0 = j0; t0 < j1; t0 += kDirTile) {
    const int cnt = (int)(j1 - t0 < kDirTile ? j1 - t0 : kDirTile);
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += kDirThreads) {
      const int64_t j = t0 + k;
      const double ux = mom[3 * j], uy = mom[3 * j + 1], uz = mom[3 * j + 2];
      s[k][0] = pos[3 * j];
      s[k][1] = pos[3 * j + 1];
      s[k][2] = pos[3 * j + 2];
      s[k][3] = ux;
      s[k][4] = uy;
      s[k][5] = uz;
      s[k][6] = sqrt(1.0 + (ux * ux + uy * uy + uz * uz));
    }
    __syncthreads();
    if (q < ntarget) {
      for (int k = 0; k < cnt; ++k) {
        const double rx = xi - s[k][0], ry = yi - s[k][1], rz = zi - s[k][2];
        const double ux = s[k][3], uy = s[k][4], uz = s[k][5];
        const double rr = rx * rx + ry * ry + rz * rz;
        const double pr = ux * rx + uy * ry + uz * rz;
        const double sq = sqrt(rr + pr * pr + kEps64);
        const double s3 = sq * sq * sq;
        const double kx = rx / s3, ky = ry / s3, kz = rz / s3;
        const double g = s[k][6];
        e0 += g * kx;
        e1 += g * ky;
        e2 += g * kz;
        b0 += uy * kz - uz * ky;
        b1 += uz * kx - ux * kz;
        b2 += ux * ky - uy * kx;
      }
    }
  }
  if (q < ntarget) {
    if (bad) e0 = e1 = e2 = b0 = b1 = b2 = __longlong_as_double(0x7ff8000000000000ll);
    double *o = part + ((int64_t)split * ntarget + q) * 6;
    o[0] = e0;
    o[1] = e1;
    o[2] = e2;
    o[3] = b0;
    o[4] = b1;
    o[5] = b2;
  }
}

__global__ void direct_reduce_kernel(int64_t ntarget, int splits, const double *__restrict__ part, double amp,
                                     double *__restrict__ oe, double *__restrict__ ob) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntarget) return;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int s = 0; s < splits; ++s)
    for (int c = 0; c < 6; ++c) v[c] += part[((int64_t)s * ntarget + q) * 6 + c];
  for (int c = 0; c < 3; ++c) {
    oe[3 * q + c] = amp * v[c];
    ob[3 * q + c] = amp * v[3 + c];
  }
}

template <class T>
__global__ void fma_peak_kernel(T *out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x * (T)1e-7, x1 = x0 + (T)1e-3, x2 = x0 + (T)2e-3, x3 = x0 + (T)3e-3;
  T x4 = x0 + (T)4e-3, x5 = x0 + (T)5e-3, x6 = x0 + (T)6e-3, x7 = x0 + (T)7e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x0 = fma(x0, a, b);
      x1 = fma(x1, a, b);
      x2 = fma(x2, a, b);
      x3 = fma(x3, a, b);
      x4 = fma(x4, a, b);
      x5 = fma(x5, a, b);
      x6 = fma(x6, a, b);
      x7 = fma(x7, a, b);
    }
  }
  T r = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (r == (T)-1.2345) out[threadIdx.x] = r;  // keeps the chains alive
}

int pick_splits(int64_t N, int64_t ntarget, int64_t max_slots) {
  int splits = 1;
  const int64_t tblocks = (ntarget + kDirThreads - 1) / kDirThreads;
  while (tblocks * splits < 148 * 8 && splits < 1024 && (N / (splits * 2)) >= kDirTile &&
         ntarget * splits * 2 <= max_slots)
    splits *= 2;
  return splits;
}

// Packed FP32x2 FMA chains (Blackwell FFMA2: two FMAs per lane per instruction).
__global__ void fma2_peak_kernel(float *out, int iters, float a, float b) {
  const float2 A = make_float2(a, a), Bv = make_float2(b, b);
  float2 x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = make_float2((float)threadIdx.x * 1e-7f + 1e-3f * k, 2e-3f * k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = __ffma2_rn(x[k], A, Bv);
  }
  float r = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) r += x[k].x + x[k].y;
  if (r == -1.2345f) out[threadIdx.x] = r;
}

int run_direct(Ctx *ctx, int64_t N, const double *d_pos, const double *d_mom, double charge, double lambda,
               int64_t ntarget, const int64_t *d_targets, double *d_e, double *d_b) {
  const int splits = pick_splits(N, ntarget, INT64_MAX);
  const int64_t tblocks = (ntarget + kDirThreads - 1) / kDirThreads;
  double *part;
  FMM_TRY(ctx->ensure("direct_part", 6 * ntarget * splits, &part));
  dim3 grid((unsigned)tblocks, (unsigned)splits);
  direct_partial_kernel<<<grid, kDirThreads, 0, ctx->stream>>>(N, d_pos, d_mom, ntarget, d_targets, splits, part,
                                                               ctx->d_status);
  direct_reduce_kernel<<<ceil_div(ntarget, 256), 256, 0, ctx->stream>>>(ntarget, splits, part,
                                                                        kRe * charge / lambda, d_e, d_b);
  FMM_TRY(ctx->check_launch("direct kernels", 2));
  return ctx->check_device_status("direct");
}

}  // namespace

extern "C" {

int fmmb200_direct_device(fmmb200_ctx *ctx, int64_t npar, const double *d_positions, const double *d_momenta,
                          double charge, double lambda, int64_t ntarget, const int64_t *d_targets,
                          double *d_efields, double *d_bfields) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (npar < 1 || !d_positions || !d_momenta || !d_efields || !d_bfields || ntarget < 1)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "direct: bad arguments");
  if (!d_targets && ntarget > npar)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "direct: ntarget > npar without a target list");
  if (!(lambda != 0.0)) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "lambda must be nonzero");
  cudaSetDevice(ctx->device);
  return run_direct(ctx, npar, d_positions, d_momenta, charge, lambda, ntarget, d_targets, d_efields, d_bfields);
}

int fmmb200_direct(fmmb200_ctx *ctx, int64_t npar, const double *positions, const double *momenta, double charge,
                   double lambda, int64_t ntarget, const int64_t *targets, double *efields, double *bfields) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (npar < 1 || !positions || !momenta || !efields || !bfields)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "direct: bad arguments");
  if (!(lambda != 0.0)) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "lambda must be nonzero");
  const int64_t nt = targets ? ntarget : npar;
  if (nt < 1) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "direct: no targets");
  for (int64_t q = 0; targets && q < nt; ++q)
    if (targets[q] < 0 || targets[q] >= npar) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "target out of range");
  cudaSetDevice(ctx->device);
  double *dp, *dm, *de, *db;
  int64_t *dt = nullptr;
  FMM_TRY(ctx->ensure("dir_pos", 3 * npar, &dp));
  FMM_TRY(ctx->ensure("dir_mom", 3 * npar, &dm));
  FMM_TRY(ctx->ensure("dir_e", 3 * nt, &de));
  FMM_TRY(ctx->ensure("dir_b", 3 * nt, &db));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dp, positions, sizeof(double) * 3 * npar, cudaMemcpyHostToDevice, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dm, momenta, sizeof(double) * 3 * npar, cudaMemcpyHostToDevice, ctx->stream));
  if (targets) {
    FMM_TRY(ctx->ensure("dir_targets", nt, &dt));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dt, targets, sizeof(int64_t) * nt, cudaMemcpyHostToDevice, ctx->stream));
  }
  FMM_TRY(run_direct(ctx, npar, dp, dm, charge, lambda, nt, dt, de, db));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(efields, de, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(bfields, db, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, ctx->stream));
  return ctx->sync();
}

int fmmb200_direct_noalloc(int64_t npar, const double *d_positions, const double *d_momenta, double charge,
                           double lambda, int64_t ntarget, const int64_t *d_targets, double *d_efields,
                           double *d_bfields, void *stream) {
  if (npar < 1 || ntarget < 1 || !d_positions || !d_momenta || !d_efields || !d_bfields || !(lambda != 0.0))
    return FMMB200_ERR_INVALID_ARGUMENT;
  if (!d_targets && ntarget > npar) return FMMB200_ERR_INVALID_ARGUMENT;
  if (ntarget > kNoAllocSlots) return FMMB200_ERR_CAPACITY;
  // This entry point owns no error state: it reads errors with cudaPeekAtLastError and
  // leaves a pending error of the caller's in place.
  if (cudaPeekAtLastError() != cudaSuccess) return FMMB200_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FMMB200_ERR_CUDA;
  double *scratch;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      // once per device, with that device current: the device address of the array
      double *p = nullptr;
      if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p) return FMMB200_ERR_CUDA;
      g_noalloc_ptr[dev] = p;
    }
    scratch = g_noalloc_ptr[dev];
  }
  const int splits = pick_splits(npar, ntarget, kNoAllocSlots);
  const int64_t tblocks = (ntarget + kDirThreads - 1) / kDirThreads;
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid((unsigned)tblocks, (unsigned)splits);
  direct_partial_kernel<<<grid, kDirThreads, 0, st>>>(npar, d_positions, d_momenta, ntarget, d_targets, splits, scratch,
                                                       nullptr);
  direct_reduce_kernel<<<ceil_div(ntarget, 256), 256, 0, st>>>(ntarget, splits, scratch, kRe * charge / lambda,
                                                               d_efields, d_bfields);
  if (cudaPeekAtLastError() != cudaSuccess) return FMMB200_ERR_CUDA;
  return FMMB200_OK;
}

int fmmb200_measure_fma_peak(fmmb200_ctx *ctx, double *fp64_tflops, double *fp32_tflops,
                             double *fp32x2_tflops) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  double *o64;
  float *o32;
  FMM_TRY(ctx->ensure("fma_out64", 1024, &o64));
  FMM_TRY(ctx->ensure("fma_out32", 1024, &o32));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int threads = 256, blocks = nsm * 8;
  double best64 = 0, best32 = 0, best2 = 0;
  for (int rep = 0; rep < 3; ++rep) {
    const int it64 = 4096, it32 = 16384;
    cudaEventRecord(a, ctx->stream);
    fma_peak_kernel<double><<<blocks, threads, 0, ctx->stream>>>(o64, it64, 0.9999999, 1e-9);
    cudaEventRecord(b, ctx->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    const double fl64 = 2.0 * 32.0 * it64 * (double)threads * blocks;
    if (ms > 0) best64 = fl64 / (ms * 1e-3) / 1e12 > best64 ? fl64 / (ms * 1e-3) / 1e12 : best64;
    cudaEventRecord(a, ctx->stream);
    fma_peak_kernel<float><<<blocks, threads, 0, ctx->stream>>>(o32, it32, 0.9999999f, 1e-9f);
    cudaEventRecord(b, ctx->stream);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    const double fl32 = 2.0 * 32.0 * it32 * (double)threads * blocks;
    if (ms > 0) best32 = fl32 / (ms * 1e-3) / 1e12 > best32 ? fl32 / (ms * 1e-3) / 1e12 : best32;
    cudaEventRecord(a, ctx->stream);
    fma2_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(o32, it32 / 2, 0.9999999f, 1e-9f);
    cudaEventRecord(b, ctx->stream);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    const double fl2 = 2.0 * 2.0 * 32.0 * (it32 / 2) * (double)threads * blocks;
    if (ms > 0) best2 = fl2 / (ms * 1e-3) / 1e12 > best2 ? fl2 / (ms * 1e-3) / 1e12 : best2;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  FMM_TRY(ctx->check_launch("fma_peak_kernel", 9));
  if (fp64_tflops) *fp64_tflops = best64;
  if (fp32_tflops) *fp32_tflops = best32;
  if (fp32x2_tflops) *fp32x2_tflops = best2;
  return FMMB200_OK;
}

}  // extern "C"
