// sort.cu -- stable LSD radix sort (8-bit digits) and an int32 exclusive scan.
//
// Per pass: (1) per-tile digit counts, (2) one block per digit scans its row of
// tile counts and adds the digit's global base, (3) each tile ranks its items
// stably (warp-serial rounds with __match_any_sync), reorders them by digit in
// shared memory and writes each digit run contiguously (coalesced).  One
// up-front kernel counts the digits of every pass so that passes whose digit is
// the same for all keys are skipped.
#include "device_util.cuh"
#include "kernels.cuh"

namespace fmmb200 {

namespace {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsThreads * kRsItems;  // 2048 items per tile
constexpr int kRsWarps = kRsThreads / 32;

__global__ void rs_hist_all_kernel(const uint64_t *__restrict__ keys, int64_t n, int npass,
                                   int64_t ntiles, unsigned int *__restrict__ hist_all) {
  __shared__ unsigned int s[8 * 256];
  for (int i = threadIdx.x; i < npass * 256; i += blockDim.x) s[i] = 0;
  __syncthreads();
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int64_t base = tile * kRsTile;
    for (int r = 0; r < kRsItems; ++r) {
      int64_t idx = base + r * kRsThreads + threadIdx.x;
      if (idx < n) {
        uint64_t k = keys[idx];
        for (int p = 0; p < npass; ++p) atomicAdd(&s[p * 256 + (int)((k >> (8 * p)) & 255)], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < npass * 256; i += blockDim.x)
    if (s[i]) atomicAdd(&hist_all[i], s[i]);
}

__global__ void rs_count_kernel(const uint64_t *__restrict__ keys, int64_t n, int shift,
                                int64_t ntiles, unsigned int *__restrict__ counts) {
  __shared__ unsigned int s[256];
  s[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int r = 0; r < kRsItems; ++r) {
    int64_t idx = base + r * kRsThreads + threadIdx.x;
    if (idx < n) atomicAdd(&s[(int)((keys[idx] >> shift) & 255)], 1u);
  }
  __syncthreads();
  counts[(int64_t)threadIdx.x * ntiles + blockIdx.x] = s[threadIdx.x];
}

// One block (1024 threads) per digit: offsets[d][tile] = base(d) + sum_{t'<t} counts[d][t'].
__global__ void rs_scan_kernel(const unsigned int *__restrict__ counts, int64_t ntiles,
                               const unsigned int *__restrict__ hist_pass,
                               unsigned int *__restrict__ offsets) {
  __shared__ int s_warp[33];
  __shared__ unsigned int s_base;
  const int d = blockIdx.x;
  // base(d) = number of keys with a smaller digit
  unsigned int part = (threadIdx.x < (unsigned)d) ? hist_pass[threadIdx.x] : 0u;
  if (threadIdx.x < 256) {
    part = warp_sum(part);
  }
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  if (threadIdx.x < 256 && (threadIdx.x & 31) == 0) atomicAdd(&s_base, part);
  __syncthreads();
  const unsigned int base = s_base;
  const unsigned int *row = counts + (int64_t)d * ntiles;
  unsigned int *orow = offsets + (int64_t)d * ntiles;
  int64_t per = (ntiles + blockDim.x - 1) / blockDim.x;
  int64_t b0 = (int64_t)threadIdx.x * per, b1 = b0 + per < ntiles ? b0 + per : ntiles;
  unsigned int local = 0;
  for (int64_t i = b0; i < b1; ++i) local += row[i];
  int excl = block_excl_scan((int)local, s_warp, nullptr);
  unsigned int run = base + (unsigned int)excl;
  for (int64_t i = b0; i < b1; ++i) {
    unsigned int c = row[i];
    orow[i] = run;
    run += c;
  }
}

template <bool HAS_VALS>
__global__ void __launch_bounds__(kRsThreads)
    rs_scatter_kernel(const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                      uint64_t *__restrict__ kout, uint32_t *__restrict__ vout, int64_t n, int shift,
                      int64_t ntiles, const unsigned int *__restrict__ offsets, int *__restrict__ status) {
  __shared__ uint64_t s_keys[kRsTile];
  __shared__ uint32_t s_vals[HAS_VALS ? kRsTile : 1];
  __shared__ unsigned int s_whist[kRsWarps][256];
  __shared__ unsigned int s_dstart[256];
  __shared__ unsigned int s_goff[256];
  __shared__ int s_warp[33];

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int i = tid; i < kRsWarps * 256; i += kRsThreads) (&s_whist[0][0])[i] = 0;
  s_goff[tid] = offsets[(int64_t)tid * ntiles + blockIdx.x];
  __syncthreads();

  uint64_t k[kRsItems];
  uint32_t v[kRsItems];
  unsigned int dg[kRsItems], rk[kRsItems];
  const unsigned int lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    int64_t idx = base + w * (32 * kRsItems) + r * 32 + lane;
    bool valid = idx < n;
    k[r] = valid ? kin[idx] : 0ull;
    if (HAS_VALS) v[r] = valid ? vin[idx] : 0u;
    dg[r] = valid ? (unsigned int)((k[r] >> shift) & 255) : 256u;
    unsigned int peers = __match_any_sync(0xffffffffu, dg[r]);
    int leader = __ffs(peers) - 1;
    unsigned int before = 0;
    if (lane == leader && dg[r] < 256u) {
      before = s_whist[w][dg[r]];
      s_whist[w][dg[r]] = before + __popc(peers);
    }
    before = __shfl_sync(0xffffffffu, before, leader);
    rk[r] = before + __popc(peers & lt_mask);
  }
  __syncthreads();
  // per digit: exclusive prefix over warps, then over digits
  unsigned int run = 0;
#pragma unroll
  for (int ww = 0; ww < kRsWarps; ++ww) {
    unsigned int c = s_whist[ww][tid];
    s_whist[ww][tid] = run;
    run += c;
  }
  int dstart = block_excl_scan((int)run, s_warp, nullptr);
  s_dstart[tid] = (unsigned int)dstart;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    if (dg[r] < 256u) {
      unsigned int pos = s_dstart[dg[r]] + s_whist[w][dg[r]] + rk[r];
      s_keys[pos] = k[r];
      if (HAS_VALS) s_vals[pos] = v[r];
    }
  }
  __syncthreads();
  int64_t cnt = n - base < kRsTile ? n - base : kRsTile;
  for (int p = tid; p < cnt; p += kRsThreads) {
    uint64_t key = s_keys[p];
    unsigned int d = (unsigned int)((key >> shift) & 255);
    unsigned int dest = s_goff[d] + ((unsigned int)p - s_dstart[d]);
    if ((int64_t)dest >= n) {  // cannot happen for consistent counts; never write out of bounds
      atomicExch(status, kDevBadIndex);
      continue;
    }
    kout[dest] = key;
    if (HAS_VALS) vout[dest] = s_vals[p];
  }
}

// ---------------------------------------------------------------- int32 scan
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void scan_block_sums(const int *__restrict__ in, int64_t n, int *__restrict__ bsum) {
  __shared__ int s_warp[33];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int local = 0;
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) local += in[base + i];
  int total;
  block_excl_scan(local, s_warp, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// single block: exclusive scan of nb block sums in place, total into *total
__global__ void scan_top(int *__restrict__ bsum, int64_t nb, long long *__restrict__ total) {
  __shared__ int s_warp[33];
  __shared__ long long s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int64_t off = 0; off < nb; off += blockDim.x) {
    int64_t i = off + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    int tot;
    int ex = block_excl_scan(v, s_warp, &tot);
    if (i < nb) bsum[i] = (int)(s_carry + ex);
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = s_carry;
}

__global__ void scan_apply(const int *__restrict__ in, int *__restrict__ out, int64_t n,
                           const int *__restrict__ bsum) {
  __shared__ int s_warp[33];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int vals[kScanItems];
  int local = 0;
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = base + i < n ? in[base + i] : 0;
    local += vals[i];
  }
  int ex = block_excl_scan(local, s_warp, nullptr) + bsum[blockIdx.x];
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = ex;
    ex += vals[i];
  }
}

}  // namespace

int exclusive_scan_i32(Ctx *ctx, const int *in, int *out, int64_t n, int64_t *total) {
  if (n <= 0) {
    if (total) *total = 0;
    return FMMB200_OK;
  }
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  int *bsum = nullptr;
  long long *d_total = nullptr;
  FMM_TRY(ctx->ensure("scan_bsum", nb, &bsum));
  FMM_TRY(ctx->ensure("scan_total", 1, &d_total));
  scan_block_sums<<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, n, bsum);
  scan_top<<<1, kScanThreads, 0, ctx->stream>>>(bsum, nb, d_total);
  scan_apply<<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, out, n, bsum);
  FMM_TRY(ctx->check_launch("exclusive_scan_i32", 3));
  if (total) {
    long long *h = nullptr;
    FMM_TRY(ctx->pinned(sizeof(long long), (void **)&h));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_total, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    FMM_TRY(ctx->sync());
    *total = (int64_t)*h;
  }
  return FMMB200_OK;
}

int radix_sort(Ctx *ctx, uint64_t *keys, uint64_t *keys_alt, uint32_t *vals, uint32_t *vals_alt,
               int64_t n, int key_bits, bool *in_alt) {
  *in_alt = false;
  if (n <= 1 || key_bits <= 0) return FMMB200_OK;
  if (n > (int64_t)0xFFFFFFFFll) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "radix_sort: n >= 2^32");
  const int npass = (key_bits + 7) / 8;
  const int64_t ntiles = (n + kRsTile - 1) / kRsTile;
  unsigned int *hist_all = nullptr, *counts = nullptr, *offsets = nullptr;
  FMM_TRY(ctx->ensure("rs_hist_all", 8 * 256, &hist_all));
  FMM_TRY(ctx->ensure("rs_counts", 256 * ntiles, &counts));
  FMM_TRY(ctx->ensure("rs_offsets", 256 * ntiles, &offsets));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(hist_all, 0, sizeof(unsigned int) * 8 * 256, ctx->stream));
  int hgrid = (int)(ntiles < 148 * 4 ? ntiles : 148 * 4);
  rs_hist_all_kernel<<<hgrid, kRsThreads, 0, ctx->stream>>>(keys, n, npass, ntiles, hist_all);
  FMM_TRY(ctx->check_launch("rs_hist_all_kernel"));
  unsigned int *h = nullptr;
  FMM_TRY(ctx->pinned(sizeof(unsigned int) * 8 * 256, (void **)&h));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h, hist_all, sizeof(unsigned int) * npass * 256,
                                    cudaMemcpyDeviceToHost, ctx->stream));
  FMM_TRY(ctx->sync());
  bool trivial[8];
  for (int p = 0; p < npass; ++p) {
    trivial[p] = false;
    for (int d = 0; d < 256; ++d)
      if ((int64_t)h[p * 256 + d] == n) trivial[p] = true;
  }
  bool cur = false;
  for (int p = 0; p < npass; ++p) {
    if (trivial[p]) continue;
    const int shift = 8 * p;
    uint64_t *ki = cur ? keys_alt : keys, *ko = cur ? keys : keys_alt;
    uint32_t *vi = cur ? vals_alt : vals, *vo = cur ? vals : vals_alt;
    rs_count_kernel<<<(unsigned)ntiles, kRsThreads, 0, ctx->stream>>>(ki, n, shift, ntiles, counts);
    rs_scan_kernel<<<256, 1024, 0, ctx->stream>>>(counts, ntiles, hist_all + p * 256, offsets);
    if (vals)
      rs_scatter_kernel<true><<<(unsigned)ntiles, kRsThreads, 0, ctx->stream>>>(ki, vi, ko, vo, n, shift,
                                                                              ntiles, offsets, ctx->d_status);
    else
      rs_scatter_kernel<false><<<(unsigned)ntiles, kRsThreads, 0, ctx->stream>>>(ki, nullptr, ko, nullptr, n,
                                                                               shift, ntiles, offsets, ctx->d_status);
    FMM_TRY(ctx->check_launch("radix_sort pass", 3));
    cur = !cur;
  }
  *in_alt = cur;
  return FMMB200_OK;
}

}  // namespace fmmb200
