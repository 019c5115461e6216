// traverse.cu -- device dual-tree traversal (the reference's dualtraversefill!,
// src/fmm/interaction_lists.jl:23-49, a host recursion there) and the CSR
// grouping by target (InteractionListsGPU, src/gpu_fmm/gpu_interaction_lists.jl:27-40).
//
// Design: a breadth-first traversal over frontiers of (target, source) pairs.
// Each step classifies every frontier pair with the reference's rules (both
// leaves -> P2P; admissible -> M2L; otherwise split the non-leaf side, or the
// side with the larger stretched diameter, ties to the source) and writes its
// outputs at offsets from a block scan, so every step is deterministic.  The
// set of emitted pairs equals the DFS's.  Both lists are then radix-sorted by
// (target, source) and grouped into CSR pointers over all clusters.
#include <algorithm>
#include <cstring>
#include <string>

#include "device_util.cuh"
#include "kernels.cuh"

namespace fmmb200 {

namespace {

// Device state of a traversal (long long words): frontier size, P2P and M2L pairs so
// far, overflow flag, the largest frontier, the steps whose frontier was not empty.
enum : int { kTsFront = 0, kTsP2P = 1, kTsM2L = 2, kTsOver = 3, kTsMaxFront = 4, kTsSteps = 5, kTsWords = 8 };

constexpr int kTvThreads = 256;
constexpr int kTvItems = 4;
constexpr int kTvTile = kTvThreads * kTvItems;

enum : int { kCatP2P = 0, kCatM2L = 1, kCatSplit = 2 };
// per-pair codes the count kernel leaves for the write kernel (kCatP2P and kCatM2L as above)
enum : int { kCodeSplitT = 2, kCodeSplitS = 3 };

// Target filter of a sharded traversal (TravFilter::L < 0: every target).  A rank that
// owns the level-L cluster g (heap id) needs the rows of g's descendants and of g's
// ancestors only; a split whose target child is neither drops that child pair.
struct TravFilter {
  int L;
  int g;
};

__device__ __forceinline__ bool trav_relevant(int t, TravFilter f) {
  if (f.L < 0) return true;
  const int lt = 31 - __clz(t + 1);
  if (lt <= f.L) return ((f.g + 1) >> (f.L - lt)) == t + 1;  // t is g or an ancestor of g
  return ((t + 1) >> (lt - f.L)) == f.g + 1;                  // t is below g
}

// Returns the category; for a split, (*ct1,*cs1),(*ct2,*cs2) are the child pairs.
__device__ __forceinline__ int classify(const ClusterGeom *__restrict__ geom, int t, int s, double s0, double s1,
                                        double s2, double eta, int *ct1, int *cs1, int *ct2, int *cs2) {
  const ClusterGeom gt = geom[t], gs = geom[s];
  if (gt.leaf && gs.leaf) return kCatP2P;
  // admissible(): max(r1,r2)/R < eta with R = norm(stretch .* (xc1 - xc2))
  double R = norm3_exact(rn_mul(s0, rn_sub(gt.xc[0], gs.xc[0])), rn_mul(s1, rn_sub(gt.xc[1], gs.xc[1])),
                         rn_mul(s2, rn_sub(gt.xc[2], gs.xc[2])));
  double m = gt.r > gs.r ? gt.r : gs.r;
  if (__ddiv_rn(m, R) < eta) return kCatM2L;
  bool split_t;
  if (gt.leaf)
    split_t = false;
  else if (gs.leaf)
    split_t = true;
  else
    split_t = gt.diam > gs.diam;
  if (split_t) {
    *ct1 = 2 * t + 1;
    *cs1 = s;
    *ct2 = 2 * t + 2;
    *cs2 = s;
  } else {
    *ct1 = t;
    *cs1 = 2 * s + 1;
    *ct2 = t;
    *cs2 = 2 * s + 2;
  }
  return kCatSplit;
}

// Counts per tile of the frontier: P2P pairs, M2L pairs and the child pairs of the
// splits (two per split, fewer when the target filter drops one).  The grid is fixed and
// strides over the tiles that the frontier (state, on the device) occupies.
__global__ void trav_count_kernel(const int2 *__restrict__ front, const long long *__restrict__ state,
                                  const ClusterGeom *__restrict__ geom, const double *__restrict__ consts, double eta,
                                  int nblk, TravFilter flt, int *__restrict__ bcount, int *__restrict__ totals,
                                  uint8_t *__restrict__ code) {
  __shared__ int s_warp[33];
  const int nf = (int)state[kTsFront];
  const int ntile = (nf + kTvTile - 1) / kTvTile;
  const double s0 = consts[3], s1 = consts[4], s2 = consts[5];
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    int c[3] = {0, 0, 0};
    const int i0 = tile * kTvTile + threadIdx.x * kTvItems;
    for (int i = 0; i < kTvItems; ++i) {
      const int q = i0 + i;
      if (q < nf) {
        const int2 p = front[q];
        int a, b, cc, d;
        const int cat = classify(geom, p.x, p.y, s0, s1, s2, eta, &a, &b, &cc, &d);
        if (cat == kCatSplit)
          c[2] += (int)trav_relevant(a, flt) + (int)trav_relevant(cc, flt);
        else
          c[cat]++;
        // the decision for trav_write_kernel: P2P, M2L, split the target, split the source
        code[q] = (uint8_t)(cat != kCatSplit ? cat : (a != p.x ? kCodeSplitT : kCodeSplitS));
      }
    }
    for (int k = 0; k < 3; ++k) {
      int tot;
      block_excl_scan(c[k], s_warp, &tot);
      if (threadIdx.x == 0) {
        bcount[k * nblk + tile] = tot;
        if (tot) atomicAdd(&totals[k], tot);
      }
      __syncthreads();
    }
  }
}

// Exclusive scan, per category, of the counts of the tiles the frontier occupies (one
// block; boff[k * nblk] = 0).
constexpr int kTileScanItems = 16;
__global__ void __launch_bounds__(1024) tile_scan_kernel(const int *__restrict__ bcount, int nblk,
                                                         const long long *__restrict__ state, int *__restrict__ boff) {
  __shared__ int s_warp[33];
  const int ntile = (int)((state[kTsFront] + kTvTile - 1) / kTvTile);
  for (int k = 0; k < 3; ++k) {
    const int *in = bcount + (int64_t)k * nblk;
    int *out = boff + (int64_t)k * nblk;
    int carry = 0;
    for (int c0 = 0; c0 < ntile; c0 += 1024 * kTileScanItems) {
      const int i0 = c0 + threadIdx.x * kTileScanItems;
      int v[kTileScanItems], sum = 0;
#pragma unroll
      for (int j = 0; j < kTileScanItems; ++j) {
        v[j] = i0 + j < ntile ? in[i0 + j] : 0;
        sum += v[j];
      }
      int chunk;
      int run = carry + block_excl_scan(sum, s_warp, &chunk);
#pragma unroll
      for (int j = 0; j < kTileScanItems; ++j) {
        if (i0 + j < ntile) out[i0 + j] = run;
        run += v[j];
      }
      carry += chunk;
      __syncthreads();
    }
  }
}

// Writes the step's pairs after the ones of the earlier steps (state) and its children as
// the next frontier, from the count kernel's decision per pair (no geometry is read again); a write past a buffer's capacity is dropped (the step's totals still
// count it, and trav_advance_kernel raises the overflow flag).
__global__ void trav_write_kernel(const int2 *__restrict__ front, const long long *__restrict__ state,
                                  const uint8_t *__restrict__ code, int nblk, TravFilter flt,
                                  const int *__restrict__ boff, int bits, uint64_t *__restrict__ p2p, long long cap_p,
                                  uint64_t *__restrict__ m2l, long long cap_m, int2 *__restrict__ next, long long cap_f) {
  __shared__ int s_warp[33];
  const int nf = (int)state[kTsFront];
  const int ntile = (nf + kTvTile - 1) / kTvTile;
  const long long base_p = state[kTsP2P], base_m = state[kTsM2L];
  for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    int cat[kTvItems];
    int2 pr[kTvItems], ch1[kTvItems], ch2[kTvItems];
    int c[3] = {0, 0, 0};
    const int i0 = tile * kTvTile + threadIdx.x * kTvItems;
    for (int i = 0; i < kTvItems; ++i) {
      const int q = i0 + i;
      cat[i] = -1;
      if (q < nf) {
        pr[i] = front[q];
        const int k = code[q];  // the count kernel's decision for this pair
        cat[i] = k < kCatSplit ? k : kCatSplit;
        if (k == kCodeSplitT) {
          ch1[i] = make_int2(2 * pr[i].x + 1, pr[i].y);
          ch2[i] = make_int2(2 * pr[i].x + 2, pr[i].y);
        } else if (k == kCodeSplitS) {
          ch1[i] = make_int2(pr[i].x, 2 * pr[i].y + 1);
          ch2[i] = make_int2(pr[i].x, 2 * pr[i].y + 2);
        }
        if (cat[i] == kCatSplit)
          c[2] += (int)trav_relevant(ch1[i].x, flt) + (int)trav_relevant(ch2[i].x, flt);
        else
          c[cat[i]]++;
      }
    }
    int pos[3];
    for (int k = 0; k < 3; ++k) {
      pos[k] = block_excl_scan(c[k], s_warp, nullptr) + boff[k * nblk + tile];
      __syncthreads();
    }
    for (int i = 0; i < kTvItems; ++i) {
      if (cat[i] < 0) continue;
      uint64_t key = ((uint64_t)pr[i].x << bits) | (uint64_t)pr[i].y;
      if (cat[i] == kCatP2P) {
        const long long o = base_p + pos[0]++;
        if (o < cap_p) p2p[o] = key;
      } else if (cat[i] == kCatM2L) {
        const long long o = base_m + pos[1]++;
        if (o < cap_m) m2l[o] = key;
      } else {
        if (trav_relevant(ch1[i].x, flt)) {
          const int o = pos[2]++;
          if (o < cap_f) next[o] = ch1[i];
        }
        if (trav_relevant(ch2[i].x, flt)) {
          const int o = pos[2]++;
          if (o < cap_f) next[o] = ch2[i];
        }
      }
    }
  }
}

// After a step: the pair counts grow by the step's totals, the frontier becomes its
// children, and the largest needs so far are kept; a need above a capacity raises the
// overflow flag.  The step's totals are reset for the next step.
__global__ void trav_advance_kernel(long long *__restrict__ state, int *__restrict__ totals, long long cap_p,
                                    long long cap_m, long long cap_f) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  state[kTsP2P] += totals[0];
  state[kTsM2L] += totals[1];
  const long long nf = totals[2];
  state[kTsFront] = nf < cap_f ? nf : cap_f;
  if (nf > state[kTsMaxFront]) state[kTsMaxFront] = nf;
  if (nf > 0) state[kTsSteps] += 1;
  if (state[kTsP2P] > cap_p || state[kTsM2L] > cap_m || nf > cap_f) state[kTsOver] = 1;
  totals[0] = totals[1] = totals[2] = 0;
}

// ptr[c] = first list position with target c (lists sorted by key), src[i] = source.
__global__ void csr_kernel(const uint64_t *__restrict__ keys, int64_t n, int bits, int64_t nc,
                           int *__restrict__ ptr) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c > nc) return;
  uint64_t want = (uint64_t)c << bits;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < want)
      lo = mid + 1;
    else
      hi = mid;
  }
  ptr[c] = (int)lo;
}

__global__ void src_kernel(const uint64_t *__restrict__ keys, int64_t n, int bits, int *__restrict__ src) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  src[i] = (int)(keys[i] & (((uint64_t)1 << bits) - 1));
}

__global__ void p2p_work_kernel(const uint64_t *__restrict__ keys, int64_t n, int bits, const int *__restrict__ lohi,
                                unsigned long long *__restrict__ out) {
  __shared__ unsigned long long s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long w = 0;
  if (i < n) {
    uint64_t k = keys[i];
    int t = (int)(k >> bits), sc = (int)(k & (((uint64_t)1 << bits) - 1));
    w = (unsigned long long)(lohi[2 * t + 1] - lohi[2 * t] + 1) * (unsigned long long)(lohi[2 * sc + 1] - lohi[2 * sc] + 1);
  }
  w = warp_sum(w);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(&s, w);
  __syncthreads();
  if (threadIdx.x == 0 && s) atomicAdd(out, s);
}

// Counts the pairs (t,s) of a sorted list whose transpose (s,t) is missing.
__global__ void transpose_missing_kernel(const uint64_t *__restrict__ keys, int64_t n, int bits,
                                         unsigned long long *__restrict__ missing) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int miss = 0;
  if (i < n) {
    const uint64_t k = keys[i], mask = ((uint64_t)1 << bits) - 1;
    const uint64_t want = ((k & mask) << bits) | (k >> bits);
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < want)
        lo = mid + 1;
      else
        hi = mid;
    }
    miss = !(lo < n && keys[lo] == want);
  }
  const unsigned long long w = warp_sum((unsigned long long)miss);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(missing, w);
}

// Union of a sorted pair list and its transpose: entry (t,s) with bit 61 if
// (t,s) is in the list and bit 62 if (s,t) is.
__global__ void union_fill_kernel(const uint64_t *__restrict__ keys, int64_t n, int bits, uint64_t *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = keys[i], mask = ((uint64_t)1 << bits) - 1;
  out[i] = k | ((uint64_t)1 << 61);
  out[n + i] = (((k & mask) << bits) | (k >> bits)) | ((uint64_t)1 << 62);
}

__global__ void union_head_kernel(const uint64_t *__restrict__ u, int64_t n, uint64_t low, int *__restrict__ head) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  head[i] = (i == 0 || (u[i] & low) != (u[i - 1] & low)) ? 1 : 0;
}

__global__ void union_compact_kernel(const uint64_t *__restrict__ u, int64_t n, uint64_t low, const int *__restrict__ head,
                                     const int *__restrict__ pos, uint64_t *__restrict__ ukeys, uint8_t *__restrict__ uflag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !head[i]) return;
  uint64_t f = u[i] >> 61;
  if (i + 1 < n && (u[i + 1] & low) == (u[i] & low)) f |= u[i + 1] >> 61;
  ukeys[pos[i]] = u[i] & low;
  uflag[pos[i]] = (uint8_t)f;
}

int sort_and_group(Ctx *ctx, const char *keys_name, const char *alt_name, const char *ptr_name,
                   const char *src_name, int64_t n, int bits) {
  uint64_t *keys = ctx->get<uint64_t>(keys_name), *alt = nullptr;
  FMM_TRY(ctx->ensure(alt_name, n, &alt));
  keys = ctx->get<uint64_t>(keys_name);
  bool in_alt = false;
  FMM_TRY(radix_sort(ctx, keys, alt, nullptr, nullptr, n, 2 * bits, &in_alt));
  // Copied back rather than swapping the two names: the keys buffer keeps the traversal's
  // capacity, so the next traversal does not reallocate it (a synchronising free and copy).
  if (in_alt && n > 0)
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(keys, alt, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  int *ptr, *src;
  FMM_TRY(ctx->ensure(ptr_name, ctx->nc + 1, &ptr));
  FMM_TRY(ctx->ensure(src_name, n, &src));
  csr_kernel<<<ceil_div(ctx->nc + 1, 256), 256, 0, ctx->stream>>>(keys, n, bits, ctx->nc, ptr);
  if (n > 0) src_kernel<<<ceil_div(n, 256), 256, 0, ctx->stream>>>(keys, n, bits, src);
  return ctx->check_launch("sort_and_group", n > 0 ? 2 : 1);
}

int build_union(Ctx *ctx, const char *keys_name, int64_t n, const char *prefix, const char *list_prefix) {
  const int bits = ctx->list_bits;
  const std::string kn = std::string(prefix) + "_keys", fn = std::string(prefix) + "_flag";
  const std::string pn = std::string(prefix) + "_ptr", sn = std::string(prefix) + "_src";
  // A symmetric list (the usual case: the traversal's rules are symmetric except for ties of
  // the diameters) is its own union, every pair in both roles: the same CSR, flags 3.
  if (n > 0) {
    unsigned long long *d_miss, *h_miss;
    FMM_TRY(ctx->ensure("union_missing", 1, &d_miss));
    FMM_CUDA_TRY(ctx, cudaMemsetAsync(d_miss, 0, sizeof(unsigned long long), ctx->stream));
    transpose_missing_kernel<<<ceil_div(n, 256), 256, 0, ctx->stream>>>(ctx->get<uint64_t>(keys_name), n, bits, d_miss);
    FMM_TRY(ctx->check_launch("transpose_missing_kernel"));
    FMM_TRY(ctx->pinned(sizeof(unsigned long long), (void **)&h_miss));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h_miss, d_miss, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    FMM_TRY(ctx->sync());
    if (*h_miss == 0) {
      uint64_t *uk;
      uint8_t *uf;
      int *ptr, *src;
      FMM_TRY(ctx->ensure(kn.c_str(), n, &uk));
      FMM_TRY(ctx->ensure(fn.c_str(), n, &uf));
      FMM_TRY(ctx->ensure(pn.c_str(), ctx->nc + 1, &ptr));
      FMM_TRY(ctx->ensure(sn.c_str(), n, &src));
      const std::string lp = std::string(list_prefix) + "_ptr", ls = std::string(list_prefix) + "_src";
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(uk, ctx->get<uint64_t>(keys_name), sizeof(uint64_t) * n,
                                        cudaMemcpyDeviceToDevice, ctx->stream));
      FMM_CUDA_TRY(ctx, cudaMemsetAsync(uf, 3, n, ctx->stream));
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(ptr, ctx->get<int>(lp.c_str()), sizeof(int) * (ctx->nc + 1),
                                        cudaMemcpyDeviceToDevice, ctx->stream));
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(src, ctx->get<int>(ls.c_str()), sizeof(int) * n, cudaMemcpyDeviceToDevice,
                                        ctx->stream));
      return FMMB200_OK;
    }
  }
  const int64_t n2 = 2 * n;
  uint64_t *u, *ua;
  int *head, *pos;
  FMM_TRY(ctx->ensure("union_u", n2, &u));
  FMM_TRY(ctx->ensure("union_ua", n2, &ua));
  FMM_TRY(ctx->ensure("union_head", n2, &head));
  FMM_TRY(ctx->ensure("union_pos", n2, &pos));
  if (n > 0) union_fill_kernel<<<ceil_div(n, 256), 256, 0, ctx->stream>>>(ctx->get<uint64_t>(keys_name), n, bits, u);
  FMM_TRY(ctx->check_launch("union_fill_kernel", n > 0 ? 1 : 0));
  bool alt = false;
  FMM_TRY(radix_sort(ctx, u, ua, nullptr, nullptr, n2, 2 * bits, &alt));
  const uint64_t *us = alt ? ua : u;
  const uint64_t low = ((uint64_t)1 << (2 * bits)) - 1;
  int64_t nu = 0;
  if (n2 > 0) {
    union_head_kernel<<<ceil_div(n2, 256), 256, 0, ctx->stream>>>(us, n2, low, head);
    FMM_TRY(ctx->check_launch("union_head_kernel"));
    FMM_TRY(exclusive_scan_i32(ctx, head, pos, n2, &nu));
  }
  uint64_t *uk;
  uint8_t *uf;
  int *ptr, *src;
  FMM_TRY(ctx->ensure(kn.c_str(), nu, &uk));
  FMM_TRY(ctx->ensure(fn.c_str(), nu, &uf));
  FMM_TRY(ctx->ensure(pn.c_str(), ctx->nc + 1, &ptr));
  FMM_TRY(ctx->ensure(sn.c_str(), nu, &src));
  if (n2 > 0) {
    union_compact_kernel<<<ceil_div(n2, 256), 256, 0, ctx->stream>>>(us, n2, low, head, pos, uk, uf);
    FMM_TRY(ctx->check_launch("union_compact_kernel"));
  }
  csr_kernel<<<ceil_div(ctx->nc + 1, 256), 256, 0, ctx->stream>>>(uk, nu, bits, ctx->nc, ptr);
  if (nu > 0) src_kernel<<<ceil_div(nu, 256), 256, 0, ctx->stream>>>(uk, nu, bits, src);
  return ctx->check_launch("union csr", nu > 0 ? 2 : 1);
}

}  // namespace

// Grow a device buffer keeping its first `used` bytes.
int grow_keep(Ctx *ctx, const char *name, size_t used, size_t need, void **out) {
  auto it = ctx->bufs.find(name);
  if (it != ctx->bufs.end() && it->second.cap >= need) {
    *out = it->second.p;
    return FMMB200_OK;
  }
  void *fresh = nullptr;
  size_t want = need + need / 2;
  want = (want + 255) & ~(size_t)255;
  if (ctx->fail_alloc_countdown > 0 && --ctx->fail_alloc_countdown == 0)
    return ctx->fail(FMMB200_ERR_OUT_OF_MEMORY, std::string("injected allocation failure for buffer '") + name + "'");
  cudaError_t e = cudaMalloc(&fresh, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return ctx->fail(FMMB200_ERR_OUT_OF_MEMORY, std::string("cudaMalloc for '") + name + "': " + cudaGetErrorString(e));
  }
  if (it != ctx->bufs.end() && it->second.p) {
    if (used) FMM_CUDA_TRY(ctx, cudaMemcpyAsync(fresh, it->second.p, used, cudaMemcpyDeviceToDevice, ctx->stream));
    FMM_TRY(ctx->sync());
    cudaFree(it->second.p);
    ctx->device_bytes -= it->second.cap;
  }
  auto &b = ctx->bufs[name];
  b.p = fresh;
  b.cap = want;
  ctx->device_bytes += want;
  *out = fresh;
  return FMMB200_OK;
}

int build_union_lists(Ctx *ctx) {
  FMM_TRY(build_union(ctx, "m2l_keys", ctx->nm2l, "m2lu", "m2l"));
  FMM_TRY(build_union(ctx, "p2p_keys", ctx->np2p, "p2pu", "p2p"));
  return FMMB200_OK;
}

int build_lists(Ctx *ctx, double eta, const double *d_consts) {
  const int64_t nc = ctx->nc;
  FMM_TRY(compute_geom(ctx, d_consts));
  int bits = 1;
  while (((int64_t)1 << bits) < nc) ++bits;
  // Capacities: what the previous traversal of the same tree shape, eta and filter needed,
  // else estimates; a traversal that outgrows one is run again with enough room (the first
  // call of a configuration).  The frontier capacity also sizes every step's grid, so the
  // needs of another configuration are not carried over.
  const double key[4] = {(double)nc, eta, (double)ctx->trav_L, (double)ctx->trav_g};
  if (std::memcmp(key, ctx->trav_key, sizeof(key)) != 0) {
    std::memcpy(ctx->trav_key, key, sizeof(key));
    ctx->trav_need_p = ctx->trav_need_m = ctx->trav_need_f = 0;
  }
  int64_t cap_p = std::max<int64_t>(ctx->trav_need_p, 64 * ctx->nleaf + 1024);
  int64_t cap_m = std::max<int64_t>(ctx->trav_need_m, 32 * nc + 1024);
  int64_t cap_f = std::max<int64_t>(ctx->trav_need_f, 4 * nc + 1024);
  // Every step adds one level to the target or the source of a pair, so the frontier is
  // empty after at most 2 ml + 1 steps; the loop runs that many without reading anything
  // back, each step's work sized on the device.
  const int max_steps = 2 * ctx->ml + 2;
  int2 *fa, *fb;
  uint64_t *p2p, *m2l;
  int *bcount, *boff, *totals;
  long long *state, *h = nullptr;
  FMM_TRY(ctx->ensure("trav_totals", 4, &totals));
  FMM_TRY(ctx->ensure("trav_state", kTsWords, &state));
  const ClusterGeom *geom = ctx->get<ClusterGeom>("geom");
  const TravFilter flt{ctx->trav_L, ctx->trav_g};
  int64_t np2p = 0, nm2l = 0, steps = 0;
  for (int attempt = 0;; ++attempt) {
    FMM_TRY(ctx->ensure("front_a", cap_f, &fa));
    FMM_TRY(ctx->ensure("front_b", cap_f, &fb));
    void *vp;
    FMM_TRY(grow_keep(ctx, "p2p_keys", 0, sizeof(uint64_t) * cap_p, &vp));
    p2p = (uint64_t *)vp;
    FMM_TRY(grow_keep(ctx, "m2l_keys", 0, sizeof(uint64_t) * cap_m, &vp));
    m2l = (uint64_t *)vp;
    const int nblk = ceil_div(cap_f, kTvTile);             // tiles the frontier can occupy
    const int grid = nblk < 148 * 8 ? nblk : 148 * 8;       // blocks, striding over the tiles in use
    FMM_TRY(ctx->ensure("trav_bcount", 3 * (int64_t)nblk, &bcount));
    FMM_TRY(ctx->ensure("trav_boff", 3 * (int64_t)nblk, &boff));
    uint8_t *code;
    FMM_TRY(ctx->ensure("trav_code", cap_f, &code));  // one decision per frontier pair
    const long long init[kTsWords] = {1, 0, 0, 0, 1, 0, 0, 0};
    const int2 root = make_int2(0, 0);
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(state, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(fa, &root, sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    FMM_CUDA_TRY(ctx, cudaMemsetAsync(totals, 0, sizeof(int) * 4, ctx->stream));
    for (int step = 0; step < max_steps; ++step) {
      const int2 *cur = step % 2 == 0 ? fa : fb;
      int2 *nxt = step % 2 == 0 ? fb : fa;
      trav_count_kernel<<<grid, kTvThreads, 0, ctx->stream>>>(cur, state, geom, d_consts, eta, nblk, flt, bcount,
                                                               totals, code);
      tile_scan_kernel<<<1, 1024, 0, ctx->stream>>>(bcount, nblk, state, boff);
      trav_write_kernel<<<grid, kTvThreads, 0, ctx->stream>>>(cur, state, code, nblk, flt, boff, bits, p2p, cap_p, m2l,
                                                               cap_m, nxt, cap_f);
      trav_advance_kernel<<<1, 32, 0, ctx->stream>>>(state, totals, cap_p, cap_m, cap_f);
      FMM_TRY(ctx->check_launch("trav_count/scan/write/advance kernels", 4));
    }
    FMM_TRY(ctx->pinned(sizeof(long long) * kTsWords, (void **)&h));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h, state, sizeof(long long) * kTsWords, cudaMemcpyDeviceToHost, ctx->stream));
    FMM_TRY(ctx->sync());
    np2p = h[kTsP2P];
    nm2l = h[kTsM2L];
    steps = h[kTsSteps] + 1;
    if (h[kTsFront] != 0) return ctx->fail(FMMB200_ERR_DEVICE, "traversal did not terminate");
    // keep the needs (never a capacity: repeated calls must not compound the headroom)
    ctx->trav_need_p = std::max<int64_t>(ctx->trav_need_p, np2p);
    ctx->trav_need_m = std::max<int64_t>(ctx->trav_need_m, nm2l);
    ctx->trav_need_f = std::max<int64_t>(ctx->trav_need_f, h[kTsMaxFront] + 1);
    if (!h[kTsOver]) break;
    if (attempt >= 8) return ctx->fail(FMMB200_ERR_DEVICE, "traversal buffers did not converge");
    // grow what overflowed; after a truncated frontier the later counts are lower bounds,
    // so a second pass may still grow a buffer
    if (np2p > cap_p) cap_p = std::max<int64_t>(2 * cap_p, np2p + 1024);
    if (nm2l > cap_m) cap_m = std::max<int64_t>(2 * cap_m, nm2l + 1024);
    if (h[kTsMaxFront] > cap_f) cap_f = std::max<int64_t>(2 * cap_f, 2 * h[kTsMaxFront]);  // a lower bound
  }
  ctx->nm2l = nm2l;
  ctx->np2p = np2p;
  ctx->traversal_steps = (int)steps;
  FMM_TRY(sort_and_group(ctx, "m2l_keys", "m2l_keys_alt", "m2l_ptr", "m2l_src", nm2l, bits));
  FMM_TRY(sort_and_group(ctx, "p2p_keys", "p2p_keys_alt", "p2p_ptr", "p2p_src", np2p, bits));
  // exact P2P work for the stats
  unsigned long long *d_work;
  FMM_TRY(ctx->ensure("p2p_work", 1, &d_work));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(d_work, 0, sizeof(unsigned long long), ctx->stream));
  if (np2p > 0) {
    p2p_work_kernel<<<ceil_div(np2p, 256), 256, 0, ctx->stream>>>(ctx->get<uint64_t>("p2p_keys"), np2p, bits,
                                                                  ctx->get<int>("lohi"), d_work);
    FMM_TRY(ctx->check_launch("p2p_work_kernel"));
  }
  unsigned long long *hw;
  FMM_TRY(ctx->pinned(sizeof(unsigned long long), (void **)&hw));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(hw, d_work, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  FMM_TRY(ctx->sync());
  ctx->stats.p2p_kernel_evals = (double)*hw;
  ctx->list_bits = bits;
  ctx->have_lists = true;
  return FMMB200_OK;
}

}  // namespace fmmb200
