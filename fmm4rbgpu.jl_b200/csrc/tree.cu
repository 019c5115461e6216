// tree.cu -- device cluster-tree build (the reference's ClusterTree /
// fillclusters!, src/cluster_tree/clusters.jl:21-70, on the host there).
//
// Design (B200): the three coordinate orders are radix-sorted once (64-bit
// order-preserving keys, ties by particle id).  Level by level (globally down to
// the first level whose nodes hold at most 4096 particles, then per subtree in
// shared memory, see subtree_kernel), every node's
// bounding box is read off the ends of its three sorted segments (exact
// min/max), the split axis is argmax(stretch .* extent) and the left child
// takes the first ceil(cnt/2) particles of the split-axis segment -- the
// k-th-element split of kpermute!, with ties broken by particle id.  The other
// two segments are partitioned stably with a global scan of the left flags, so
// every segment stays sorted.  This is O(N) streaming work per level instead of
// a serial quickselect.  Finally the particle ids inside each leaf are put in
// ascending order (a stable sort by leaf id), the canonical form of the
// reference's per-leaf sets.
#include <cmath>
#include <vector>

#include "device_util.cuh"
#include "interp_util.cuh"
#include "kernels.cuh"

namespace fmmb200 {

namespace {

// ---------------------------------------------------------------- p_avg
// Leaves of Base.mapreduce_impl: sequential sums of [first, last].
__global__ void pw_leaf_kernel(const double *__restrict__ mom, const int64_t *__restrict__ lf,
                               const int64_t *__restrict__ ll, int nleaf, double *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaf) return;
  int64_t first = lf[i], last = ll[i];
  double s0, s1, s2;
  if (first == last) {
    s0 = mom[3 * first];
    s1 = mom[3 * first + 1];
    s2 = mom[3 * first + 2];
  } else {
    s0 = rn_add(mom[3 * first], mom[3 * first + 3]);
    s1 = rn_add(mom[3 * first + 1], mom[3 * first + 4]);
    s2 = rn_add(mom[3 * first + 2], mom[3 * first + 5]);
    for (int64_t k = first + 2; k <= last; ++k) {
      s0 = rn_add(s0, mom[3 * k]);
      s1 = rn_add(s1, mom[3 * k + 1]);
      s2 = rn_add(s2, mom[3 * k + 2]);
    }
  }
  out[3 * i] = s0;
  out[3 * i + 1] = s1;
  out[3 * i + 2] = s2;
}

// Internal nodes of the pairwise recursion, combined height by height
// (single block).  ref >= 0 is a leaf sum, ref < 0 the internal node -ref-1.
__global__ void pw_combine_kernel(const int *__restrict__ nl, const int *__restrict__ nr,
                                  const int *__restrict__ order, const int *__restrict__ hoff, int H,
                                  const double *__restrict__ leafsum, double *__restrict__ nodesum,
                                  int root, int64_t N, double *__restrict__ consts) {
  for (int h = 0; h < H; ++h) {
    for (int idx = hoff[h] + threadIdx.x; idx < hoff[h + 1]; idx += blockDim.x) {
      int k = order[idx];
      int a = nl[k], b = nr[k];
      const double *va = a >= 0 ? leafsum + 3 * a : nodesum + 3 * (-a - 1);
      const double *vb = b >= 0 ? leafsum + 3 * b : nodesum + 3 * (-b - 1);
      nodesum[3 * k] = rn_add(va[0], vb[0]);
      nodesum[3 * k + 1] = rn_add(va[1], vb[1]);
      nodesum[3 * k + 2] = rn_add(va[2], vb[2]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double *v = root >= 0 ? leafsum + 3 * root : nodesum + 3 * (-root - 1);
    double dn = (double)N;
    double p0 = __ddiv_rn(v[0], dn), p1 = __ddiv_rn(v[1], dn), p2 = __ddiv_rn(v[2], dn);
    consts[0] = p0;
    consts[1] = p1;
    consts[2] = p2;
    consts[3] = 1.0;
    consts[4] = 1.0;
    consts[5] = __dsqrt_rn(rn_add(1.0, rn_add(rn_add(rn_mul(p0, p0), rn_mul(p1, p1)), rn_mul(p2, p2))));
  }
}

struct PwPlan {
  std::vector<int64_t> lf, ll;
  std::vector<int> nl, nr, h;
};

// Returns the reference (leaf index >= 0 or -(internal+1)) and its height.
int pw_build(PwPlan &P, int64_t first, int64_t last, int *height) {
  if (first == last || last - first < 1024) {
    P.lf.push_back(first);
    P.ll.push_back(last);
    *height = 0;
    return (int)P.lf.size() - 1;
  }
  int64_t mid = first + ((last - first) >> 1);
  int ha, hb;
  int a = pw_build(P, first, mid, &ha);
  int b = pw_build(P, mid + 1, last, &hb);
  P.nl.push_back(a);
  P.nr.push_back(b);
  int hh = (ha > hb ? ha : hb) + 1;
  P.h.push_back(hh);
  *height = hh;
  return -(int)P.nl.size();
}

// ---------------------------------------------------------------- tree levels
__device__ __forceinline__ int descend(int j, int l, int N, int *lo_out, int *hi_out) {
  int lo = 0, hi = N - 1, k = 0;
  for (int t = 0; t < l; ++t) {
    int mid = (lo + hi) >> 1;
    if (j <= mid) {
      hi = mid;
      k = 2 * k + 1;
    } else {
      lo = mid + 1;
      k = 2 * k + 2;
    }
  }
  *lo_out = lo;
  *hi_out = hi;
  return k;
}

__global__ void keys_kernel(const double *__restrict__ pos, int N, int axis, uint64_t *__restrict__ keys,
                            uint32_t *__restrict__ vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  keys[i] = double_key(pos[3 * (int64_t)i + axis]);
  vals[i] = (uint32_t)i;
}

// One thread per node of level l: bbox (+ extremal particle ids) from the ends
// of the three sorted segments; for l < ml the split axis, the left size and the
// children's ranges.
__global__ void node_kernel(int l, int ml, int N, const double *__restrict__ pos,
                            const uint32_t *__restrict__ lists, int *__restrict__ lohi,
                            const double *__restrict__ consts, double *__restrict__ bbox,
                            int *__restrict__ argext, int *__restrict__ split, int *__restrict__ half) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int cnt_level = 1 << l;
  if (idx >= cnt_level) return;
  int k = cnt_level - 1 + idx;
  int lo = lohi[2 * k], hi = lohi[2 * k + 1];
  double bmin[3], bmax[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    uint32_t pmin = lists[(int64_t)d * N + lo], pmax = lists[(int64_t)d * N + hi];
    bmin[d] = pos[3 * (int64_t)pmin + d];
    bmax[d] = pos[3 * (int64_t)pmax + d];
    bbox[6 * (int64_t)k + d] = bmin[d];
    bbox[6 * (int64_t)k + 3 + d] = bmax[d];
    argext[6 * (int64_t)k + d] = (int)pmin;
    argext[6 * (int64_t)k + 3 + d] = (int)pmax;
  }
  if (l < ml) {
    // splitdir = argmax(stretch .* (bbox[2] - bbox[1])), first maximum
    double v0 = rn_mul(consts[3], rn_sub(bmax[0], bmin[0]));
    double v1 = rn_mul(consts[4], rn_sub(bmax[1], bmin[1]));
    double v2 = rn_mul(consts[5], rn_sub(bmax[2], bmin[2]));
    int dir = 0;
    double best = v0;
    if (v1 > best) {
      best = v1;
      dir = 1;
    }
    if (v2 > best) dir = 2;
    int mid = (lo + hi) >> 1;
    split[k] = dir;
    half[k] = mid - lo + 1;
    int c1 = 2 * k + 1, c2 = 2 * k + 2;
    lohi[2 * c1] = lo;
    lohi[2 * c1 + 1] = mid;
    lohi[2 * c2] = mid + 1;
    lohi[2 * c2 + 1] = hi;
  }
}

// flag[p] = 1 if particle p goes to the left child of its level-l node.  Each thread takes
// kFlagItems positions blockDim apart and descends again only past its node's end (a node
// of a global level holds thousands of particles).
constexpr int kFlagItems = 4;
__global__ void flag_kernel(int l, int N, const uint32_t *__restrict__ lists, const int *__restrict__ split,
                            uint8_t *__restrict__ flag) {
  const int j0 = blockIdx.x * blockDim.x * kFlagItems + threadIdx.x;
  int lo = 0, hi = -1, k = 0;
#pragma unroll
  for (int i = 0; i < kFlagItems; ++i) {
    const int j = j0 + i * blockDim.x;
    if (j >= N) break;
    if (j > hi) k = descend(j, l, N, &lo, &hi);
    const uint32_t p = lists[(int64_t)split[k] * N + j];
    flag[p] = (j <= ((lo + hi) >> 1)) ? 1 : 0;
  }
}

constexpr int kPtThreads = 256;
constexpr int kPtItems = 8;
constexpr int kPtTile = kPtThreads * kPtItems;

// Left flags of the three lists in list order (fa[a][j]) and their per-tile
// counts.  In the list of the node's split axis the flag is j <= mid; the other
// two look the particle up in `flag` -- the level's only random reads.
// fa rows are fs bytes apart (fs: N rounded up to a multiple of 8).
__global__ void part_count_kernel(int l, int N, const uint32_t *__restrict__ lists, const uint8_t *__restrict__ flag,
                                  const int *__restrict__ split, int ntiles, int *__restrict__ tcount,
                                  uint8_t *__restrict__ fa, int64_t fs) {
  __shared__ int s_warp[33];
  const int j0 = blockIdx.x * kPtTile + threadIdx.x * kPtItems;
  int sp[kPtItems];
  uint8_t inl[kPtItems];  // j <= mid of its node
  int lo = 0, hi = -1, k = 0;  // the node of the last item; descend again past its end
  for (int i = 0; i < kPtItems; ++i) {
    const int j = j0 + i;
    sp[i] = -1;
    inl[i] = 0;
    if (j < N) {
      if (j > hi) k = descend(j, l, N, &lo, &hi);
      sp[i] = split[k];
      inl[i] = j <= ((lo + hi) >> 1) ? 1 : 0;
    }
  }
  for (int a = 0; a < 3; ++a) {
    int c = 0;
    uint8_t f[kPtItems];
    for (int i = 0; i < kPtItems; ++i) {
      const int j = j0 + i;
      f[i] = 0;
      if (j < N) f[i] = sp[i] == a ? inl[i] : flag[lists[(int64_t)a * N + j]];
      c += f[i];
    }
    if (j0 + kPtItems <= N) {  // 8 consecutive bytes, 8-byte aligned (j0 is a multiple of 8)
      uint64_t w = 0;
      for (int i = 0; i < kPtItems; ++i) w |= (uint64_t)f[i] << (8 * i);
      *reinterpret_cast<uint64_t *>(fa + a * fs + j0) = w;
    } else {
      for (int i = 0; i < kPtItems; ++i)
        if (j0 + i < N) fa[a * fs + j0 + i] = f[i];
    }
    int tot;
    block_excl_scan(c, s_warp, &tot);
    if (threadIdx.x == 0) tcount[a * ntiles + blockIdx.x] = tot;
  }
}

__global__ void part_scatter_kernel(int l, int N, const uint32_t *__restrict__ lists,
                                    const uint8_t *__restrict__ fa, int64_t fs, int ntiles, const int *__restrict__ toff,
                                    const int *__restrict__ nodebase, uint32_t *__restrict__ next,
                                    int *__restrict__ status) {
  __shared__ int s_warp[33];
  int j0 = blockIdx.x * kPtTile + threadIdx.x * kPtItems;
  int lo_[kPtItems], mid_[kPtItems], hi_[kPtItems], kk_[kPtItems];
  int lo = 0, hi = -1, k = 0;  // the node of the last item; descend again past its end
  for (int i = 0; i < kPtItems; ++i) {
    int j = j0 + i;
    if (j < N) {
      if (j > hi) k = descend(j, l, N, &lo, &hi);
      lo_[i] = lo;
      hi_[i] = hi;
      mid_[i] = (lo + hi) >> 1;
      kk_[i] = k - ((1 << l) - 1);
    } else {
      lo_[i] = mid_[i] = hi_[i] = kk_[i] = 0;
    }
  }
  for (int a = 0; a < 3; ++a) {
    uint32_t p[kPtItems];
    int f[kPtItems];
    int c = 0;
    for (int i = 0; i < kPtItems; ++i) {
      int j = j0 + i;
      if (j < N) {
        p[i] = lists[(int64_t)a * N + j];
        f[i] = fa[a * fs + j];
      } else {
        p[i] = 0;
        f[i] = 0;
      }
      c += f[i];
    }
    int ex = block_excl_scan(c, s_warp, nullptr);
    int P = toff[a * ntiles + blockIdx.x] - toff[a * ntiles] + ex;
    for (int i = 0; i < kPtItems; ++i) {
      int j = j0 + i;
      if (j < N) {
        int lb = P - nodebase[kk_[i]];  // left-flagged particles before j inside the node
        int dest = f[i] ? lo_[i] + lb : mid_[i] + 1 + ((j - lo_[i]) - lb);
        if (dest < lo_[i] || dest > hi_[i])  // stays inside the node by construction
          atomicExch(status, kDevBadIndex);
        else
          next[(int64_t)a * N + dest] = p[i];
      }
      P += f[i];
    }
  }
}

__global__ void leafof_kernel(int ml, int N, const uint32_t *__restrict__ list0, uint64_t *__restrict__ keys,
                              uint32_t *__restrict__ vals) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int lo, hi;
  int k = descend(j, ml, N, &lo, &hi);
  uint32_t p = list0[j];
  keys[p] = (uint64_t)(k - ((1 << ml) - 1));
  vals[p] = p;
}

__global__ void gather64_kernel(int N, const uint32_t *__restrict__ perm, const double *__restrict__ pos,
                                const double *__restrict__ mom, double *__restrict__ rec) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int64_t p = perm[j];
  double x = pos[3 * p], y = pos[3 * p + 1], z = pos[3 * p + 2];
  double ux = mom[3 * p], uy = mom[3 * p + 1], uz = mom[3 * p + 2];
  double g = sqrt(1.0 + (ux * ux + uy * uy + uz * uz));
  double2 *r = reinterpret_cast<double2 *>(rec + 8 * (int64_t)j);
  r[0] = make_double2(x, y);
  r[1] = make_double2(z, g);
  r[2] = make_double2(ux, uy);
  r[3] = make_double2(uz, 0.0);
}

// ---------------------------------------------------------------- bottom levels in shared memory
// One CTA per node of level L0 (at most kStCap particles) completes its subtree:
// the node's three sorted lists are loaded once and renamed to local 16-bit ids
// (one scatter and one gather through `lid`), then every remaining level reads
// its boxes off the segment ends, flags the split-axis halves and partitions the
// three lists stably with block scans -- the same steps, in the same order, as
// the global levels.  At the leaves the particle ids are written in ascending
// order (rank within the leaf), which replaces the final sort by leaf.
constexpr int kStCap = 4096;
constexpr int kStThreads = 256;
constexpr int kStItems = kStCap / kStThreads;
constexpr int kStMaxSub = 512;    // sub-nodes of one level that split (depth <= 9)
constexpr int kStSmem = 2 * 3 * kStCap * 2 + kStCap * 4 + 3 * kStCap * 2 + kStCap;

// Exclusive block-wide prefix sum of 64-bit values.  s_w: 33 words of shared memory; the
// caller orders any later reuse of s_w after a barrier.
__device__ __forceinline__ uint64_t block_excl_scan_u64(uint64_t v, uint64_t *s_w) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_w[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const uint64_t w = lane < nw ? s_w[lane] : 0ull;
    uint64_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < nw) s_w[lane] = wi - w;
  }
  __syncthreads();
  return s_w[wid] + inc - v;
}

// Range of sub-node s (left to right) `depth` levels below [lo0, hi0].
__device__ __forceinline__ void sub_range(int lo0, int hi0, int depth, int s, int *lo, int *hi) {
  int l = lo0, h = hi0;
  for (int t = depth - 1; t >= 0; --t) {
    const int mid = (l + h) >> 1;
    if ((s >> t) & 1)
      l = mid + 1;
    else
      h = mid;
  }
  *lo = l;
  *hi = h;
}

// Sub-node (and its range) `depth` levels below [lo0, hi0] that holds position p.
__device__ __forceinline__ int sub_of(int lo0, int hi0, int depth, int p, int *lo, int *hi) {
  int l = lo0, h = hi0, s = 0;
  for (int t = 0; t < depth; ++t) {
    const int mid = (l + h) >> 1;
    if (p <= mid) {
      h = mid;
      s = 2 * s;
    } else {
      l = mid + 1;
      s = 2 * s + 1;
    }
  }
  *lo = l;
  *hi = h;
  return s;
}

// 126 registers, two CTAs per SM.  A bound of three CTAs per SM (80 registers, a 16-byte
// spill) made the tree stage 0.2 ms slower at N = 2^24.
__global__ void __launch_bounds__(kStThreads)
    subtree_kernel(int L0, int ml, int N, const double *__restrict__ pos, const uint32_t *__restrict__ lists,
                   int *__restrict__ lohi, const double *__restrict__ consts, double *__restrict__ bbox,
                   int *__restrict__ argext, uint32_t *__restrict__ perm, int *__restrict__ lid,
                   int *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint16_t *Lbuf = (uint16_t *)smem;                             // [2][3][kStCap] local ids
  uint32_t *gid = (uint32_t *)(smem + 2 * 3 * kStCap * 2);       // local id -> particle id
  uint16_t *scan = (uint16_t *)(gid + kStCap);                   // [3][kStCap] left flags before each position
  uint8_t *flag = (uint8_t *)(scan + 3 * kStCap);                // left flag per local id
  __shared__ uint64_t s_warp64[33];
  __shared__ int s_split[kStMaxSub], s_mid[kStMaxSub];
  const int tid = threadIdx.x;
  const int k0 = (1 << L0) - 1 + blockIdx.x;
  const int lo0 = lohi[2 * k0], hi0 = lohi[2 * k0 + 1], cnt = hi0 - lo0 + 1;
  if (cnt < 1 || cnt > kStCap || ml - L0 > 10) {  // excluded by the host's choice of L0
    if (tid == 0) atomicExch(status, kDevBadIndex);
    return;
  }
  auto L = [&](int buf, int a) { return Lbuf + (buf * 3 + a) * kStCap; };
  for (int j = tid; j < cnt; j += kStThreads) {
    const uint32_t p = lists[lo0 + j];
    gid[j] = p;
    lid[p] = j;
  }
  __syncthreads();
  for (int j = tid; j < cnt; j += kStThreads) {
    L(0, 0)[j] = (uint16_t)j;
    L(0, 1)[j] = (uint16_t)lid[lists[(int64_t)N + lo0 + j]];
    L(0, 2)[j] = (uint16_t)lid[lists[2 * (int64_t)N + lo0 + j]];
  }
  __syncthreads();
  int cur = 0;
  for (int l = L0; l <= ml; ++l) {
    const int depth = l - L0, nsub = 1 << depth;
    for (int s = tid; s < nsub; s += kStThreads) {
      int lo, hi;
      sub_range(lo0, hi0, depth, s, &lo, &hi);
      const int64_t k = ((int64_t)1 << l) - 1 + (int64_t)blockIdx.x * nsub + s;
      lohi[2 * k] = lo;
      lohi[2 * k + 1] = hi;
      double bmin[3], bmax[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const uint32_t pmin = gid[L(cur, d)[lo - lo0]], pmax = gid[L(cur, d)[hi - lo0]];
        bmin[d] = pos[3 * (int64_t)pmin + d];
        bmax[d] = pos[3 * (int64_t)pmax + d];
        bbox[6 * k + d] = bmin[d];
        bbox[6 * k + 3 + d] = bmax[d];
        argext[6 * k + d] = (int)pmin;
        argext[6 * k + 3 + d] = (int)pmax;
      }
      if (l < ml) {
        // splitdir = argmax(stretch .* (bbox[2] - bbox[1])), first maximum
        const double v0 = rn_mul(consts[3], rn_sub(bmax[0], bmin[0]));
        const double v1 = rn_mul(consts[4], rn_sub(bmax[1], bmin[1]));
        const double v2 = rn_mul(consts[5], rn_sub(bmax[2], bmin[2]));
        int dir = 0;
        double best = v0;
        if (v1 > best) {
          best = v1;
          dir = 1;
        }
        if (v2 > best) dir = 2;
        s_split[s] = dir;
        s_mid[s] = (lo + hi) >> 1;
      }
    }
    __syncthreads();
    if (l == ml) break;
    // left flags: the first ceil(cnt/2) of each node's split-axis segment
    for (int p = tid; p < cnt; p += kStThreads) {
      int lo, hi;
      const int s = sub_of(lo0, hi0, depth, lo0 + p, &lo, &hi);
      flag[L(cur, s_split[s])[p]] = (lo0 + p <= s_mid[s]) ? 1 : 0;
    }
    __syncthreads();
    // the three lists' flags at this thread's positions as bit masks, their counts packed in
    // 16-bit fields (a node holds at most kStCap < 2^16), one block scan for all three
    const int b0 = tid * kStItems;
    uint32_t fm[3];
    uint64_t c = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      uint32_t m = 0;
#pragma unroll
      for (int i = 0; i < kStItems; ++i) {
        const int p = b0 + i;
        if (p < cnt && flag[L(cur, a)[p]]) m |= 1u << i;
      }
      fm[a] = m;
      c |= (uint64_t)__popc(m) << (16 * a);
    }
    const uint64_t ex = block_excl_scan_u64(c, s_warp64);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int run = (int)((ex >> (16 * a)) & 0xFFFFu);
#pragma unroll
      for (int i = 0; i < kStItems; ++i) {
        const int p = b0 + i;
        if (p < cnt) scan[a * kStCap + p] = (uint16_t)run;
        run += (fm[a] >> i) & 1u;
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kStItems; ++i) {
      const int p = b0 + i;
      if (p < cnt) {
        int lo, hi;
        const int s = sub_of(lo0, hi0, depth, lo0 + p, &lo, &hi);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int lb = (int)scan[a * kStCap + p] - (int)scan[a * kStCap + lo - lo0];  // left flags before p in its node
          const int dest = ((fm[a] >> i) & 1u) ? lo + lb : s_mid[s] + 1 + ((lo0 + p - lo) - lb);
          if (dest < lo || dest > hi)  // stays inside the node by construction
            atomicExch(status, kDevBadIndex);
          else
            L(cur ^ 1, a)[dest - lo0] = L(cur, a)[p];
        }
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  // leaves: particle ids in ascending order
  uint32_t *vals = (uint32_t *)scan;
  for (int p = tid; p < cnt; p += kStThreads) vals[p] = gid[L(cur, 0)[p]];
  __syncthreads();
  const int depth = ml - L0;
  for (int p = tid; p < cnt; p += kStThreads) {
    int lo, hi;
    sub_of(lo0, hi0, depth, lo0 + p, &lo, &hi);
    const uint32_t v = vals[p];
    int r = 0;
    for (int q = lo - lo0; q <= hi - lo0; ++q) r += vals[q] < v ? 1 : 0;
    perm[lo + r] = v;
  }
}

// ---------------------------------------------------------------- refit of an existing tree
// For a tree of the same N and N0 (same node ranges), new positions give the same
// tree exactly when every internal node still splits its particles the same way:
// with the boxes refitted bottom-up (exact min/max; the extremal particle is the
// first / last in (coordinate, id) order, as the sorted segment ends give it), the
// node's split axis argmax(stretch .* extent) must leave the left child's last
// particle before the right child's first in (coordinate, id) order.  Then the
// permutation, boxes and extremal particles equal what build_tree would compute.
__device__ __forceinline__ bool lex_less(double a, int ia, double b, int ib) {
  return a < b || (a == b && ia < ib);
}

__global__ void refit_leaf_kernel(int64_t leaf0, int64_t nleaf, const int *__restrict__ lohi,
                                  const uint32_t *__restrict__ perm, const double *__restrict__ pos,
                                  double *__restrict__ bbox, int *__restrict__ argext) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaf) return;
  const int64_t c = leaf0 + i;
  const int lo = lohi[2 * c], hi = lohi[2 * c + 1];
  double vmin[3], vmax[3];
  int imin[3], imax[3];
  {
    const int p = (int)perm[lo];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      vmin[d] = vmax[d] = pos[3 * (int64_t)p + d];
      imin[d] = imax[d] = p;
    }
  }
  for (int j = lo + 1; j <= hi; ++j) {
    const int p = (int)perm[j];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = pos[3 * (int64_t)p + d];
      if (lex_less(v, p, vmin[d], imin[d])) {
        vmin[d] = v;
        imin[d] = p;
      }
      if (lex_less(vmax[d], imax[d], v, p)) {
        vmax[d] = v;
        imax[d] = p;
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    bbox[6 * c + d] = vmin[d];
    bbox[6 * c + 3 + d] = vmax[d];
    argext[6 * c + d] = imin[d];
    argext[6 * c + 3 + d] = imax[d];
  }
}

__global__ void refit_up_kernel(int l, const double *__restrict__ consts, double *__restrict__ bbox,
                                int *__restrict__ argext, int *__restrict__ changed) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ((int64_t)1 << l)) return;
  const int64_t k = ((int64_t)1 << l) - 1 + idx, a = 2 * k + 1, b = 2 * k + 2;
  double lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const bool la = lex_less(bbox[6 * a + d], argext[6 * a + d], bbox[6 * b + d], argext[6 * b + d]);
    lo[d] = la ? bbox[6 * a + d] : bbox[6 * b + d];
    argext[6 * k + d] = la ? argext[6 * a + d] : argext[6 * b + d];
    const bool hb = lex_less(bbox[6 * a + 3 + d], argext[6 * a + 3 + d], bbox[6 * b + 3 + d], argext[6 * b + 3 + d]);
    hi[d] = hb ? bbox[6 * b + 3 + d] : bbox[6 * a + 3 + d];
    argext[6 * k + 3 + d] = hb ? argext[6 * b + 3 + d] : argext[6 * a + 3 + d];
    bbox[6 * k + d] = lo[d];
    bbox[6 * k + 3 + d] = hi[d];
  }
  // the split this node would get from the new positions (node_kernel's rule)
  const double v0 = rn_mul(consts[3], rn_sub(hi[0], lo[0]));
  const double v1 = rn_mul(consts[4], rn_sub(hi[1], lo[1]));
  const double v2 = rn_mul(consts[5], rn_sub(hi[2], lo[2]));
  int dir = 0;
  double best = v0;
  if (v1 > best) {
    best = v1;
    dir = 1;
  }
  if (v2 > best) dir = 2;
  if (!lex_less(bbox[6 * a + 3 + dir], argext[6 * a + 3 + dir], bbox[6 * b + dir], argext[6 * b + dir]))
    atomicOr(changed, 1);
}

// Leaf-local FP32 records: coordinates relative to the leaf's box centre.
__global__ void gather32_kernel(int ml, int N, const uint32_t *__restrict__ perm,
                                const double *__restrict__ pos, const double *__restrict__ mom,
                                const double *__restrict__ bbox, const int *__restrict__ leafpos,
                                float *__restrict__ rec, float4 *__restrict__ rec_x2) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int lo, hi;
  int k = leafpos ? leafpos[j] : descend(j, ml, N, &lo, &hi);
  const double *bb = bbox + 6 * (int64_t)k;
  int64_t p = perm[j];
  double cx = 0.5 * (bb[0] + bb[3]), cy = 0.5 * (bb[1] + bb[4]), cz = 0.5 * (bb[2] + bb[5]);
  double ux = mom[3 * p], uy = mom[3 * p + 1], uz = mom[3 * p + 2];
  double g = sqrt(1.0 + (ux * ux + uy * uy + uz * uz));
  const double lx = pos[3 * p] - cx, ly = pos[3 * p + 1] - cy, lz = pos[3 * p + 2] - cz;
  const float hx = (float)lx, hy = (float)ly, hz = (float)lz;
  float4 *r = reinterpret_cast<float4 *>(rec + 8 * (int64_t)j);
  r[0] = make_float4(hx, hy, hz, (float)g);
  r[1] = make_float4((float)ux, (float)uy, (float)uz, 0.0f);
  // The P2P source record: hi + lo parts of the local coordinates (hi + lo
  // reproduces the coordinate to ~2^-48 relative, and P2P forms the difference of
  // two nearby particles exactly from the hi parts, Sterbenz), negated, then
  // gamma and u; every value duplicated for packed FP32x2 arithmetic.
  const float nlx = -(float)(lx - (double)hx), nly = -(float)(ly - (double)hy), nlz = -(float)(lz - (double)hz);
  const float gf = (float)g, uxf = (float)ux, uyf = (float)uy, uzf = (float)uz;
  float4 *x2 = rec_x2 + 5 * (int64_t)j;
  x2[0] = make_float4(-hx, -hx, -hy, -hy);
  x2[1] = make_float4(-hz, -hz, nlx, nlx);
  x2[2] = make_float4(nly, nly, nlz, nlz);
  x2[3] = make_float4(gf, gf, uxf, uxf);
  x2[4] = make_float4(uyf, uyf, uzf, uzf);
}

// nodes[c][d][i] = a + (cos(pi*i/n) + 1)/2 * (b - a)  (barylg.jl:25-27, 0-based i)
__global__ void nodes_kernel(int64_t nc, int M, int NS, ChebT ct, const double *__restrict__ bbox,
                             double *__restrict__ nodes) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double *bb = bbox + 6 * c;
  double *o = nodes + c * NS;
  for (int d = 0; d < 3; ++d) {
    double a = bb[d], b = bb[3 + d];
    double w = rn_sub(b, a);
    for (int i = 0; i < M; ++i) o[d * M + i] = rn_add(a, rn_mul(ct.t[i], w));
  }
  for (int i = 3 * M; i < NS; ++i) o[i] = 0.0;
}

// admissible()/diameter() ingredients with the reference's operation order
// (interaction_lists.jl:10-21, bbox.jl:9-11).
__global__ void geom_kernel(int64_t nc, int64_t leaf0, const double *__restrict__ bbox,
                            const double *__restrict__ consts, ClusterGeom *__restrict__ geom) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double *bb = bbox + 6 * c;
  const double s0 = consts[3], s1 = consts[4], s2 = consts[5];
  ClusterGeom g;
  for (int d = 0; d < 3; ++d) g.xc[d] = __ddiv_rn(rn_add(bb[d], bb[3 + d]), 2.0);
  g.r = norm3_exact(rn_mul(s0, rn_sub(bb[3], g.xc[0])), rn_mul(s1, rn_sub(bb[4], g.xc[1])),
                    rn_mul(s2, rn_sub(bb[5], g.xc[2])));
  g.diam = norm3_exact(__ddiv_rn(rn_mul(s0, rn_sub(bb[3], bb[0])), 2.0), __ddiv_rn(rn_mul(s1, rn_sub(bb[4], bb[1])), 2.0),
                       __ddiv_rn(rn_mul(s2, rn_sub(bb[5], bb[2])), 2.0));
  g.leaf = c >= leaf0 ? 1 : 0;
  g.pad = 0;
  geom[c] = g;
}

}  // namespace

int node_stride(int n) {
  int s = 3 * (n + 1);
  return (s + 1) & ~1;  // even -> 16-byte aligned records
}

int compute_pavg_stretch(Ctx *ctx, const double *d_mom, int64_t N, double *d_consts) {
  if (ctx->pw_N != N) {
    PwPlan P;
    int h0 = 0;
    int root;
    if (N < 16) {
      P.lf.push_back(0);
      P.ll.push_back(N - 1);
      root = 0;
    } else {
      root = pw_build(P, 0, N - 1, &h0);
    }
    int nint = (int)P.nl.size();
    int H = 0;
    for (int i = 0; i < nint; ++i) H = P.h[i] > H ? P.h[i] : H;
    std::vector<int> order(nint), hoff(H + 1, 0), cnt(H + 1, 0);
    for (int i = 0; i < nint; ++i) cnt[P.h[i] - 1]++;
    for (int h = 0; h < H; ++h) hoff[h + 1] = hoff[h] + cnt[h];
    std::vector<int> fill(hoff.begin(), hoff.end());
    for (int i = 0; i < nint; ++i) order[fill[P.h[i] - 1]++] = i;
    int64_t *lf, *ll;
    int *nl, *nr, *ord, *dho;
    int nleaf = (int)P.lf.size();
    FMM_TRY(ctx->ensure("pw_lf", nleaf, &lf));
    FMM_TRY(ctx->ensure("pw_ll", nleaf, &ll));
    FMM_TRY(ctx->ensure("pw_nl", nint, &nl));
    FMM_TRY(ctx->ensure("pw_nr", nint, &nr));
    FMM_TRY(ctx->ensure("pw_order", nint, &ord));
    FMM_TRY(ctx->ensure("pw_hoff", H + 1, &dho));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(lf, P.lf.data(), sizeof(int64_t) * nleaf, cudaMemcpyHostToDevice, ctx->stream));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(ll, P.ll.data(), sizeof(int64_t) * nleaf, cudaMemcpyHostToDevice, ctx->stream));
    if (nint > 0) {
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(nl, P.nl.data(), sizeof(int) * nint, cudaMemcpyHostToDevice, ctx->stream));
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(nr, P.nr.data(), sizeof(int) * nint, cudaMemcpyHostToDevice, ctx->stream));
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(ord, order.data(), sizeof(int) * nint, cudaMemcpyHostToDevice, ctx->stream));
    }
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dho, hoff.data(), sizeof(int) * (H + 1), cudaMemcpyHostToDevice, ctx->stream));
    FMM_TRY(ctx->sync());  // host vectors go out of scope
    ctx->pw_N = N;
    ctx->pw_nleaf = nleaf;
    ctx->pw_nint = nint;
    ctx->pw_root = root;
    ctx->pw_hoff = hoff;
  }
  int nleaf = ctx->pw_nleaf, nint = ctx->pw_nint;
  double *leafsum, *nodesum;
  FMM_TRY(ctx->ensure("pw_leafsum", 3 * nleaf, &leafsum));
  FMM_TRY(ctx->ensure("pw_nodesum", 3 * (nint > 0 ? nint : 1), &nodesum));
  pw_leaf_kernel<<<ceil_div(nleaf, 128), 128, 0, ctx->stream>>>(d_mom, ctx->get<int64_t>("pw_lf"),
                                                                 ctx->get<int64_t>("pw_ll"), nleaf, leafsum);
  pw_combine_kernel<<<1, 1024, 0, ctx->stream>>>(ctx->get<int>("pw_nl"), ctx->get<int>("pw_nr"),
                                                  ctx->get<int>("pw_order"), ctx->get<int>("pw_hoff"),
                                                  (int)ctx->pw_hoff.size() - 1, leafsum, nodesum,
                                                  ctx->pw_root, N, d_consts);
  return ctx->check_launch("compute_pavg_stretch", 2);
}

int build_tree(Ctx *ctx, const double *d_pos, int64_t N64, int64_t N0, const double *d_consts,
               const std::function<int()> &after_sorts, int depth) {
  if (N64 > 0x7FFFFFFF) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "npar must be < 2^31");
  const int N = (int)N64;
  // tree shape (treeinfo.jl:6-26) with the reference's floating-point formula, unless the
  // depth is given (the subtree of a sharded beam has the whole tree's remaining depth)
  int ml = N > N0 ? (int)std::ceil(std::log((double)N / (double)N0) / std::log(2.0)) : 0;
  if (depth >= 0) ml = depth;
  if (ml > 29) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "tree depth > 29 (N0 too small for npar)");
  // every level-ml node must be a leaf and every node above must split
  int64_t maxc_ml = (N64 + ((int64_t)1 << ml) - 1) >> ml;
  int64_t minc_above = ml > 0 ? (N64 >> (ml - 1)) : N64 + N0 + 1;
  if (maxc_ml > N0 || minc_above <= N0)
    return ctx->fail(FMMB200_ERR_TREE_SHAPE,
                     "cluster tree would have a leaf above the maximum level (npar=" + std::to_string(N64) +
                         ", N0=" + std::to_string(N0) +
                         "); the reference leaves such nodes undefined (clusters.jl:36-48, treeinfo.jl:6-8)");
  const int64_t nc = ((int64_t)1 << (ml + 1)) - 1;
  const int64_t leaf0 = ((int64_t)1 << ml) - 1;
  ctx->have_tree = ctx->have_lists = ctx->have_forward = ctx->saved = false;

  uint64_t *kA, *kB;
  uint32_t *vA, *vB, *lists, *next, *perm;
  int *lohi, *argext, *split, *half, *nodebase, *tcount, *toff;
  double *bbox;
  uint8_t *flag;
  FMM_TRY(ctx->ensure("keysA", N, &kA));
  FMM_TRY(ctx->ensure("keysB", N, &kB));
  FMM_TRY(ctx->ensure("valsA", N, &vA));
  FMM_TRY(ctx->ensure("valsB", N, &vB));
  FMM_TRY(ctx->ensure("lists", 3 * (int64_t)N, &lists));
  FMM_TRY(ctx->ensure("lists_next", 3 * (int64_t)N, &next));
  FMM_TRY(ctx->ensure("perm", N, &perm));
  FMM_TRY(ctx->ensure("lohi", 2 * nc, &lohi));
  FMM_TRY(ctx->ensure("bbox", 6 * nc, &bbox));
  FMM_TRY(ctx->ensure("argext", 6 * nc, &argext));
  FMM_TRY(ctx->ensure("split", nc, &split));
  FMM_TRY(ctx->ensure("half", nc, &half));
  FMM_TRY(ctx->ensure("nodebase", nc, &nodebase));
  FMM_TRY(ctx->ensure("flag", N, &flag));
  uint8_t *fa;
  const int64_t fs = ((int64_t)N + 7) & ~(int64_t)7;  // 8-byte aligned rows for 8-byte stores
  FMM_TRY(ctx->ensure("flag3", 3 * fs, &fa));
  const int ntiles = ceil_div(N, kPtTile);
  FMM_TRY(ctx->ensure("tcount", 3 * (int64_t)ntiles, &tcount));
  FMM_TRY(ctx->ensure("toff", 3 * (int64_t)ntiles, &toff));

  const int TB = 256;
  // 1. three sorted coordinate orders
  for (int a = 0; a < 3; ++a) {
    keys_kernel<<<ceil_div(N, TB), TB, 0, ctx->stream>>>(d_pos, N, a, kA, vA);
    FMM_TRY(ctx->check_launch("keys_kernel"));
    bool alt = false;
    FMM_TRY(radix_sort(ctx, kA, kB, vA, vB, N, 64, &alt));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(lists + (int64_t)a * N, alt ? vB : vA, sizeof(uint32_t) * N,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (after_sorts) FMM_TRY(after_sorts());
  // 2. levels: globally down to L0, the first level whose nodes fit one CTA (and at
  // most 10 levels above the leaves), then each level-L0 subtree in shared memory
  int L0 = 0;
  while (L0 < ml && (((N64 + ((int64_t)1 << L0) - 1) >> L0) > kStCap || ml - L0 > 10)) ++L0;
  // leaves larger than one CTA (N0 > kStCap): every level globally, then the sort by leaf
  const bool subtree = ((N64 + ((int64_t)1 << L0) - 1) >> L0) <= kStCap;
  if (!subtree) L0 = ml + 1;
  int root[2] = {0, N - 1};
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(lohi, root, sizeof(root), cudaMemcpyHostToDevice, ctx->stream));
  for (int l = 0; l < L0; ++l) {
    const int cnt_level = 1 << l;
    node_kernel<<<ceil_div(cnt_level, TB), TB, 0, ctx->stream>>>(l, ml, N, d_pos, lists, lohi, d_consts, bbox,
                                                                  argext, split, half);
    FMM_TRY(ctx->check_launch("node_kernel"));
    if (l == ml) break;
    FMM_TRY(exclusive_scan_i32(ctx, half + (cnt_level - 1), nodebase, cnt_level, nullptr));
    flag_kernel<<<ceil_div(N, TB * kFlagItems), TB, 0, ctx->stream>>>(l, N, lists, split, flag);
    part_count_kernel<<<ntiles, kPtThreads, 0, ctx->stream>>>(l, N, lists, flag, split, ntiles, tcount, fa, fs);
    FMM_TRY(ctx->check_launch("flag/part_count kernels", 2));
    FMM_TRY(exclusive_scan_i32(ctx, tcount, toff, 3 * (int64_t)ntiles, nullptr));
    part_scatter_kernel<<<ntiles, kPtThreads, 0, ctx->stream>>>(l, N, lists, fa, fs, ntiles, toff, nodebase, next,
                                                                 ctx->d_status);
    FMM_TRY(ctx->check_launch("part_scatter_kernel"));
    uint32_t *t = lists;
    lists = next;
    next = t;
  }
  // the buffers may have swapped roles: keep names consistent for later stages
  if (lists != ctx->get<uint32_t>("lists")) std::swap(ctx->bufs["lists"], ctx->bufs["lists_next"]);
  // 3. levels L0 .. ml and the canonical order (particle ids ascending inside each leaf)
  if (subtree) {
    int *lid;
    FMM_TRY(ctx->ensure("tree_lid", N, &lid));
    FMM_TRY(opt_in_smem(ctx, subtree_kernel, kStSmem));
    subtree_kernel<<<1u << L0, kStThreads, kStSmem, ctx->stream>>>(L0, ml, N, d_pos, lists, lohi, d_consts, bbox,
                                                                    argext, perm, lid, ctx->d_status);
    FMM_TRY(ctx->check_launch("subtree_kernel"));
  } else {
    leafof_kernel<<<ceil_div(N, TB), TB, 0, ctx->stream>>>(ml, N, lists, kA, vA);
    FMM_TRY(ctx->check_launch("leafof_kernel"));
    bool alt = false;
    FMM_TRY(radix_sort(ctx, kA, kB, vA, vB, N, ml, &alt));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(perm, alt ? vB : vA, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
  }

  ctx->N = N;
  ctx->N0 = N0;
  ctx->ml = ml;
  ctx->nc = nc;
  ctx->nleaf = (int64_t)1 << ml;
  ctx->leaf0 = leaf0;
  ctx->max_leaf = (N64 + ((int64_t)1 << ml) - 1) >> ml;
  ctx->have_tree = true;
  return FMMB200_OK;
}

int refit_tree(Ctx *ctx, const double *d_pos, int64_t N, int64_t N0, const double *d_consts, bool *same) {
  *same = false;
  if (!ctx->have_tree || ctx->N != N || ctx->N0 != N0) return FMMB200_OK;
  const int ml = ctx->ml;
  int *changed, *h;
  FMM_TRY(ctx->ensure("refit_flag", 1, &changed));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(changed, 0, sizeof(int), ctx->stream));
  double *bbox = ctx->get<double>("bbox");
  int *argext = ctx->get<int>("argext");
  refit_leaf_kernel<<<ceil_div(ctx->nleaf, 128), 128, 0, ctx->stream>>>(
      ctx->leaf0, ctx->nleaf, ctx->get<int>("lohi"), ctx->get<uint32_t>("perm"), d_pos, bbox, argext);
  FMM_TRY(ctx->check_launch("refit_leaf_kernel"));
  for (int l = ml - 1; l >= 0; --l) {
    refit_up_kernel<<<ceil_div(1 << l, 256), 256, 0, ctx->stream>>>(l, d_consts, bbox, argext, changed);
    FMM_TRY(ctx->check_launch("refit_up_kernel"));
  }
  FMM_TRY(ctx->pinned(sizeof(int), (void **)&h));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h, changed, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  FMM_TRY(ctx->sync());
  *same = h[0] == 0;
  ctx->have_lists = ctx->have_forward = ctx->saved = false;
  return FMMB200_OK;
}

int gather_particles(Ctx *ctx, const double *d_pos, const double *d_mom, bool mixed, const int *leafpos) {
  const int N = (int)ctx->N;
  const int TB = 256;
  double *rec;
  FMM_TRY(ctx->ensure("prec64", 8 * (int64_t)N, &rec));
  gather64_kernel<<<ceil_div(N, TB), TB, 0, ctx->stream>>>(N, ctx->get<uint32_t>("perm"), d_pos, d_mom, rec);
  FMM_TRY(ctx->check_launch("gather64_kernel"));
  if (mixed) {
    float *r32;
    float4 *x2;
    FMM_TRY(ctx->ensure("prec32", 8 * (int64_t)N, &r32));
    FMM_TRY(ctx->ensure("prec32x2", 5 * (int64_t)N, &x2));
    gather32_kernel<<<ceil_div(N, TB), TB, 0, ctx->stream>>>(ctx->ml, N, ctx->get<uint32_t>("perm"), d_pos, d_mom,
                                                              ctx->get<double>("bbox"), leafpos, r32, x2);
    FMM_TRY(ctx->check_launch("gather32_kernel"));
  }
  return FMMB200_OK;
}

int compute_geom(Ctx *ctx, const double *d_consts) {
  ClusterGeom *geom;
  FMM_TRY(ctx->ensure("geom", ctx->nc, &geom));
  geom_kernel<<<ceil_div(ctx->nc, 256), 256, 0, ctx->stream>>>(ctx->nc, ctx->leaf0, ctx->get<double>("bbox"), d_consts,
                                                                geom);
  return ctx->check_launch("geom_kernel");
}

int compute_nodes(Ctx *ctx, int n) {
  const int M = n + 1, NS = node_stride(n);
  ChebT ct;
  for (int i = 0; i < kMaxNodes1D; ++i) ct.t[i] = 0.0;
  for (int i = 0; i < M; ++i) ct.t[i] = (std::cos(M_PI * (double)i / (double)n) + 1.0) / 2.0;
  double *nodes;
  FMM_TRY(ctx->ensure("nodes", (int64_t)NS * ctx->nc, &nodes));
  nodes_kernel<<<ceil_div(ctx->nc, 256), 256, 0, ctx->stream>>>(ctx->nc, M, NS, ct, ctx->get<double>("bbox"), nodes);
  return ctx->check_launch("nodes_kernel");
}

}  // namespace fmmb200
