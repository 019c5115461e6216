// api.cu -- the C-ABI of libfmmb200.so (declared in include/fmmb200.h).
//
// The forward pipeline mirrors update_particles_field!(particles, FMMGPU(...); lambda)
// (src/update_particles_field.jl:66-148) with every host step of the reference
// (tree build :82, interaction lists :113) moved onto the device:
//   p_avg/stretch -> tree -> tree-order records -> P2M -> M2M -> traversal ->
//   M2L -> P2P -> L2L -> L2P (+ near field, * amp, scatter to caller order).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_util.cuh"
#include "kernels.cuh"

using namespace fmmb200;

namespace {

constexpr int kEvStart = 0, kEvH2D = 1, kEvTree = 2, kEvUp = 3, kEvLists = 4, kEvM2L = 5, kEvP2P = 6,
              kEvDown = 7, kEvD2H = 8, kEvBwd0 = 9, kEvBwd1 = 10;

void mark(Ctx *ctx, int i) {
  if (!ctx->timing) return;
  if (!ctx->ev_ready) {
    for (auto &e : ctx->ev) cudaEventCreate(&e);
    ctx->ev_ready = true;
  }
  cudaEventRecord(ctx->ev[i], ctx->stream);
}

float ev_ms(Ctx *ctx, int a, int b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

__global__ void finite_check_kernel(const double *__restrict__ a, int64_t n, int *__restrict__ flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int bad = 0;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) bad |= !isfinite(a[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(flag, 1);
}

// Sharded forward (fmmb200_set_shard): heap cluster c at level l covers the leaves
// [(c + 1 - 2^l) 2^(ml - l), (c + 2 - 2^l) 2^(ml - l)); a shard keeps the M2L rows of
// the clusters whose leaves meet its own [lo, hi).  cnt has nc + 1 entries (the last 0).
__device__ __forceinline__ bool shard_owns(int64_t c, int ml, int64_t lo, int64_t hi) {
  const int l = 63 - __clzll((long long)(c + 1));
  const int64_t first = (c + 1 - (1ll << l)) << (ml - l), last = first + (1ll << (ml - l));
  return first < hi && last > lo;
}

__global__ void shard_rows_kernel(int64_t nc, int ml, int64_t lo, int64_t hi, const int *__restrict__ ptr,
                                  int *__restrict__ cnt) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c > nc) return;
  cnt[c] = (c < nc && shard_owns(c, ml, lo, hi)) ? ptr[c + 1] - ptr[c] : 0;
}

__global__ void shard_copy_kernel(int64_t nc, int ml, int64_t lo, int64_t hi, const int *__restrict__ ptr,
                                  const int *__restrict__ src, const int *__restrict__ ptr2, int *__restrict__ src2) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || !shard_owns(c, ml, lo, hi)) return;
  const int b = ptr[c], e = ptr[c + 1], o = ptr2[c];
  for (int k = b; k < e; ++k) src2[o + k - b] = src[k];
}

__global__ void iota_kernel(int first, int n, int *__restrict__ ids) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ids[i] = first + i;
}

__global__ void widen_kernel(const float *__restrict__ a, int64_t n, double *__restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

// stretch = (1, 1, sqrt(1 + p.p)) for a caller-given p_avg (update_particles_field.jl:46-47)
__global__ void stretch_kernel(double *__restrict__ consts) {
  const double p0 = consts[0], p1 = consts[1], p2 = consts[2];
  consts[3] = 1.0;
  consts[4] = 1.0;
  consts[5] = __dsqrt_rn(rn_add(1.0, rn_add(rn_add(rn_mul(p0, p0), rn_mul(p1, p1)), rn_mul(p2, p2))));
}

// out[3*perm[j] + q] += near[q*N + j]  (explicit stage entry points)
__global__ void scatter_add_kernel(int N, const uint32_t *__restrict__ perm, const double *__restrict__ near,
                                   double *__restrict__ oe, double *__restrict__ ob) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int64_t o = 3 * (int64_t)perm[j];
  for (int q = 0; q < 3; ++q) {
    oe[o + q] += near[(int64_t)q * N + j];
    ob[o + q] += near[(int64_t)(q + 3) * N + j];
  }
}

int check_common(Ctx *ctx, int64_t N, int n, int64_t N0, int precision) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (N < 1) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "npar must be >= 1");
  if (N > 0x7FFFFFFF) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "npar must be < 2^31");
  if (n < 1 || n > kMaxDegree) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "degree n must be in 1..10");
  if (N0 < 1) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "N0 must be >= 1");
  if (precision != FMMB200_PRECISION_FP64 && precision != FMMB200_PRECISION_MIXED)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "precision must be FMMB200_PRECISION_FP64 or _MIXED");
  return FMMB200_OK;
}

int ensure_expansions(Ctx *ctx, int n, bool mixed) {
  const int64_t NN = (int64_t)(n + 1) * (n + 1) * (n + 1);
  if (mixed) {
    float *m, *l;
    FMM_TRY(ctx->ensure("mom32", 4 * NN * ctx->nc, &m));
    FMM_TRY(ctx->ensure("loc32", 6 * NN * ctx->nc, &l));
  } else {
    double *m, *l;
    FMM_TRY(ctx->ensure("mom64", 4 * NN * ctx->nc, &m));
    FMM_TRY(ctx->ensure("loc64", 6 * NN * ctx->nc, &l));
  }
  double *nr;
  FMM_TRY(ctx->ensure("near", 6 * ctx->N, &nr));
  return FMMB200_OK;
}

// A shard's own leaves (ids) and its compacted M2L target lists, which the M2L
// launchers read until the keys are reset.
int prepare_shard(Ctx *ctx, const int **ids, int64_t *n_own) {
  const int64_t nl = ctx->nleaf, w = ctx->shard_world, r = ctx->shard_rank;
  const int64_t lo = nl * r / w, hi = nl * (r + 1) / w, nc = ctx->nc;
  int *d_ids, *cnt, *ptr2, *src2;
  FMM_TRY(ctx->ensure("shard_leaves", hi > lo ? hi - lo : 1, &d_ids));
  FMM_TRY(ctx->ensure("shard_cnt", nc + 1, &cnt));
  FMM_TRY(ctx->ensure("m2l_ptr_sh", nc + 1, &ptr2));
  FMM_TRY(ctx->ensure("m2l_src_sh", ctx->nm2l > 0 ? ctx->nm2l : 1, &src2));
  if (hi > lo) {
    iota_kernel<<<ceil_div(hi - lo, 256), 256, 0, ctx->stream>>>((int)(ctx->leaf0 + lo), (int)(hi - lo), d_ids);
    FMM_TRY(ctx->check_launch("iota_kernel"));
  }
  const int *ptr = ctx->get<int>("m2l_ptr"), *src = ctx->get<int>("m2l_src");
  shard_rows_kernel<<<ceil_div(nc + 1, 256), 256, 0, ctx->stream>>>(nc, ctx->ml, lo, hi, ptr, cnt);
  FMM_TRY(ctx->check_launch("shard_rows_kernel"));
  FMM_TRY(exclusive_scan_i32(ctx, cnt, ptr2, nc + 1, nullptr));
  shard_copy_kernel<<<ceil_div(nc, 256), 256, 0, ctx->stream>>>(nc, ctx->ml, lo, hi, ptr, src, ptr2, src2);
  FMM_TRY(ctx->check_launch("shard_copy_kernel"));
  ctx->m2l_ptr_key = "m2l_ptr_sh";
  ctx->m2l_src_key = "m2l_src_sh";
  *ids = d_ids;
  *n_own = hi - lo;
  return FMMB200_OK;
}

// The device forward.  d_pos/d_mom: AoS device arrays; d_E/d_B: AoS outputs.
// mom_ready (optional): an event after which d_mom holds the momenta; the work before
// it (finite check of the positions, the radix sorts of the tree build) reads only d_pos.
int run_forward(Ctx *ctx, int64_t N, const double *d_pos, const double *d_mom, double charge, double lambda, int n,
                int64_t N0, double eta, int precision, const double *pavg_host, bool save, double *d_E,
                double *d_B, cudaEvent_t mom_ready = nullptr) {
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  const int64_t launches0 = ctx->launches;
  const bool sharded = ctx->shard_world > 1;
  if (sharded && save)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "save_for_backward needs an unsharded forward (world 1)");
  ctx->m2l_ptr_key = "m2l_ptr";
  ctx->m2l_src_key = "m2l_src";
  double *consts;
  int *flag;
  FMM_TRY(ctx->ensure("consts", 8, &consts));
  FMM_TRY(ctx->ensure("finite_flag", 1, &flag));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
  finite_check_kernel<<<592, 256, 0, ctx->stream>>>(d_pos, 3 * N, flag);
  FMM_TRY(ctx->check_launch("finite_check_kernel"));
  // everything that reads the momenta: their finite check and p_avg / stretch
  bool mom_done = false;
  auto momentum_steps = [&]() -> int {
    if (mom_done) return FMMB200_OK;
    mom_done = true;
    if (mom_ready) FMM_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, mom_ready, 0));
    finite_check_kernel<<<592, 256, 0, ctx->stream>>>(d_mom, 3 * N, flag);
    FMM_TRY(ctx->check_launch("finite_check_kernel"));
    if (pavg_host) {
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync(consts, pavg_host, 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      stretch_kernel<<<1, 1, 0, ctx->stream>>>(consts);
      return ctx->check_launch("stretch_kernel");
    }
    return compute_pavg_stretch(ctx, d_mom, N, consts);
  };
  ctx->pavg_from_momenta = pavg_host == nullptr;
  bool reused = false;
  if (ctx->tree_reuse) {  // the refit checks the splits with the stretch
    FMM_TRY(momentum_steps());
    FMM_TRY(refit_tree(ctx, d_pos, N, N0, consts, &reused));
  }
  if (!reused) FMM_TRY(build_tree(ctx, d_pos, N, N0, consts, momentum_steps));
  FMM_TRY(momentum_steps());
  FMM_TRY(gather_particles(ctx, d_pos, d_mom, mixed));
  FMM_TRY(compute_nodes(ctx, n));
  ctx->n = n;
  ctx->precision = precision;
  ctx->eta = eta;
  ctx->charge = charge;
  ctx->lambda = lambda;
  FMM_TRY(ensure_expansions(ctx, n, mixed));
  mark(ctx, kEvTree);
  // upward pass (update_particles_field.jl:100-110)
  FMM_TRY(launch_p2m(ctx, n, mixed, nullptr, ctx->nleaf, false));
  for (int l = ctx->ml - 1; l >= 0; --l) FMM_TRY(launch_m2m(ctx, n, mixed, l, false));
  mark(ctx, kEvUp);
  // dual-tree traversal (:112-116, 123-125)
  FMM_TRY(build_lists(ctx, eta, consts));
  mark(ctx, kEvLists);
  // a shard: its own leaves and the M2L rows of the clusters above them
  const int *own = nullptr;
  int64_t n_own = ctx->nleaf;
  if (sharded) FMM_TRY(prepare_shard(ctx, &own, &n_own));
  // interactions (:118-128)
  const int m2l_st = launch_m2l(ctx, n, mixed, false);
  ctx->m2l_ptr_key = "m2l_ptr";
  ctx->m2l_src_key = "m2l_src";
  FMM_TRY(m2l_st);
  mark(ctx, kEvM2L);
  FMM_TRY(launch_p2p(ctx, mixed, own, n_own, false));
  mark(ctx, kEvP2P);
  // downward pass, amp and write-back (:130-147)
  for (int l = 1; l <= ctx->ml; ++l) FMM_TRY(launch_l2l(ctx, n, mixed, l));
  const double amp = kRe * charge / lambda;
  if (sharded) {  // the other shards' particles read 0
    FMM_CUDA_TRY(ctx, cudaMemsetAsync(d_E, 0, sizeof(double) * 3 * N, ctx->stream));
    FMM_CUDA_TRY(ctx, cudaMemsetAsync(d_B, 0, sizeof(double) * 3 * N, ctx->stream));
  }
  FMM_TRY(launch_l2p(ctx, n, mixed, own, n_own, 1, amp, d_E, d_B));
  mark(ctx, kEvDown);
  FMM_TRY(ctx->check_device_status("forward"));
  int *h;
  FMM_TRY(ctx->pinned(sizeof(int) * 8, (void **)&h));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  double *hc = (double *)(h + 2);
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(hc, consts, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  FMM_TRY(ctx->sync());
  if (h[0]) {
    ctx->have_forward = false;
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "positions and momenta must be finite");
  }
  for (int i = 0; i < 3; ++i) {
    ctx->pavg[i] = hc[i];
    ctx->stretch[i] = hc[3 + i];
  }
  ctx->have_forward = true;
  ctx->saved = save;
  // stats
  fmmb200_stats &st = ctx->stats;
  const double p2p_evals = st.p2p_kernel_evals;
  st = fmmb200_stats{};
  st.npar = N;
  st.n = n;
  st.N0 = N0;
  st.max_level = ctx->ml;
  st.ncluster = ctx->nc;
  st.nleaf = ctx->nleaf;
  st.nm2l = ctx->nm2l;
  st.np2p = ctx->np2p;
  st.traversal_steps = ctx->traversal_steps;
  st.device_bytes = (int64_t)ctx->device_bytes;
  for (int i = 0; i < 3; ++i) {
    st.pavg[i] = ctx->pavg[i];
    st.stretch[i] = ctx->stretch[i];
  }
  const double NN = (double)(n + 1) * (n + 1) * (n + 1);
  st.m2l_kernel_evals = (double)ctx->nm2l * NN * NN;
  st.kernel_launches = ctx->launches - launches0;
  st.tree_reused = reused ? 1 : 0;
  st.p2p_kernel_evals = p2p_evals;
  if (ctx->timing) {
    st.ms_tree = ev_ms(ctx, kEvH2D, kEvTree);
    st.ms_upward = ev_ms(ctx, kEvTree, kEvUp);
    st.ms_lists = ev_ms(ctx, kEvUp, kEvLists);
    st.ms_m2l = ev_ms(ctx, kEvLists, kEvM2L);
    st.ms_p2p = ev_ms(ctx, kEvM2L, kEvP2P);
    st.ms_downward = ev_ms(ctx, kEvP2P, kEvDown);
  }
  return FMMB200_OK;
}

struct Guard {
  Ctx *ctx;
  int prev = -1;
  explicit Guard(Ctx *c) : ctx(c) {
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
  }
  ~Guard() {
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  }
};

// ---- helpers for the explicit stage entry points ----------------------------

int upload(Ctx *ctx, const char *name, const void *h, size_t bytes, void **d) {
  FMM_TRY(ctx->ensure_bytes(name, bytes, d));
  if (bytes) FMM_CUDA_TRY(ctx, cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return FMMB200_OK;
}

// Julia-layout moments (gammas[NN*nc], mp_momenta[3*NN*nc]) <-> [Gamma|Mx|My|Mz] records
template <class T>
void mom_to_records(int64_t nc, int64_t NN, const double *g, const double *m, std::vector<T> &out) {
  out.assign((size_t)(4 * NN * nc), T(0));
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t a = 0; a < NN; ++a) {
      out[c * 4 * NN + a] = (T)(g ? g[NN * c + a] : 0.0);
      for (int q = 0; q < 3; ++q) out[c * 4 * NN + (1 + q) * NN + a] = (T)(m ? m[3 * (NN * c + a) + q] : 0.0);
    }
}
template <class T>
void records_to_mom(int64_t nc, int64_t NN, const std::vector<T> &rec, double *g, double *m) {
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t a = 0; a < NN; ++a) {
      if (g) g[NN * c + a] = (double)rec[c * 4 * NN + a];
      for (int q = 0; q < 3; ++q)
        if (m) m[3 * (NN * c + a) + q] = (double)rec[c * 4 * NN + (1 + q) * NN + a];
    }
}
// Julia-layout locals (efields/bfields [3*NN*nc]) <-> [Ex|Ey|Ez|Bx|By|Bz] records
template <class T>
void loc_to_records(int64_t nc, int64_t NN, const double *e, const double *b, std::vector<T> &out) {
  out.assign((size_t)(6 * NN * nc), T(0));
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t a = 0; a < NN; ++a)
      for (int q = 0; q < 3; ++q) {
        out[c * 6 * NN + q * NN + a] = (T)(e ? e[3 * (NN * c + a) + q] : 0.0);
        out[c * 6 * NN + (3 + q) * NN + a] = (T)(b ? b[3 * (NN * c + a) + q] : 0.0);
      }
}
template <class T>
void records_to_loc(int64_t nc, int64_t NN, const std::vector<T> &rec, double *e, double *b) {
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t a = 0; a < NN; ++a)
      for (int q = 0; q < 3; ++q) {
        if (e) e[3 * (NN * c + a) + q] = (double)rec[c * 6 * NN + q * NN + a];
        if (b) b[3 * (NN * c + a) + q] = (double)rec[c * 6 * NN + (3 + q) * NN + a];
      }
}

// Sets up an explicit cluster set (nc clusters with bboxes and optional ranges)
// in the context: lohi, bbox, nodes.  The stage kernels then run on it.
int setup_clusters(Ctx *ctx, int n, int64_t nc, const int64_t *parlohis, const double *bboxes) {
  if (nc < 1 || nc > 0x3FFFFFFF) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "nc out of range");
  ctx->have_tree = ctx->have_lists = ctx->have_forward = ctx->saved = false;
  ctx->nc = nc;
  ctx->leaf0 = 0;
  ctx->ml = 0;
  std::vector<int> lohi((size_t)(2 * nc), 0);
  if (parlohis)
    for (int64_t i = 0; i < 2 * nc; ++i) lohi[i] = (int)parlohis[i];
  void *d;
  FMM_TRY(upload(ctx, "lohi", lohi.data(), sizeof(int) * 2 * nc, &d));
  FMM_TRY(upload(ctx, "bbox", bboxes, sizeof(double) * 6 * nc, &d));
  FMM_TRY(compute_nodes(ctx, n));
  return ctx->sync();
}

// Particles in tree order from an explicit permutation; leafpos from ranges.
int setup_particles(Ctx *ctx, int64_t N, const double *pos, const double *mom, const int64_t *parindices,
                    int64_t nleaf, const int64_t *leaf_ids, const int64_t *parlohis, bool mixed) {
  std::vector<uint32_t> perm((size_t)N);
  for (int64_t j = 0; j < N; ++j) {
    if (parindices[j] < 0 || parindices[j] >= N) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "parindices out of range");
    perm[j] = (uint32_t)parindices[j];
  }
  std::vector<int> leafpos((size_t)N, 0);
  int64_t maxleaf = 1;
  for (int64_t l = 0; l < nleaf; ++l) {
    const int64_t c = leaf_ids[l];
    if (c < 0 || c >= ctx->nc) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "leaf id out of range");
    const int64_t lo = parlohis[2 * c], hi = parlohis[2 * c + 1];
    if (lo < 0 || hi >= N || hi < lo) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "bad parlohis range");
    for (int64_t j = lo; j <= hi; ++j) leafpos[j] = (int)c;
    maxleaf = hi - lo + 1 > maxleaf ? hi - lo + 1 : maxleaf;
  }
  ctx->N = N;
  ctx->max_leaf = maxleaf;
  void *d, *dp, *dm, *dl;
  FMM_TRY(upload(ctx, "perm", perm.data(), sizeof(uint32_t) * N, &d));
  FMM_TRY(upload(ctx, "in_pos", pos, sizeof(double) * 3 * N, &dp));
  FMM_TRY(upload(ctx, "in_mom", mom ? (const void *)mom : (const void *)pos, sizeof(double) * 3 * N, &dm));
  FMM_TRY(upload(ctx, "leafpos", leafpos.data(), sizeof(int) * N, &dl));
  if (!mom) FMM_CUDA_TRY(ctx, cudaMemsetAsync(dm, 0, sizeof(double) * 3 * N, ctx->stream));
  FMM_TRY(gather_particles(ctx, (const double *)dp, (const double *)dm, mixed, (const int *)dl));
  return ctx->sync();
}

int upload_ids(Ctx *ctx, int64_t cnt, const int64_t *ids, int **d) {
  std::vector<int> v((size_t)(cnt > 0 ? cnt : 1));
  for (int64_t i = 0; i < cnt; ++i) v[i] = (int)ids[i];
  return upload(ctx, "leaf_ids", v.data(), sizeof(int) * (cnt > 0 ? cnt : 1), (void **)d);
}

// Pair list -> sorted keys -> CSR (m2l_* or p2p_* buffers).
int setup_pairs(Ctx *ctx, const char *prefix, int64_t npairs, const int64_t *pairs) {
  int bits = 1;
  while (((int64_t)1 << bits) < ctx->nc) ++bits;
  std::vector<uint64_t> keys((size_t)(npairs > 0 ? npairs : 1));
  for (int64_t i = 0; i < npairs; ++i) {
    const int64_t t = pairs[2 * i], s = pairs[2 * i + 1];
    if (t < 0 || s < 0 || t >= ctx->nc || s >= ctx->nc) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "pair index out of range");
    keys[i] = ((uint64_t)t << bits) | (uint64_t)s;
  }
  std::sort(keys.begin(), keys.begin() + npairs);
  std::vector<int> ptr((size_t)ctx->nc + 1, 0), src((size_t)(npairs > 0 ? npairs : 1), 0);
  for (int64_t i = 0; i < npairs; ++i) {
    ptr[(keys[i] >> bits) + 1]++;
    src[i] = (int)(keys[i] & (((uint64_t)1 << bits) - 1));
  }
  for (int64_t c = 0; c < ctx->nc; ++c) ptr[c + 1] += ptr[c];
  std::string pn = std::string(prefix) + "_ptr", sn = std::string(prefix) + "_src";
  void *d;
  FMM_TRY(upload(ctx, pn.c_str(), ptr.data(), sizeof(int) * (ctx->nc + 1), &d));
  FMM_TRY(upload(ctx, sn.c_str(), src.data(), sizeof(int) * (npairs > 0 ? npairs : 1), &d));
  return ctx->sync();
}

int download_tree(Ctx *ctx, int64_t *parindices, int64_t *levels, int64_t *parlohis, int64_t *parents,
                  int64_t *children, double *bboxes) {
  const int64_t N = ctx->N, nc = ctx->nc;
  if (parindices) {
    std::vector<uint32_t> p((size_t)N);
    FMM_CUDA_TRY(ctx, cudaMemcpy(p.data(), ctx->get<uint32_t>("perm"), sizeof(uint32_t) * N, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < N; ++i) parindices[i] = p[i];
  }
  if (parlohis) {
    std::vector<int> v((size_t)(2 * nc));
    FMM_CUDA_TRY(ctx, cudaMemcpy(v.data(), ctx->get<int>("lohi"), sizeof(int) * 2 * nc, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < 2 * nc; ++i) parlohis[i] = v[i];
  }
  if (bboxes)
    FMM_CUDA_TRY(ctx, cudaMemcpy(bboxes, ctx->get<double>("bbox"), sizeof(double) * 6 * nc, cudaMemcpyDeviceToHost));
  for (int64_t k = 0; k < nc; ++k) {
    int lev = 0;
    while (((int64_t)2 << lev) - 1 <= k) ++lev;
    if (levels) levels[k] = lev;
    if (parents) parents[k] = (k + 1) / 2 - 1;
    if (children) {
      const bool leaf = k >= ctx->leaf0;
      children[2 * k] = leaf ? -1 : 2 * k + 1;
      children[2 * k + 1] = leaf ? -1 : 2 * k + 2;
    }
  }
  return FMMB200_OK;
}

}  // namespace

// ---- helpers of the per-rank steps of a sharded beam (shard.cu) ----------------
namespace fmmb200 {

int shard_check(Ctx *ctx, int64_t N, int n, int64_t N0, int precision) {
  return check_common(ctx, N, n, N0, precision);
}

int shard_consts(Ctx *ctx, const double *pavg_host, double **d_consts) {
  FMM_TRY(ctx->ensure("consts", 8, d_consts));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(*d_consts, pavg_host, 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  stretch_kernel<<<1, 1, 0, ctx->stream>>>(*d_consts);
  return ctx->check_launch("stretch_kernel");
}

int shard_expansions(Ctx *ctx, int n, bool mixed) { return ensure_expansions(ctx, n, mixed); }

}  // namespace fmmb200

// ============================================================================ exports
extern "C" {

int fmmb200_version(void) { return FMMB200_API_VERSION; }

int fmmb200_create(fmmb200_ctx **out, int device) {
  if (!out) return FMMB200_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return FMMB200_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return FMMB200_ERR_INVALID_ARGUMENT;
  Ctx *ctx = new Ctx();
  ctx->device = device;
  bool ok;
  {
    Guard g(ctx);
    ok = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&ctx->ev_copy[0], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&ctx->ev_copy[1], cudaEventDisableTiming) == cudaSuccess &&
         cudaMalloc(&ctx->d_status, sizeof(int)) == cudaSuccess &&
         cudaMemset(ctx->d_status, 0, sizeof(int)) == cudaSuccess;
    if (!ok) cudaGetLastError();
    ctx->stream = ctx->own_stream;
  }
  if (!ok) {  // releases whatever was created
    fmmb200_destroy(ctx);
    return FMMB200_ERR_CUDA;
  }
  *out = ctx;
  return FMMB200_OK;
}

int fmmb200_destroy(fmmb200_ctx *ctx) {
  if (!ctx) return FMMB200_OK;
  {
    Guard g(ctx);
    cudaStreamSynchronize(ctx->stream);
    for (auto &kv : ctx->bufs)
      if (kv.second.p) cudaFree(kv.second.p);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->ev_ready)
      for (auto &e : ctx->ev) cudaEventDestroy(e);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    for (auto &e : ctx->ev_copy)
      if (e) cudaEventDestroy(e);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  }
  delete ctx;
  return FMMB200_OK;
}

const char *fmmb200_last_error(const fmmb200_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fmmb200_set_stream(fmmb200_ctx *ctx, void *stream) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return FMMB200_OK;
}

int fmmb200_set_timing(fmmb200_ctx *ctx, int enable) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  ctx->timing = enable != 0;
  return FMMB200_OK;
}

int fmmb200_set_m2l_engine(fmmb200_ctx *ctx, int engine) {
  if (!ctx || engine < FMMB200_M2L_AUTO || engine > FMMB200_M2L_TENSOR_CORES) return FMMB200_ERR_INVALID_ARGUMENT;
  ctx->m2l_engine = engine;
  return FMMB200_OK;
}

int fmmb200_set_tree_reuse(fmmb200_ctx *ctx, int enable) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  ctx->tree_reuse = enable != 0;
  return FMMB200_OK;
}

int fmmb200_set_shard(fmmb200_ctx *ctx, int rank, int world) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (world < 1 || rank < 0 || rank >= world)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard: need 0 <= rank < world");
  ctx->shard_rank = rank;
  ctx->shard_world = world;
  return FMMB200_OK;
}

int fmmb200_debug_fail_alloc(fmmb200_ctx *ctx, int64_t k) {
  if (!ctx || k < 0) return FMMB200_ERR_INVALID_ARGUMENT;
  ctx->fail_alloc_countdown = k;
  return FMMB200_OK;
}

int fmmb200_forward_device(fmmb200_ctx *ctx, int64_t npar, const double *d_pos, const double *d_mom, double charge,
                           double lambda, int32_t n, int64_t N0, double eta, int32_t precision, const double *pavg,
                           int32_t save_for_backward, double *d_e, double *d_b) {
  FMM_TRY(check_common(ctx, npar, n, N0, precision));
  if (!d_pos || !d_mom || !d_e || !d_b) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (!(lambda != 0.0) || !std::isfinite(lambda) || !std::isfinite(charge) || std::isnan(eta))
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "lambda must be finite and nonzero; charge finite; eta not NaN");
  Guard g(ctx);
  mark(ctx, kEvStart);
  mark(ctx, kEvH2D);
  int s = run_forward(ctx, npar, d_pos, d_mom, charge, lambda, n, N0, eta, precision, pavg, save_for_backward != 0,
                      d_e, d_b);
  if (s == FMMB200_OK && ctx->timing) {
    mark(ctx, kEvD2H);
    ctx->sync();
    ctx->stats.ms_total = ev_ms(ctx, kEvStart, kEvD2H);
  }
  return s;
}

int fmmb200_forward(fmmb200_ctx *ctx, int64_t npar, const double *pos, const double *mom, double charge,
                    double lambda, int32_t n, int64_t N0, double eta, int32_t precision, const double *pavg,
                    int32_t save_for_backward, double *efields, double *bfields) {
  FMM_TRY(check_common(ctx, npar, n, N0, precision));
  if (!pos || !mom || !efields || !bfields) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (!(lambda != 0.0) || !std::isfinite(lambda) || !std::isfinite(charge) || std::isnan(eta))
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "lambda must be finite and nonzero; charge finite; eta not NaN");
  Guard g(ctx);
  double *dp, *dm, *de, *db;
  FMM_TRY(ctx->ensure("in_pos", 3 * npar, &dp));
  FMM_TRY(ctx->ensure("in_mom", 3 * npar, &dm));
  FMM_TRY(ctx->ensure("out_e", 3 * npar, &de));
  FMM_TRY(ctx->ensure("out_b", 3 * npar, &db));
  mark(ctx, kEvStart);
  // positions on the stream; momenta on the copy stream once the positions are in (the two
  // copies would otherwise share the link and delay the positions), overlapping the
  // position-only start of the tree build (finite check, radix sorts)
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dp, pos, sizeof(double) * 3 * npar, cudaMemcpyHostToDevice, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_copy[0], ctx->stream));
  FMM_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_copy[0], 0));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dm, mom, sizeof(double) * 3 * npar, cudaMemcpyHostToDevice, ctx->copy_stream));
  FMM_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_copy[1], ctx->copy_stream));
  mark(ctx, kEvH2D);
  const int fs = run_forward(ctx, npar, dp, dm, charge, lambda, n, N0, eta, precision, pavg, save_for_backward != 0,
                             de, db, ctx->ev_copy[1]);
  if (fs != FMMB200_OK) {  // the caller's buffers must outlive the copies in flight
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamSynchronize(ctx->stream);
    cudaGetLastError();
    return fs;
  }
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(efields, de, sizeof(double) * 3 * npar, cudaMemcpyDeviceToHost, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(bfields, db, sizeof(double) * 3 * npar, cudaMemcpyDeviceToHost, ctx->stream));
  mark(ctx, kEvD2H);
  FMM_TRY(ctx->sync());
  if (ctx->timing) {
    ctx->stats.ms_h2d = ev_ms(ctx, kEvStart, kEvH2D);
    ctx->stats.ms_d2h = ev_ms(ctx, kEvDown, kEvD2H);
    ctx->stats.ms_total = ev_ms(ctx, kEvStart, kEvD2H);
  }
  return FMMB200_OK;
}

int fmmb200_update_particles_field(fmmb200_ctx *ctx, int64_t npar, double charge, const double *positions,
                                   const double *momenta, double *efields, double *bfields, int32_t n, int64_t N0,
                                   double eta, double lambda, int32_t precision) {
  return fmmb200_forward(ctx, npar, positions, momenta, charge, lambda, n, N0, eta, precision, nullptr, 0, efields,
                         bfields);
}

int fmmb200_get_stats(const fmmb200_ctx *ctx, fmmb200_stats *out) {
  if (!ctx || !out) return FMMB200_ERR_INVALID_ARGUMENT;
  *out = ctx->stats;
  return FMMB200_OK;
}

int fmmb200_get_tree_info(const fmmb200_ctx *ctx, int64_t *info) {
  if (!ctx || !info) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_tree) return const_cast<Ctx *>(ctx)->fail(FMMB200_ERR_NO_STATE, "no tree in this context");
  info[0] = ctx->N;
  info[1] = ctx->N0;
  info[2] = ctx->ml;
  info[3] = ctx->nc;
  info[4] = ctx->have_lists ? ctx->nm2l : -1;
  info[5] = ctx->have_lists ? ctx->np2p : -1;
  info[6] = ctx->n;
  return FMMB200_OK;
}

int fmmb200_get_tree(fmmb200_ctx *ctx, int64_t *parindices, int64_t *levels, int64_t *parlohis, int64_t *parents,
                     int64_t *children, double *bboxes) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_tree) return ctx->fail(FMMB200_ERR_NO_STATE, "no tree in this context");
  Guard g(ctx);
  FMM_TRY(ctx->sync());
  return download_tree(ctx, parindices, levels, parlohis, parents, children, bboxes);
}

int fmmb200_get_lists(fmmb200_ctx *ctx, int64_t *m2l_pairs, int64_t *p2p_pairs) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_lists) return ctx->fail(FMMB200_ERR_NO_STATE, "no interaction lists in this context");
  Guard g(ctx);
  FMM_TRY(ctx->sync());
  const int bits = ctx->list_bits;
  const uint64_t mask = ((uint64_t)1 << bits) - 1;
  const char *names[2] = {"m2l_keys", "p2p_keys"};
  int64_t *outs[2] = {m2l_pairs, p2p_pairs};
  int64_t counts[2] = {ctx->nm2l, ctx->np2p};
  for (int w = 0; w < 2; ++w) {
    if (!outs[w] || counts[w] == 0) continue;
    std::vector<uint64_t> k((size_t)counts[w]);
    FMM_CUDA_TRY(ctx, cudaMemcpy(k.data(), ctx->get<uint64_t>(names[w]), sizeof(uint64_t) * counts[w],
                                 cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < counts[w]; ++i) {
      outs[w][2 * i] = (int64_t)(k[i] >> bits);
      outs[w][2 * i + 1] = (int64_t)(k[i] & mask);
    }
  }
  return FMMB200_OK;
}

int fmmb200_get_expansions(fmmb200_ctx *ctx, double *gammas, double *mp_momenta, double *mp_efields,
                           double *mp_bfields) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_forward) return ctx->fail(FMMB200_ERR_NO_STATE, "no forward state in this context");
  Guard g(ctx);
  FMM_TRY(ctx->sync());
  const int64_t NN = (int64_t)(ctx->n + 1) * (ctx->n + 1) * (ctx->n + 1), nc = ctx->nc;
  const bool mixed = ctx->precision == FMMB200_PRECISION_MIXED;
  if (gammas || mp_momenta) {
    if (mixed) {
      std::vector<float> r((size_t)(4 * NN * nc));
      FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), ctx->get<float>("mom32"), sizeof(float) * r.size(), cudaMemcpyDeviceToHost));
      records_to_mom(nc, NN, r, gammas, mp_momenta);
    } else {
      std::vector<double> r((size_t)(4 * NN * nc));
      FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), ctx->get<double>("mom64"), sizeof(double) * r.size(), cudaMemcpyDeviceToHost));
      records_to_mom(nc, NN, r, gammas, mp_momenta);
    }
  }
  if (mp_efields || mp_bfields) {
    if (mixed) {
      std::vector<float> r((size_t)(6 * NN * nc));
      FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), ctx->get<float>("loc32"), sizeof(float) * r.size(), cudaMemcpyDeviceToHost));
      records_to_loc(nc, NN, r, mp_efields, mp_bfields);
    } else {
      std::vector<double> r((size_t)(6 * NN * nc));
      FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), ctx->get<double>("loc64"), sizeof(double) * r.size(), cudaMemcpyDeviceToHost));
      records_to_loc(nc, NN, r, mp_efields, mp_bfields);
    }
  }
  return FMMB200_OK;
}

int fmmb200_cluster_tree(fmmb200_ctx *ctx, int64_t npar, const double *positions, int64_t N0, const double *stretch,
                         int64_t *parindices, int64_t *levels, int64_t *parlohis, int64_t *parents,
                         int64_t *children, double *bboxes) {
  FMM_TRY(check_common(ctx, npar, 1, N0, 0));
  if (!positions || !stretch) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  Guard g(ctx);
  double *dp, *consts;
  FMM_TRY(ctx->ensure("in_pos", 3 * npar, &dp));
  FMM_TRY(ctx->ensure("consts", 8, &consts));
  double c[8] = {0, 0, 0, stretch[0], stretch[1], stretch[2], 0, 0};
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dp, positions, sizeof(double) * 3 * npar, cudaMemcpyHostToDevice, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(consts, c, sizeof(c), cudaMemcpyHostToDevice, ctx->stream));
  FMM_TRY(build_tree(ctx, dp, npar, N0, consts));
  for (int i = 0; i < 3; ++i) ctx->stretch[i] = stretch[i];
  FMM_TRY(ctx->check_device_status("cluster_tree"));
  return download_tree(ctx, parindices, levels, parlohis, parents, children, bboxes);
}

int fmmb200_interaction_lists(fmmb200_ctx *ctx, const double *stretch, double eta, int64_t *counts) {
  if (!ctx || !stretch) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_tree) return ctx->fail(FMMB200_ERR_NO_STATE, "no tree in this context");
  Guard g(ctx);
  double *consts;
  FMM_TRY(ctx->ensure("consts", 8, &consts));
  double c[8] = {ctx->pavg[0], ctx->pavg[1], ctx->pavg[2], stretch[0], stretch[1], stretch[2], 0, 0};
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(consts, c, sizeof(c), cudaMemcpyHostToDevice, ctx->stream));
  FMM_TRY(build_lists(ctx, eta, consts));
  FMM_TRY(ctx->check_device_status("interaction_lists"));
  if (counts) {
    counts[0] = ctx->nm2l;
    counts[1] = ctx->np2p;
  }
  return FMMB200_OK;
}

int fmmb200_p2m(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t npar, const double *positions,
                const double *momenta, const int64_t *parindices, int64_t nc, const int64_t *parlohis,
                const double *bboxes, int64_t nleaf, const int64_t *leaf_ids, double *gammas, double *mp_momenta) {
  FMM_TRY(check_common(ctx, npar, n, 1, precision));
  if (!positions || !momenta || !parindices || !parlohis || !bboxes || !leaf_ids || !gammas || !mp_momenta)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  Guard g(ctx);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  const int64_t NN = (int64_t)(n + 1) * (n + 1) * (n + 1);
  FMM_TRY(setup_clusters(ctx, n, nc, parlohis, bboxes));
  FMM_TRY(setup_particles(ctx, npar, positions, momenta, parindices, nleaf, leaf_ids, parlohis, mixed));
  int *ids;
  FMM_TRY(upload_ids(ctx, nleaf, leaf_ids, &ids));
  void *d;
  if (mixed) {
    std::vector<float> r;
    mom_to_records(nc, NN, gammas, mp_momenta, r);
    FMM_TRY(upload(ctx, "mom32", r.data(), sizeof(float) * r.size(), &d));
    FMM_TRY(launch_p2m(ctx, n, true, ids, nleaf, true));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), d, sizeof(float) * r.size(), cudaMemcpyDeviceToHost));
    records_to_mom(nc, NN, r, gammas, mp_momenta);
  } else {
    std::vector<double> r;
    mom_to_records(nc, NN, gammas, mp_momenta, r);
    FMM_TRY(upload(ctx, "mom64", r.data(), sizeof(double) * r.size(), &d));
    FMM_TRY(launch_p2m(ctx, n, false, ids, nleaf, true));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), d, sizeof(double) * r.size(), cudaMemcpyDeviceToHost));
    records_to_mom(nc, NN, r, gammas, mp_momenta);
  }
  return ctx->check_device_status("p2m");
}

int fmmb200_m2m(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t nc, const int64_t *children,
                const double *bboxes, int64_t level, double *gammas, double *mp_momenta) {
  FMM_TRY(check_common(ctx, 1, n, 1, precision));
  if (!children || !bboxes || !gammas || !mp_momenta) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (level < 0 || level > 29 || (((int64_t)2 << (level + 1)) - 1) > nc)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "level out of range for nc clusters");
  for (int64_t p = ((int64_t)1 << level) - 1; p < ((int64_t)2 << level) - 1; ++p)
    if (children[2 * p] != 2 * p + 1 || children[2 * p + 1] != 2 * p + 2)
      return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "every parent at `level` must have heap children (2k+1, 2k+2)");
  Guard g(ctx);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  const int64_t NN = (int64_t)(n + 1) * (n + 1) * (n + 1);
  FMM_TRY(setup_clusters(ctx, n, nc, nullptr, bboxes));
  void *d;
  if (mixed) {
    std::vector<float> r;
    mom_to_records(nc, NN, gammas, mp_momenta, r);
    FMM_TRY(upload(ctx, "mom32", r.data(), sizeof(float) * r.size(), &d));
    FMM_TRY(launch_m2m(ctx, n, true, (int)level, true));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), d, sizeof(float) * r.size(), cudaMemcpyDeviceToHost));
    records_to_mom(nc, NN, r, gammas, mp_momenta);
  } else {
    std::vector<double> r;
    mom_to_records(nc, NN, gammas, mp_momenta, r);
    FMM_TRY(upload(ctx, "mom64", r.data(), sizeof(double) * r.size(), &d));
    FMM_TRY(launch_m2m(ctx, n, false, (int)level, true));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(r.data(), d, sizeof(double) * r.size(), cudaMemcpyDeviceToHost));
    records_to_mom(nc, NN, r, gammas, mp_momenta);
  }
  return FMMB200_OK;
}

int fmmb200_m2l(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t nc, const double *bboxes,
                const double *gammas, const double *mp_momenta, int64_t npairs, const int64_t *pairs,
                const double *pavg, double *mp_efields, double *mp_bfields) {
  FMM_TRY(check_common(ctx, 1, n, 1, precision));
  if (!bboxes || !gammas || !mp_momenta || (!pairs && npairs) || !pavg || !mp_efields || !mp_bfields)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  Guard g(ctx);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  const int64_t NN = (int64_t)(n + 1) * (n + 1) * (n + 1);
  FMM_TRY(setup_clusters(ctx, n, nc, nullptr, bboxes));
  FMM_TRY(setup_pairs(ctx, "m2l", npairs, pairs));
  ctx->eta = INFINITY;  // arbitrary pairs: target and source nodes may coincide
  double *consts;
  FMM_TRY(ctx->ensure("consts", 8, &consts));
  double c[8] = {pavg[0], pavg[1], pavg[2], 1, 1, 1, 0, 0};
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(consts, c, sizeof(c), cudaMemcpyHostToDevice, ctx->stream));
  void *dm, *dl;
  if (mixed) {
    std::vector<float> r, l;
    mom_to_records(nc, NN, gammas, mp_momenta, r);
    loc_to_records(nc, NN, mp_efields, mp_bfields, l);
    FMM_TRY(upload(ctx, "mom32", r.data(), sizeof(float) * r.size(), &dm));
    FMM_TRY(upload(ctx, "loc32", l.data(), sizeof(float) * l.size(), &dl));
    FMM_TRY(launch_m2l(ctx, n, true, true));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(l.data(), dl, sizeof(float) * l.size(), cudaMemcpyDeviceToHost));
    records_to_loc(nc, NN, l, mp_efields, mp_bfields);
  } else {
    std::vector<double> r, l;
    mom_to_records(nc, NN, gammas, mp_momenta, r);
    loc_to_records(nc, NN, mp_efields, mp_bfields, l);
    FMM_TRY(upload(ctx, "mom64", r.data(), sizeof(double) * r.size(), &dm));
    FMM_TRY(upload(ctx, "loc64", l.data(), sizeof(double) * l.size(), &dl));
    FMM_TRY(launch_m2l(ctx, n, false, true));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(l.data(), dl, sizeof(double) * l.size(), cudaMemcpyDeviceToHost));
    records_to_loc(nc, NN, l, mp_efields, mp_bfields);
  }
  return ctx->check_device_status("m2l");
}

int fmmb200_p2p(fmmb200_ctx *ctx, int32_t precision, int64_t npar, const double *positions, const double *momenta,
                const int64_t *parindices, int64_t nc, const int64_t *parlohis, const double *bboxes, int64_t npairs,
                const int64_t *pairs, double *efields, double *bfields) {
  FMM_TRY(check_common(ctx, npar, 1, 1, precision));
  if (!positions || !momenta || !parindices || !parlohis || !bboxes || (!pairs && npairs) || !efields || !bfields)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  Guard g(ctx);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  FMM_TRY(setup_clusters(ctx, 1, nc, parlohis, bboxes));
  // every target of a pair is treated as a leaf
  std::vector<int64_t> tl;
  {
    std::vector<char> seen((size_t)nc, 0);
    for (int64_t i = 0; i < npairs; ++i) {
      const int64_t t = pairs[2 * i], s = pairs[2 * i + 1];
      if (t < 0 || t >= nc || s < 0 || s >= nc) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "pair index out of range");
      if (!seen[t]) tl.push_back(t);
      seen[t] = 1;
      if (!seen[s]) tl.push_back(s);  // sources need leaf-local records too
      seen[s] = 1;
    }
  }
  FMM_TRY(setup_particles(ctx, npar, positions, momenta, parindices, (int64_t)tl.size(), tl.data(), parlohis, mixed));
  FMM_TRY(setup_pairs(ctx, "p2p", npairs, pairs));
  int *ids;
  FMM_TRY(upload_ids(ctx, (int64_t)tl.size(), tl.data(), &ids));
  double *near, *de, *db;
  FMM_TRY(ctx->ensure("near", 6 * npar, &near));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(near, 0, sizeof(double) * 6 * npar, ctx->stream));
  FMM_TRY(launch_p2p(ctx, mixed, ids, (int64_t)tl.size(), false));
  FMM_TRY(upload(ctx, "out_e", efields, sizeof(double) * 3 * npar, (void **)&de));
  FMM_TRY(upload(ctx, "out_b", bfields, sizeof(double) * 3 * npar, (void **)&db));
  scatter_add_kernel<<<ceil_div(npar, 256), 256, 0, ctx->stream>>>((int)npar, ctx->get<uint32_t>("perm"), near, de, db);
  FMM_TRY(ctx->check_launch("scatter_add_kernel"));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(efields, de, sizeof(double) * 3 * npar, cudaMemcpyDeviceToHost, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(bfields, db, sizeof(double) * 3 * npar, cudaMemcpyDeviceToHost, ctx->stream));
  FMM_TRY(ctx->sync());
  return ctx->check_device_status("p2p");
}

int fmmb200_l2l(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t nc, const int64_t *parents,
                const double *bboxes, int64_t level, double *mp_efields, double *mp_bfields) {
  FMM_TRY(check_common(ctx, 1, n, 1, precision));
  if (!parents || !bboxes || !mp_efields || !mp_bfields) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (level < 1 || level > 29 || (((int64_t)2 << level) - 1) > nc)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "level out of range for nc clusters");
  for (int64_t c = ((int64_t)1 << level) - 1; c < ((int64_t)2 << level) - 1; ++c)
    if (parents[c] != (c + 1) / 2 - 1) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "parents must be heap parents");
  Guard g(ctx);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  const int64_t NN = (int64_t)(n + 1) * (n + 1) * (n + 1);
  FMM_TRY(setup_clusters(ctx, n, nc, nullptr, bboxes));
  void *dl;
  if (mixed) {
    std::vector<float> l;
    loc_to_records(nc, NN, mp_efields, mp_bfields, l);
    FMM_TRY(upload(ctx, "loc32", l.data(), sizeof(float) * l.size(), &dl));
    FMM_TRY(launch_l2l(ctx, n, true, (int)level));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(l.data(), dl, sizeof(float) * l.size(), cudaMemcpyDeviceToHost));
    records_to_loc(nc, NN, l, mp_efields, mp_bfields);
  } else {
    std::vector<double> l;
    loc_to_records(nc, NN, mp_efields, mp_bfields, l);
    FMM_TRY(upload(ctx, "loc64", l.data(), sizeof(double) * l.size(), &dl));
    FMM_TRY(launch_l2l(ctx, n, false, (int)level));
    FMM_TRY(ctx->sync());
    FMM_CUDA_TRY(ctx, cudaMemcpy(l.data(), dl, sizeof(double) * l.size(), cudaMemcpyDeviceToHost));
    records_to_loc(nc, NN, l, mp_efields, mp_bfields);
  }
  return FMMB200_OK;
}

int fmmb200_l2p(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t npar, const double *positions,
                const int64_t *parindices, int64_t nc, const int64_t *parlohis, const double *bboxes, int64_t nleaf,
                const int64_t *leaf_ids, const double *mp_efields, const double *mp_bfields, double *efields,
                double *bfields) {
  FMM_TRY(check_common(ctx, npar, n, 1, precision));
  if (!positions || !parindices || !parlohis || !bboxes || !leaf_ids || !mp_efields || !mp_bfields || !efields || !bfields)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  Guard g(ctx);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  const int64_t NN = (int64_t)(n + 1) * (n + 1) * (n + 1);
  FMM_TRY(setup_clusters(ctx, n, nc, parlohis, bboxes));
  FMM_TRY(setup_particles(ctx, npar, positions, nullptr, parindices, nleaf, leaf_ids, parlohis, mixed));
  int *ids;
  FMM_TRY(upload_ids(ctx, nleaf, leaf_ids, &ids));
  void *dl;
  if (mixed) {
    std::vector<float> l;
    loc_to_records(nc, NN, mp_efields, mp_bfields, l);
    FMM_TRY(upload(ctx, "loc32", l.data(), sizeof(float) * l.size(), &dl));
  } else {
    std::vector<double> l;
    loc_to_records(nc, NN, mp_efields, mp_bfields, l);
    FMM_TRY(upload(ctx, "loc64", l.data(), sizeof(double) * l.size(), &dl));
  }
  double *near, *de, *db;
  FMM_TRY(ctx->ensure("near", 6 * npar, &near));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(near, 0, sizeof(double) * 6 * npar, ctx->stream));
  FMM_TRY(launch_l2p(ctx, n, mixed, ids, nleaf, 0, 1.0, nullptr, nullptr));
  FMM_TRY(upload(ctx, "out_e", efields, sizeof(double) * 3 * npar, (void **)&de));
  FMM_TRY(upload(ctx, "out_b", bfields, sizeof(double) * 3 * npar, (void **)&db));
  scatter_add_kernel<<<ceil_div(npar, 256), 256, 0, ctx->stream>>>((int)npar, ctx->get<uint32_t>("perm"), near, de, db);
  FMM_TRY(ctx->check_launch("scatter_add_kernel"));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(efields, de, sizeof(double) * 3 * npar, cudaMemcpyDeviceToHost, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(bfields, db, sizeof(double) * 3 * npar, cudaMemcpyDeviceToHost, ctx->stream));
  return ctx->sync();
}

int fmmb200_backward_device(fmmb200_ctx *ctx, const double *d_ge, const double *d_gb, double *d_gx,
                            double *d_gu) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->saved || !ctx->have_forward)
    return ctx->fail(FMMB200_ERR_NO_STATE, "no forward saved for backward (call forward with save_for_backward=1)");
  if (!d_ge || !d_gb || !d_gx || !d_gu) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  Guard g(ctx);
  mark(ctx, kEvBwd0);
  if (ctx->precision == FMMB200_PRECISION_MIXED) {
    // the adjoint runs in FP64 on the saved FP32 expansions
    const int64_t NN = (int64_t)(ctx->n + 1) * (ctx->n + 1) * (ctx->n + 1);
    double *m64, *l64;
    FMM_TRY(ctx->ensure("mom64", 4 * NN * ctx->nc, &m64));
    FMM_TRY(ctx->ensure("loc64", 6 * NN * ctx->nc, &l64));
    widen_kernel<<<592, 256, 0, ctx->stream>>>(ctx->get<float>("mom32"), 4 * NN * ctx->nc, m64);
    widen_kernel<<<592, 256, 0, ctx->stream>>>(ctx->get<float>("loc32"), 6 * NN * ctx->nc, l64);
    FMM_TRY(ctx->check_launch("widen_kernel", 2));
  }
  FMM_TRY(build_union_lists(ctx));
  FMM_TRY(run_backward(ctx, d_ge, d_gb, d_gx, d_gu));
  mark(ctx, kEvBwd1);
  FMM_TRY(ctx->check_device_status("backward"));
  if (ctx->timing) ctx->stats.ms_backward = ev_ms(ctx, kEvBwd0, kEvBwd1);
  return FMMB200_OK;
}

int fmmb200_backward(fmmb200_ctx *ctx, const double *ge, const double *gb, double *gx, double *gu) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ge || !gb || !gx || !gu) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (!ctx->saved || !ctx->have_forward)
    return ctx->fail(FMMB200_ERR_NO_STATE, "no forward saved for backward (call forward with save_for_backward=1)");
  Guard g(ctx);
  const int64_t N = ctx->N;
  double *dge, *dgb, *dgx, *dgu;
  FMM_TRY(ctx->ensure("bwd_in_ge", 3 * N, &dge));
  FMM_TRY(ctx->ensure("bwd_in_gb", 3 * N, &dgb));
  FMM_TRY(ctx->ensure("bwd_out_gx", 3 * N, &dgx));
  FMM_TRY(ctx->ensure("bwd_out_gu", 3 * N, &dgu));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dge, ge, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(dgb, gb, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, ctx->stream));
  FMM_TRY(fmmb200_backward_device(ctx, dge, dgb, dgx, dgu));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(gx, dgx, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, ctx->stream));
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(gu, dgu, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, ctx->stream));
  return ctx->sync();
}

}  // extern "C"
