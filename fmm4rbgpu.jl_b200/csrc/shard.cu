// shard.cu -- the per-rank steps of one beam spread over several GPUs with each rank
// holding only its part of the tree (no counterpart in the reference, whose FMMGPU runs
// the whole beam on one device, src/update_particles_field.jl:66-148).
//
// The caller (fmmb200/sharded.py) splits the beam's tree at level L = log2(ranks): the
// first L levels are partitioned across the ranks, and rank r then owns the subtree of
// the level-L cluster g = 2^L - 1 + r.  Per rank:
//   fmmb200_shard_subtree   builds g's subtree from g's particles (the whole tree's
//                           remaining depth, the given p_avg) and runs P2M and M2M on it
//   fmmb200_shard_boxes     its clusters' boxes, which the ranks all-gather
//   fmmb200_shard_lists     the traversal of the whole tree from the all-gathered boxes,
//                           keeping only the rows of g's subtree and of g's ancestors
//   fmmb200_shard_pack      moments of its clusters and particle records of its leaves
//                           that other ranks asked for
//   fmmb200_shard_evaluate  everything else for its own particles, with the top of the
//                           tree, the remote clusters and the halo particles appended
//                           after its own clusters and particles
// Every kernel is the one of the single-GPU forward, on the same data in the same
// order, so the fields equal the single-GPU forward's (given the same p_avg) bit for bit.
#include "device_util.cuh"
#include "kernels.cuh"

using namespace fmmb200;

namespace {

// out[k] = rec[ids[k]], records of w 16-byte words
__global__ void pack_records_kernel(int64_t count, const int *__restrict__ ids, int w, const uint4 *__restrict__ rec,
                                    uint4 *__restrict__ out, int64_t nrec, int *__restrict__ status) {
  const int64_t k = blockIdx.x;
  if (k >= count) return;
  const int c = ids[k];
  if (c < 0 || c >= nrec) {
    if (threadIdx.x == 0) atomicCAS(status, kDevOk, kDevBadIndex);
    return;
  }
  for (int e = threadIdx.x; e < w; e += blockDim.x) out[k * w + e] = rec[(int64_t)c * w + e];
}

// Particle records of leaf ids[k] (range lohi) to out from record offs[k] on.
__global__ void pack_leaves_kernel(int64_t count, const int *__restrict__ ids, const int64_t *__restrict__ offs,
                                   const int *__restrict__ lohi, int w, const uint4 *__restrict__ rec,
                                   uint4 *__restrict__ out, int64_t nc, int64_t nrec, int *__restrict__ status) {
  const int64_t k = blockIdx.x;
  if (k >= count) return;
  const int c = ids[k];
  if (c < 0 || c >= nc) {
    if (threadIdx.x == 0) atomicCAS(status, kDevOk, kDevBadIndex);
    return;
  }
  const int lo = lohi[2 * c], hi = lohi[2 * c + 1];
  if (lo < 0 || hi >= nrec) {
    if (threadIdx.x == 0) atomicCAS(status, kDevOk, kDevBadIndex);
    return;
  }
  const int64_t o = offs[k];
  for (int64_t e = threadIdx.x; e < (int64_t)(hi - lo + 1) * w; e += blockDim.x) out[o * w + e] = rec[(int64_t)lo * w + e];
}

// lohi of the appended clusters: halo ranges shifted past the own particles; an empty
// range (hi < lo) stays empty.
__global__ void lohi_ext_kernel(int64_t next, const int *__restrict__ ext, int shift, int64_t nhalo,
                                int *__restrict__ out, int *__restrict__ status) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= next) return;
  int lo = ext[2 * k], hi = ext[2 * k + 1];
  if (hi >= lo && (lo < 0 || hi >= nhalo)) {
    atomicCAS(status, kDevOk, kDevBadIndex);
    lo = 0;
    hi = -1;
  }
  if (hi < lo) {
    lo = 0;
    hi = -1;
  } else {
    lo += shift;
    hi += shift;
  }
  out[2 * k] = lo;
  out[2 * k + 1] = hi;
}

// Caller-made CSR lists over nc clusters: ptr[0] = 0, rows non-decreasing, ptr[nc] =
// nnz, every source in [0, nc); P2P sources (check_ranges) hold a particle range inside
// the nrec records.  Any violation sets *bad (the lists are then not used).
__global__ void validate_csr_kernel(int64_t nc, const int *__restrict__ ptr, const int *__restrict__ src, int64_t nnz,
                                    const int *__restrict__ lohi, int check_ranges, int64_t nrec,
                                    int *__restrict__ bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 == 0 && (ptr[0] != 0 || ptr[nc] != nnz)) atomicExch(bad, 1);
  for (int64_t c = i0; c < nc; c += stride)
    if (ptr[c + 1] < ptr[c]) atomicExch(bad, 1);
  for (int64_t k = i0; k < nnz; k += stride) {
    const int s = src[k];
    if (s < 0 || s >= nc) {
      atomicExch(bad, 1);
    } else if (check_ranges) {
      const int lo = lohi[2 * s], hi = lohi[2 * s + 1];
      if (lo < 0 || hi < lo || hi >= nrec) atomicExch(bad, 1);
    }
  }
}

// Buffer `name` grown to `keep + add` bytes with its first `keep` bytes kept and `add`
// bytes from `src` appended (src null: zeros).  Grown in place when its capacity allows,
// which it does from the second call on (the growth leaves headroom).
int extend_buffer(Ctx *ctx, const char *name, size_t keep, const void *src, size_t add) {
  void *p = nullptr;
  FMM_TRY(grow_keep(ctx, name, keep, keep + add, &p));
  if (add) {
    if (src)
      FMM_CUDA_TRY(ctx, cudaMemcpyAsync((char *)p + keep, src, add, cudaMemcpyDeviceToDevice, ctx->stream));
    else
      FMM_CUDA_TRY(ctx, cudaMemsetAsync((char *)p + keep, 0, add, ctx->stream));
  }
  return FMMB200_OK;
}

int copy_in(Ctx *ctx, const char *name, const void *src, size_t bytes) {
  void *d = nullptr;
  FMM_TRY(ctx->ensure_bytes(name, bytes, &d));
  if (bytes && src) FMM_CUDA_TRY(ctx, cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  return FMMB200_OK;
}

size_t moment_bytes(int n, bool mixed) {
  const size_t NN = (size_t)(n + 1) * (n + 1) * (n + 1);
  return 4 * NN * (mixed ? sizeof(float) : sizeof(double));
}
size_t particle_bytes(bool mixed) { return mixed ? 80 : 64; }

struct Guard {
  int prev = -1;
  explicit Guard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
    else prev = -1;
  }
  ~Guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

int fmmb200_shard_record_bytes(int32_t n, int32_t precision, int64_t *moment_record, int64_t *particle_record) {
  if (n < 1 || n > kMaxDegree || (precision != FMMB200_PRECISION_FP64 && precision != FMMB200_PRECISION_MIXED))
    return FMMB200_ERR_INVALID_ARGUMENT;
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  if (moment_record) *moment_record = (int64_t)moment_bytes(n, mixed);
  if (particle_record) *particle_record = (int64_t)particle_bytes(mixed);
  return FMMB200_OK;
}

int fmmb200_shard_subtree(fmmb200_ctx *ctx, int64_t npar, const double *d_positions, const double *d_momenta,
                          int64_t N0, int32_t depth, const double *pavg, int32_t n, int32_t precision) {
  FMM_TRY(shard_check(ctx, npar, n, N0, precision));
  if (!d_positions || !d_momenta || !pavg) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_subtree: null pointer");
  if (depth < 0 || depth > 29) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_subtree: depth must be in 0..29");
  Guard g(ctx->device);
  const bool mixed = precision == FMMB200_PRECISION_MIXED;
  ctx->shard_rank = 0;
  ctx->shard_world = 1;
  double *consts;
  FMM_TRY(shard_consts(ctx, pavg, &consts));
  ctx->pavg_from_momenta = false;
  FMM_TRY(build_tree(ctx, d_positions, npar, N0, consts, {}, depth));
  FMM_TRY(gather_particles(ctx, d_positions, d_momenta, mixed));
  FMM_TRY(compute_nodes(ctx, n));
  ctx->n = n;
  ctx->precision = precision;
  FMM_TRY(shard_expansions(ctx, n, mixed));
  FMM_TRY(launch_p2m(ctx, n, mixed, nullptr, ctx->nleaf, false));
  for (int l = ctx->ml - 1; l >= 0; --l) FMM_TRY(launch_m2m(ctx, n, mixed, l, false));
  FMM_TRY(ctx->check_device_status("shard_subtree"));
  ctx->have_forward = false;
  ctx->saved = false;
  return FMMB200_OK;
}

int fmmb200_shard_boxes(fmmb200_ctx *ctx, double *d_bboxes) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_tree) return ctx->fail(FMMB200_ERR_NO_STATE, "shard_boxes: no subtree");
  if (!d_bboxes) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_boxes: null pointer");
  Guard g(ctx->device);
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(d_bboxes, ctx->get<double>("bbox"), sizeof(double) * 6 * ctx->nc,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
  return ctx->sync();
}

int fmmb200_shard_pack(fmmb200_ctx *ctx, int64_t nclusters, const int32_t *d_cluster_ids, void *d_moments,
                       int64_t nleaves, const int32_t *d_leaf_ids, const int64_t *d_leaf_offsets, void *d_records) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_tree) return ctx->fail(FMMB200_ERR_NO_STATE, "shard_pack: no subtree");
  if (nclusters < 0 || nleaves < 0 || (nclusters > 0 && (!d_cluster_ids || !d_moments)) ||
      (nleaves > 0 && (!d_leaf_ids || !d_leaf_offsets || !d_records)))
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_pack: bad arguments");
  Guard g(ctx->device);
  const bool mixed = ctx->precision == FMMB200_PRECISION_MIXED;
  if (nclusters > 0) {
    const int w = (int)(moment_bytes(ctx->n, mixed) / 16);
    const uint4 *rec = mixed ? (const uint4 *)ctx->get<float>("mom32") : (const uint4 *)ctx->get<double>("mom64");
    pack_records_kernel<<<(unsigned)nclusters, 128, 0, ctx->stream>>>(nclusters, d_cluster_ids, w, rec,
                                                                      (uint4 *)d_moments, ctx->nc, ctx->d_status);
    FMM_TRY(ctx->check_launch("pack_records_kernel"));
  }
  if (nleaves > 0) {
    const int w = (int)(particle_bytes(mixed) / 16);
    const uint4 *rec = mixed ? (const uint4 *)ctx->get<float4>("prec32x2") : (const uint4 *)ctx->get<double>("prec64");
    pack_leaves_kernel<<<(unsigned)nleaves, 128, 0, ctx->stream>>>(nleaves, d_leaf_ids, d_leaf_offsets,
                                                                   ctx->get<int>("lohi"), w, rec, (uint4 *)d_records,
                                                                   ctx->nc, ctx->N, ctx->d_status);
    FMM_TRY(ctx->check_launch("pack_leaves_kernel"));
  }
  return ctx->check_device_status("shard_pack");
}

int fmmb200_shard_lists(fmmb200_ctx *ctx, int64_t nc, int32_t max_level, const double *d_bboxes, const double *pavg,
                        double eta, int32_t L, int32_t rank, int64_t *counts) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (max_level < 0 || max_level > 29 || nc != ((int64_t)2 << max_level) - 1 || !d_bboxes || !pavg)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_lists: nc must be 2^(max_level+1) - 1");
  if (L < 0 || L > max_level || rank < 0 || rank >= (1 << L))
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_lists: need 0 <= L <= max_level, 0 <= rank < 2^L");
  if (!(eta >= 0.0)) return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_lists: eta must be >= 0");
  Guard g(ctx->device);
  ctx->have_tree = ctx->have_lists = ctx->have_forward = ctx->saved = false;
  double *consts;
  FMM_TRY(shard_consts(ctx, pavg, &consts));
  ctx->nc = nc;
  ctx->ml = max_level;
  ctx->leaf0 = ((int64_t)1 << max_level) - 1;
  ctx->nleaf = (int64_t)1 << max_level;
  FMM_TRY(copy_in(ctx, "bbox", d_bboxes, sizeof(double) * 6 * nc));
  // the traversal's work statistics read particle counts; only the box geometry is known here
  int *lohi;
  FMM_TRY(ctx->ensure("lohi", 2 * nc, &lohi));
  FMM_CUDA_TRY(ctx, cudaMemsetAsync(lohi, 0, sizeof(int) * 2 * nc, ctx->stream));
  ctx->trav_L = L;
  ctx->trav_g = (1 << L) - 1 + rank;
  const int st = build_lists(ctx, eta, consts);
  ctx->trav_L = -1;
  FMM_TRY(st);
  if (counts) {
    counts[0] = ctx->nm2l;
    counts[1] = ctx->np2p;
  }
  ctx->stats.device_bytes = (int64_t)ctx->device_bytes;
  return FMMB200_OK;
}

int fmmb200_shard_get_lists(fmmb200_ctx *ctx, int32_t *d_m2l_ptr, int32_t *d_m2l_src, int32_t *d_p2p_ptr,
                            int32_t *d_p2p_src) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_lists) return ctx->fail(FMMB200_ERR_NO_STATE, "shard_get_lists: no lists");
  Guard g(ctx->device);
  const size_t P = sizeof(int) * (ctx->nc + 1);
  if (d_m2l_ptr) FMM_CUDA_TRY(ctx, cudaMemcpyAsync(d_m2l_ptr, ctx->get<int>("m2l_ptr"), P, cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_m2l_src && ctx->nm2l)
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(d_m2l_src, ctx->get<int>("m2l_src"), sizeof(int) * ctx->nm2l,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_p2p_ptr) FMM_CUDA_TRY(ctx, cudaMemcpyAsync(d_p2p_ptr, ctx->get<int>("p2p_ptr"), P, cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_p2p_src && ctx->np2p)
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(d_p2p_src, ctx->get<int>("p2p_src"), sizeof(int) * ctx->np2p,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
  return ctx->sync();
}

int fmmb200_shard_evaluate(fmmb200_ctx *ctx, int32_t L, int32_t rank, int64_t max_leaf, double eta, int64_t next,
                           const double *d_bboxes_ext, const void *d_moments_ext, const int32_t *d_lohi_ext,
                           int64_t nhalo, const void *d_halo_records, const int32_t *d_m2l_ptr,
                           const int32_t *d_m2l_src, int64_t nm2l, const int32_t *d_p2p_ptr, const int32_t *d_p2p_src,
                           int64_t np2p, double charge, double lambda, double *d_efields, double *d_bfields) {
  if (!ctx) return FMMB200_ERR_INVALID_ARGUMENT;
  if (!ctx->have_tree) return ctx->fail(FMMB200_ERR_NO_STATE, "shard_evaluate: no subtree (fmmb200_shard_subtree)");
  const int64_t nc_sub = ctx->nc, n_sub = ctx->N, ntop = ((int64_t)2 << L) - 1;
  if (L < 1 || L > 20 || rank < 0 || rank >= (1 << L))
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_evaluate: need 1 <= L <= 20 and 0 <= rank < 2^L");
  if (next < ntop || nhalo < 0 || nm2l < 0 || np2p < 0 || max_leaf < 1 || !(eta >= 0.0) || !(lambda != 0.0) ||
      !d_bboxes_ext || !d_moments_ext || !d_lohi_ext || (nhalo > 0 && !d_halo_records) || !d_m2l_ptr ||
      !d_p2p_ptr || (nm2l > 0 && !d_m2l_src) || (np2p > 0 && !d_p2p_src) || !d_efields || !d_bfields)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_evaluate: bad arguments");
  const int64_t nc_loc = nc_sub + next;
  if (nc_loc > 0x3FFFFFFF || n_sub + nhalo > 0x7FFFFFFF)
    return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_evaluate: too many clusters or particles");
  Guard g(ctx->device);
  const int n = ctx->n;
  const bool mixed = ctx->precision == FMMB200_PRECISION_MIXED;
  const int ml_sub = ctx->ml;
  const int64_t leaf0_sub = ctx->leaf0, nleaf_sub = ctx->nleaf;
  ctx->have_tree = false;  // the cluster arrays are extended below; a new subtree is needed afterwards
  // 1. the appended clusters (top of the tree at nc_sub .. nc_sub + ntop, then remote
  //    clusters): boxes, moments, particle ranges into the appended halo records
  FMM_TRY(extend_buffer(ctx, "bbox", sizeof(double) * 6 * nc_sub, d_bboxes_ext, sizeof(double) * 6 * next));
  const size_t mb = moment_bytes(n, mixed);
  FMM_TRY(extend_buffer(ctx, mixed ? "mom32" : "mom64", mb * nc_sub, d_moments_ext, mb * next));
  FMM_TRY(extend_buffer(ctx, "lohi", sizeof(int) * 2 * nc_sub, nullptr, sizeof(int) * 2 * next));
  lohi_ext_kernel<<<ceil_div(next, 256), 256, 0, ctx->stream>>>(next, d_lohi_ext, (int)n_sub, nhalo,
                                                                ctx->get<int>("lohi") + 2 * nc_sub, ctx->d_status);
  FMM_TRY(ctx->check_launch("lohi_ext_kernel"));
  const size_t pb = particle_bytes(mixed);
  FMM_TRY(extend_buffer(ctx, mixed ? "prec32x2" : "prec64", pb * n_sub, d_halo_records, pb * nhalo));
  ctx->nc = nc_loc;
  FMM_TRY(compute_nodes(ctx, n));
  // 2. moments of the top levels from the level-L ones (every rank's root)
  for (int l = L - 1; l >= 0; --l) FMM_TRY(launch_m2m_heap(ctx, n, mixed, l, (int)nc_sub));
  // 3. lists in local cluster numbers
  FMM_TRY(copy_in(ctx, "sh_m2l_ptr", d_m2l_ptr, sizeof(int) * (nc_loc + 1)));
  FMM_TRY(copy_in(ctx, "sh_m2l_src", d_m2l_src, sizeof(int) * (nm2l > 0 ? nm2l : 0)));
  FMM_TRY(copy_in(ctx, "p2p_ptr", d_p2p_ptr, sizeof(int) * (nc_loc + 1)));
  FMM_TRY(copy_in(ctx, "p2p_src", d_p2p_src, sizeof(int) * (np2p > 0 ? np2p : 0)));
  {
    void *d;
    FMM_TRY(ctx->ensure_bytes(mixed ? "loc32" : "loc64", (mb / 4) * 6 * nc_loc, &d));
    double *nr;
    FMM_TRY(ctx->ensure("near", 6 * n_sub, &nr));
  }
  // the lists come from the caller: check every entry before a kernel follows them
  {
    int *bad, *h;
    FMM_TRY(ctx->ensure("sh_bad", 1, &bad));
    FMM_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
    validate_csr_kernel<<<148, 256, 0, ctx->stream>>>(nc_loc, ctx->get<int>("sh_m2l_ptr"), ctx->get<int>("sh_m2l_src"),
                                                      nm2l, nullptr, 0, 0, bad);
    validate_csr_kernel<<<148, 256, 0, ctx->stream>>>(nc_loc, ctx->get<int>("p2p_ptr"), ctx->get<int>("p2p_src"),
                                                      np2p, ctx->get<int>("lohi"), 1, n_sub + nhalo, bad);
    FMM_TRY(ctx->check_launch("validate_csr_kernel", 2));
    FMM_TRY(ctx->pinned(sizeof(int) * 4, (void **)&h));
    FMM_CUDA_TRY(ctx, cudaMemcpyAsync(h, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    FMM_TRY(ctx->sync());
    if (h[0]) {
      ctx->nc = nc_sub;
      return ctx->fail(FMMB200_ERR_INVALID_ARGUMENT, "shard_evaluate: inconsistent lists (a row, source or range "
                                                     "outside the local clusters and records)");
    }
  }
  FMM_TRY(ctx->check_device_status("shard_evaluate (appended ranges)"));
  ctx->eta = eta;
  ctx->charge = charge;
  ctx->lambda = lambda;
  ctx->nm2l = nm2l;
  ctx->np2p = np2p;
  // 4. M2L over every local target (rows other than the own subtree's and its ancestors' are empty)
  ctx->m2l_ptr_key = "sh_m2l_ptr";
  ctx->m2l_src_key = "sh_m2l_src";
  int st = launch_m2l(ctx, n, mixed, false);
  ctx->m2l_ptr_key = "m2l_ptr";
  ctx->m2l_src_key = "m2l_src";
  FMM_TRY(st);
  // 5. P2P of the own leaves; the lane grouping follows the whole tree's largest leaf
  ctx->leaf0 = leaf0_sub;
  ctx->nleaf = nleaf_sub;
  ctx->max_leaf = max_leaf;
  FMM_TRY(launch_p2p(ctx, mixed, nullptr, nleaf_sub, false));
  // 6. L2L: the top levels, then the own root's parent into the own root, then the subtree
  for (int l = 1; l < L; ++l) FMM_TRY(launch_l2l_heap(ctx, n, mixed, l, (int)nc_sub));
  int2 *pc;
  FMM_TRY(ctx->ensure("sh_pc", 1, &pc));
  const int groot = (1 << L) - 1 + rank;
  const int2 h_pc = make_int2((int)nc_sub + (groot - 1) / 2, 0);
  FMM_CUDA_TRY(ctx, cudaMemcpyAsync(pc, &h_pc, sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
  FMM_TRY(launch_l2l_pairs(ctx, n, mixed, pc, 1));
  for (int l = 1; l <= ml_sub; ++l) FMM_TRY(launch_l2l(ctx, n, mixed, l));
  // 7. L2P with the near field, amp, and the own particles' order
  FMM_TRY(launch_l2p(ctx, n, mixed, nullptr, nleaf_sub, 1, kRe * charge / lambda, d_efields, d_bfields));
  st = ctx->check_device_status("shard_evaluate");
  ctx->nc = nc_sub;
  ctx->stats.device_bytes = (int64_t)ctx->device_bytes;
  FMM_TRY(st);
  return FMMB200_OK;
}

}  // extern "C"
