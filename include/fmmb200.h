/*
 * fmmb200.h -- C-ABI of libfmmb200.so, the B200 (sm_100a) interpolation-based
 * FMM for relativistic space-charge E/B fields.
 *
 * The library is a drop-in for FMM4RBGPU.jl's `FMMGPU` field evaluation:
 *   update_particles_field!(particles, FMMGPU(n=n, N0=N0, eta=eta); lambda)
 *   (src/update_particles_field.jl:66-148)
 * Every stage -- cluster-tree build, dual-tree traversal, P2M/M2M, M2L, P2P,
 * L2L/L2P -- runs as a CUDA kernel on one GPU.  There is no CPU fallback.
 *
 * Conventions
 *  - Particle vectors are AoS double[3*npar] (x,y,z per particle): the memory of
 *    a Julia Vector{SVector{3,Float64}} (src/particles.jl:1-9), passed as
 *    pointer(reinterpret(Float64, v)).
 *  - Index arrays are int64 and 0-based (the reference is 1-based: subtract 1).
 *    Cluster k (0-based) is the reference's node k+1 of the heap-numbered tree;
 *    its children are 2k+1 and 2k+2 and its parent (k+1)/2-1.
 *  - Moment / local arrays use the reference's Array{T,4} layout (n+1,n+1,n+1,nc)
 *    with i fastest; vector quantities interleave their 3 components
 *    (Array{SVector{3,Float64},4}).
 *  - Every function returns an int status (FMMB200_OK == 0) and never aborts or
 *    traps; fmmb200_last_error() gives the message of the last failure.
 *  - Host buffers are caller-owned and only accessed during the call.  Device
 *    memory, the stream and the saved forward state are owned by the context.
 *    A context is not re-entrant; separate contexts may be used from separate
 *    threads.  Host-pointer calls are synchronous (they return after the D2H copy).
 */
#ifndef FMMB200_H
#define FMMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FMMB200_API_VERSION 1

#define FMMB200_OK 0
#define FMMB200_ERR_INVALID_ARGUMENT 1
#define FMMB200_ERR_OUT_OF_MEMORY 2
#define FMMB200_ERR_CUDA 3
#define FMMB200_ERR_TREE_SHAPE 4   /* a leaf would occur above the maximum level */
#define FMMB200_ERR_NO_STATE 5     /* no forward state saved in the context */
#define FMMB200_ERR_DEVICE 6       /* a kernel raised its device status word */
#define FMMB200_ERR_CAPACITY 7     /* larger than a fixed-size scratch array allows */

#define FMMB200_PRECISION_FP64 0   /* plain FP64 path (the drop-in) */
#define FMMB200_PRECISION_MIXED 1  /* FP32 arithmetic, FP32 partials folded into FP64 sums, FP64 geometry */

typedef struct fmmb200_ctx fmmb200_ctx;

/* Per-call statistics of the last forward (and backward) on a context. */
typedef struct fmmb200_stats {
  int64_t npar, n, N0, max_level, ncluster, nleaf;
  int64_t nm2l, np2p, m2l_groups, p2p_groups;
  int64_t traversal_steps, device_bytes;
  double pavg[3], stretch[3];
  /* stage times in ms (CUDA events on the context stream; 0 unless timing is on) */
  double ms_h2d, ms_tree, ms_lists, ms_upward, ms_m2l, ms_p2p, ms_downward, ms_d2h, ms_total;
  double ms_backward;
  /* exact work counts from this call's lists */
  double m2l_kernel_evals; /* sum over M2L pairs of (n+1)^6 */
  double p2p_kernel_evals; /* sum over P2P pairs of |t|*|s| */
  int64_t kernel_launches; /* CUDA kernels launched by the last forward */
  int64_t tree_reused;     /* 1 if the last forward refitted the previous tree (fmmb200_set_tree_reuse) */
} fmmb200_stats;

/* ---- lifecycle ------------------------------------------------------------ */
int fmmb200_version(void);
int fmmb200_create(fmmb200_ctx **ctx, int device);
int fmmb200_destroy(fmmb200_ctx *ctx);
const char *fmmb200_last_error(const fmmb200_ctx *ctx);
/* Run on a caller-provided cudaStream_t (NULL restores the context's own stream, a
 * cudaStreamNonBlocking stream that is not ordered after work on the legacy default
 * stream).  To run after work on the legacy default stream (torch's default stream,
 * whose handle reads as 0), pass cudaStreamLegacy. */
int fmmb200_set_stream(fmmb200_ctx *ctx, void *stream);
/* Record per-stage CUDA events (stats ms_*); off by default. */
int fmmb200_set_timing(fmmb200_ctx *ctx, int enable);
/* Engine of the mixed-form M2L (no counterpart in the reference, whose M2L is one
 * FP64 kernel).  FMMB200_M2L_AUTO (default) and FMMB200_M2L_CUDA_CORES: the
 * packed FP32x2 CUDA-core kernel.  FMMB200_M2L_TENSOR_CORES: tcgen05 TF32 MMAs
 * with hi/lo splitting for n <= 4 and eta <= 1/2 (the CUDA-core kernel
 * otherwise), on the factored sums; the source pairs whose boxes nearly touch,
 * where factoring loses FP32 precision, still run on the CUDA cores.  Same
 * accuracy class, slower at n = 4 on B200.  The FP64 path is not affected. */
#define FMMB200_M2L_AUTO 0
#define FMMB200_M2L_CUDA_CORES 1
#define FMMB200_M2L_TENSOR_CORES 2
int fmmb200_set_m2l_engine(fmmb200_ctx *ctx, int engine);
/* Tree reuse across calls (no counterpart in the reference, which rebuilds the tree on
 * the host every call).  When enabled and the next forward has the same npar and N0 as
 * the previous tree, the library refits the boxes to the new positions and checks on
 * the device that every node would split its particles exactly as before (same split
 * axis, the left half still before the right half in coordinate-then-id order).  If so
 * the tree is kept -- it is bit-identical to a rebuild, so the fields are the same --
 * and the radix sorts and partitions are skipped; otherwise the tree is rebuilt.  For
 * time-stepping loops whose particles move little per step.  Off by default. */
int fmmb200_set_tree_reuse(fmmb200_ctx *ctx, int enable);
/* One beam over several GPUs (no counterpart in the reference, whose FMMGPU runs on one
 * GPU).  With world > 1, each forward builds the whole tree, the pair lists and all
 * moments from the whole beam, then runs M2L, P2P, L2L and L2P only for the clusters over
 * the leaves [rank nleaf / world, (rank + 1) nleaf / world) (heap order) and writes the
 * fields of the particles in those leaves; every other particle's field is set to 0.
 * The sum over rank = 0 .. world-1 is bit-identical to the unsharded forward, so the
 * caller combines the ranks with one sum-reduction (reduce-scatter or all-reduce).  The
 * adjoint needs an unsharded forward: save_for_backward with world > 1 is rejected.
 * 0 <= rank < world; world = 1 (the default) computes every field. */
int fmmb200_set_shard(fmmb200_ctx *ctx, int rank, int world);
/* Fault injection for tests: the k-th next device allocation fails (k >= 1; 0 disables). */
int fmmb200_debug_fail_alloc(fmmb200_ctx *ctx, int64_t k);

/* ---- drop-in field evaluation ---------------------------------------------
 * Replaces update_particles_field!(particles, FMMGPU(n,N0,eta); lambda)
 * (src/update_particles_field.jl:66-148).  efields/bfields are OVERWRITTEN with
 * the fields at every particle in the original particle order; positions and
 * momenta are unchanged.  1 <= n <= 10, N0 >= 1. */
int fmmb200_update_particles_field(fmmb200_ctx *ctx, int64_t npar, double charge,
                                   const double *positions, const double *momenta,
                                   double *efields, double *bfields, int32_t n, int64_t N0,
                                   double eta, double lambda, int32_t precision);

/* Forward with options.  pavg: NULL computes p_avg = sum(momenta)/npar on the
 * device with the pairwise summation of Julia's Base.sum (the serial FMM's
 * update_particles_field.jl:45); else the given 3 doubles are used.
 * save_for_backward keeps the tree, lists, moments and locals for
 * fmmb200_backward (no counterpart in the reference). */
int fmmb200_forward(fmmb200_ctx *ctx, int64_t npar, const double *positions,
                    const double *momenta, double charge, double lambda, int32_t n, int64_t N0,
                    double eta, int32_t precision, const double *pavg, int32_t save_for_backward,
                    double *efields, double *bfields);
/* Same with device pointers (AoS double[3*npar] in device memory); asynchronous
 * on the context stream.  pavg, if given, is a HOST pointer. */
int fmmb200_forward_device(fmmb200_ctx *ctx, int64_t npar, const double *d_positions,
                           const double *d_momenta, double charge, double lambda, int32_t n,
                           int64_t N0, double eta, int32_t precision, const double *pavg,
                           int32_t save_for_backward, double *d_efields, double *d_bfields);

/* Adjoint of the last saved forward (no counterpart in the reference): given
 * dL/dE and dL/dB (AoS, original order) returns dL/dpositions and dL/dmomenta.
 * The tree and lists are held fixed (the map is piecewise smooth). */
int fmmb200_backward(fmmb200_ctx *ctx, const double *grad_efields, const double *grad_bfields,
                     double *grad_positions, double *grad_momenta);
int fmmb200_backward_device(fmmb200_ctx *ctx, const double *d_grad_efields,
                            const double *d_grad_bfields, double *d_grad_positions,
                            double *d_grad_momenta);

int fmmb200_get_stats(const fmmb200_ctx *ctx, fmmb200_stats *out);

/* ---- introspection of the last forward / cluster_tree call ----------------- */
/* info: {npar, N0, max_level, ncluster, nm2l, np2p, n} */
int fmmb200_get_tree_info(const fmmb200_ctx *ctx, int64_t *info);
/* ClusterTree / Clusters fields (src/cluster_tree/clusters.jl:4-19); any may be NULL.
 * parindices[npar]; levels[nc]; parlohis[2nc]; parents[nc]; children[2nc]; bboxes[6nc]
 * as (xmin,ymin,zmin,xmax,ymax,zmax).  Particle ids inside a leaf are ascending. */
int fmmb200_get_tree(fmmb200_ctx *ctx, int64_t *parindices, int64_t *levels, int64_t *parlohis,
                     int64_t *parents, int64_t *children, double *bboxes);
/* InteractionListsGPU pair lists (src/gpu_fmm/gpu_interaction_lists.jl:3-12) as
 * (target, source) pairs sorted by (target, source); either may be NULL. */
int fmmb200_get_lists(fmmb200_ctx *ctx, int64_t *m2l_pairs, int64_t *p2p_pairs);
/* Macro-particle moments (gammas, momenta) and local fields (efields, bfields) of
 * the last saved forward, in the reference's Array{T,4} layouts; any may be NULL. */
int fmmb200_get_expansions(fmmb200_ctx *ctx, double *gammas, double *mp_momenta,
                           double *mp_efields, double *mp_bfields);

/* ---- stage entry points (kernel-level parity) -----------------------------
 * ClusterTree(particles; N0, stretch) (src/cluster_tree/cluster_tree.jl:12-18)
 * built on the device; outputs as in fmmb200_get_tree (any may be NULL). */
int fmmb200_cluster_tree(fmmb200_ctx *ctx, int64_t npar, const double *positions, int64_t N0,
                         const double *stretch, int64_t *parindices, int64_t *levels,
                         int64_t *parlohis, int64_t *parents, int64_t *children, double *bboxes);
/* InteractionListsGPU(clusters; stretch, eta) (src/gpu_fmm/gpu_interaction_lists.jl:27-40)
 * on the tree of the last fmmb200_cluster_tree call.  counts = {nm2l, np2p}. */
int fmmb200_interaction_lists(fmmb200_ctx *ctx, const double *stretch, double eta,
                              int64_t *counts);

/* gpu_P2M! (src/gpu_fmm/gpu_upwardpass.jl:3-85): moments of the listed leaf
 * clusters ADDED into gammas (nc*(n+1)^3) / mp_momenta (3*nc*(n+1)^3). */
int fmmb200_p2m(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t npar,
                const double *positions, const double *momenta, const int64_t *parindices,
                int64_t nc, const int64_t *parlohis, const double *bboxes, int64_t nleaf,
                const int64_t *leaf_ids, double *gammas, double *mp_momenta);
/* gpu_M2M! (src/gpu_fmm/gpu_upwardpass.jl:87-163) for every parent at `level`
 * that has children: parent moments += interpolated children moments. */
int fmmb200_m2m(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t nc,
                const int64_t *children, const double *bboxes, int64_t level, double *gammas,
                double *mp_momenta);
/* gpu_M2L! (src/gpu_fmm/gpu_interaction.jl:3-41): local fields of each pair's
 * target += kernel-weighted moments of its source. */
int fmmb200_m2l(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t nc, const double *bboxes,
                const double *gammas, const double *mp_momenta, int64_t npairs,
                const int64_t *pairs, const double *pavg, double *mp_efields,
                double *mp_bfields);
/* gpu_P2P! (src/gpu_fmm/gpu_interaction.jl:43-86): particle fields += near field. */
int fmmb200_p2p(fmmb200_ctx *ctx, int32_t precision, int64_t npar, const double *positions,
                const double *momenta, const int64_t *parindices, int64_t nc,
                const int64_t *parlohis, const double *bboxes, int64_t npairs,
                const int64_t *pairs, double *efields, double *bfields);
/* gpu_L2L! (src/gpu_fmm/gpu_downwardpass.jl:4-74) for every cluster at `level`:
 * child locals += parent locals interpolated at the child's nodes. */
int fmmb200_l2l(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t nc,
                const int64_t *parents, const double *bboxes, int64_t level,
                double *mp_efields, double *mp_bfields);
/* gpu_L2P! (src/gpu_fmm/gpu_downwardpass.jl:76-145): particle fields += leaf
 * locals interpolated at the particle. */
int fmmb200_l2p(fmmb200_ctx *ctx, int32_t n, int32_t precision, int64_t npar,
                const double *positions, const int64_t *parindices, int64_t nc,
                const int64_t *parlohis, const double *bboxes, int64_t nleaf,
                const int64_t *leaf_ids, const double *mp_efields, const double *mp_bfields,
                double *efields, double *bfields);

/* ---- diagnostics (no counterpart in the reference) ------------------------- */
/* FP64 direct sum on the GPU (the reference's BruteForce, update_particles_field.jl:21-38,
 * serial host code there) for `ntarget` target particles (targets NULL: all npar),
 * host pointers; efields/bfields receive 3*ntarget values (amp included). */
int fmmb200_direct(fmmb200_ctx *ctx, int64_t npar, const double *positions, const double *momenta,
                   double charge, double lambda, int64_t ntarget, const int64_t *targets,
                   double *efields, double *bfields);
/* Same with device pointers (d_targets: ntarget particle indices in [0, npar); NULL =
 * particles 0..ntarget-1, which needs ntarget <= npar).  Returns once the kernels have
 * finished: an index of d_targets outside [0, npar) is never read, and the call returns
 * FMMB200_ERR_DEVICE with NaN fields for that target. */
int fmmb200_direct_device(fmmb200_ctx *ctx, int64_t npar, const double *d_positions,
                          const double *d_momenta, double charge, double lambda, int64_t ntarget,
                          const int64_t *d_targets, double *d_efields, double *d_bfields);
/* The FP64 direct sum of fmmb200_direct_device without allocating anything: no
 * context, no cudaMalloc/cudaFree, no allocating library call (no counterpart in
 * the reference).  It is for callers that cannot let a library allocate device
 * memory: code whose device memory is owned by its own pool allocator (CUDA.jl's
 * pool, a framework that reserved the GPU up front), where a private cudaMalloc
 * may fail or fragment that pool, and loops in which the implicit device
 * synchronisation of cudaMalloc/cudaFree is not acceptable.  The caller passes
 * device inputs and outputs (d_targets: ntarget particle indices in [0, npar), NULL =
 * particles 0..ntarget-1, which needs ntarget <= npar) and a cudaStream_t (NULL =
 * default stream); the call is asynchronous on it.  The device cannot report a bad
 * index without a synchronisation, so an index of d_targets outside [0, npar) is not
 * read and gives NaN fields for that target.  The call reads the CUDA error state with
 * cudaPeekAtLastError and leaves a pending error of the caller's in place (it then
 * returns FMMB200_ERR_CUDA without launching).
 * Scratch: a file-scope __device__ array of 6*65536 doubles (3 MiB), held by every
 * GPU that loads the library until the process exits.  ntarget > 65536 returns
 * FMMB200_ERR_CAPACITY.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the array and it keeps the last
 * call's contents (each call writes every slot it reads); calls that overlap on
 * the GPU, e.g. on different streams, race on it. */
int fmmb200_direct_noalloc(int64_t npar, const double *d_positions, const double *d_momenta,
                           double charge, double lambda, int64_t ntarget, const int64_t *d_targets,
                           double *d_efields, double *d_bfields, void *stream);
/* ---- one beam over several GPUs, each holding part of the tree ------------------
 * No counterpart in the reference, whose FMMGPU evaluates the whole beam on one device
 * (src/update_particles_field.jl:66-148; its tree is built by ClusterTree,
 * src/cluster_tree/cluster_tree.jl:12-18, and traversed by dualtraversefill!,
 * src/fmm/interaction_lists.jl:23-49).  With 2^L ranks the tree is split at level L:
 * the caller partitions the first L levels across the ranks exactly as ClusterTree
 * would (the left child takes the first ceil(cnt/2) particles in (coordinate, index)
 * order along argmax(stretch .* extent)), so rank r holds the particles of the level-L
 * cluster g = 2^L - 1 + r, in ascending global index order.  Then, per rank (device
 * pointers, on the context stream, returning after the work is done):
 *   shard_subtree   builds g's subtree with `depth` = the whole tree's max level - L
 *                   levels and the given p_avg (HOST double[3], the whole beam's), and
 *                   computes its moments (P2M, M2M);
 *   shard_boxes     its nc_sub = 2^(depth+1) - 1 boxes (double[6 nc_sub], subtree heap
 *                   order), for the caller to all-gather into the whole tree's boxes;
 *   shard_lists     the dual traversal of the whole tree (nc = 2^(max_level+1) - 1 boxes in
 *                   heap order) keeping the rows of g's subtree and g's ancestors only
 *                   (counts = {nm2l, np2p}); shard_get_lists copies them out as CSR over
 *                   the nc targets (whole-tree cluster ids, sources ascending per row);
 *   shard_pack      moment records of the listed subtree clusters and particle records of
 *                   the listed subtree leaves (leaf k's records from record
 *                   d_leaf_offsets[k] on), which other ranks need;
 *   shard_evaluate  the fields of its own particles.  Local cluster numbers are: the
 *                   subtree (0 .. nc_sub-1), then `next` appended clusters: first the
 *                   whole tree's top 2^(L+1) - 1 clusters in heap order (level L: every
 *                   rank's subtree root, with its moments; above: computed here), then
 *                   remote clusters.  d_lohi_ext gives each appended cluster's range in
 *                   the nhalo appended particle records (hi < lo: none).  The lists are
 *                   CSR over the nc_sub + next local clusters, rows in the whole tree's
 *                   order.  max_leaf is the whole tree's largest leaf.  Fields go to the
 *                   own particles in the order shard_subtree received them.
 * Record sizes: shard_record_bytes (moments: 4 (n+1)^3 values of the precision's type;
 * particles: 64 bytes FP64, 80 bytes mixed).  The fields equal the single-GPU forward's
 * with the same p_avg bit for bit.  No adjoint is kept. */
int fmmb200_shard_record_bytes(int32_t n, int32_t precision, int64_t *moment_record,
                               int64_t *particle_record);
int fmmb200_shard_subtree(fmmb200_ctx *ctx, int64_t npar, const double *d_positions,
                          const double *d_momenta, int64_t N0, int32_t depth, const double *pavg,
                          int32_t n, int32_t precision);
int fmmb200_shard_boxes(fmmb200_ctx *ctx, double *d_bboxes);
int fmmb200_shard_pack(fmmb200_ctx *ctx, int64_t nclusters, const int32_t *d_cluster_ids,
                       void *d_moments, int64_t nleaves, const int32_t *d_leaf_ids,
                       const int64_t *d_leaf_offsets, void *d_records);
int fmmb200_shard_lists(fmmb200_ctx *ctx, int64_t nc, int32_t max_level, const double *d_bboxes,
                        const double *pavg, double eta, int32_t L, int32_t rank, int64_t *counts);
int fmmb200_shard_get_lists(fmmb200_ctx *ctx, int32_t *d_m2l_ptr, int32_t *d_m2l_src,
                            int32_t *d_p2p_ptr, int32_t *d_p2p_src);
int fmmb200_shard_evaluate(fmmb200_ctx *ctx, int32_t L, int32_t rank, int64_t max_leaf, double eta,
                           int64_t next, const double *d_bboxes_ext, const void *d_moments_ext,
                           const int32_t *d_lohi_ext, int64_t nhalo, const void *d_halo_records,
                           const int32_t *d_m2l_ptr, const int32_t *d_m2l_src, int64_t nm2l,
                           const int32_t *d_p2p_ptr, const int32_t *d_p2p_src, int64_t np2p,
                           double charge, double lambda, double *d_efields, double *d_bfields);

/* Attainable rate (kernel evaluations per second) of the mixed P2P kernel's evaluation body
 * on this device: the kernel's own per-source load and evaluation code over source records
 * held in shared memory, at the kernel's residency (six CTAs of 128 threads per SM), with no
 * staging, barriers or FP64 folds.  far: R from the hi parts (tiles apart by more than
 * 1/256 of their extent); near: from hi and lo parts.  The ceiling of p2p_x2_kernel's
 * rate for this instruction mix; no counterpart in the reference. */
int fmmb200_measure_p2p_body(fmmb200_ctx *ctx, double *far_evals_per_s, double *near_evals_per_s);
/* Measured CUDA-core FMA throughput (TFLOP/s, 2 flops per FMA) of the device with
 * scalar FP64, scalar FP32 and packed FP32x2 (FFMA2) chains: the roofline
 * denominators of the M2L / P2P kernels. */
int fmmb200_measure_fma_peak(fmmb200_ctx *ctx, double *fp64_tflops, double *fp32_tflops,
                             double *fp32x2_tflops);

#ifdef __cplusplus
}
#endif
#endif /* FMMB200_H */
