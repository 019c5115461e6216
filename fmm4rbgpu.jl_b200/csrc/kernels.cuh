// kernels.cuh -- host-side launchers shared between the translation units.
#pragma once

#include <functional>

#include "context.cuh"

namespace fmmb200 {

// Lets kernel `k` use `dyn` bytes of dynamic shared memory (static shared memory
// counts against the same 48 KB default, so opt in whenever the sum may exceed it).
template <class K>
inline int opt_in_smem(Ctx *ctx, K k, int dyn) {
  if (dyn <= 16 * 1024) return FMMB200_OK;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  if (e != cudaSuccess) return ctx->fail(FMMB200_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  return FMMB200_OK;
}

// ---------------------------------------------------------------- sort.cu
// Stable LSD radix sort by key bits [0, key_bits) (8-bit digits, passes whose
// digit is constant are skipped).  vals/vals_alt may be null (keys only).
// On return *in_alt tells whether the sorted data is in the *_alt buffers.
int radix_sort(Ctx *ctx, uint64_t *keys, uint64_t *keys_alt, uint32_t *vals, uint32_t *vals_alt,
               int64_t n, int key_bits, bool *in_alt);
// Exclusive scan of n int32 values (in and out may alias); *total (host) if not null.
int exclusive_scan_i32(Ctx *ctx, const int *in, int *out, int64_t n, int64_t *total);

// ---------------------------------------------------------------- tree.cu
// Device p_avg with the pairwise summation structure of Julia's Base.sum and
// stretch = (1, 1, sqrt(1 + p.p)) into d_consts[0..5].
int compute_pavg_stretch(Ctx *ctx, const double *d_mom_aos, int64_t N, double *d_consts);
// Build the cluster tree of N particles (AoS positions on device) with the
// stretch in d_consts[3..5]; fills ctx tree buffers and ctx->{N,N0,ml,nc,...}.
// after_sorts, if given, is called once the three coordinate orders are sorted and
// before anything reads d_consts (the radix sorts need the positions only).  depth >= 0
// replaces the maximum level computed from N and N0 (the shape rules still apply).
int build_tree(Ctx *ctx, const double *d_pos_aos, int64_t N, int64_t N0, const double *d_consts,
               const std::function<int()> &after_sorts = {}, int depth = -1);
// Refit the existing tree (same N, N0) to new positions: boxes and extremal
// particles bottom-up, and *same = true when every node would split as before, in
// which case the tree equals what build_tree would give.  Otherwise the refitted
// boxes are garbage and the caller rebuilds.
int refit_tree(Ctx *ctx, const double *d_pos_aos, int64_t N, int64_t N0, const double *d_consts, bool *same);
// Particle records in tree order ("prec64": x,y,z,gamma,ux,uy,uz,0) and, for
// the mixed form, leaf-local FP32 records ("prec32": x,y,z,gamma,ux,uy,uz,0
// relative to the leaf's box centre) and the P2P source records ("prec32x2":
// five float4 of duplicated values -x_hi,-y_hi,-z_hi,-x_lo,-y_lo,-z_lo,gamma,ux,uy,uz).
// leafpos (optional): leaf cluster of every tree-order position (explicit trees).
int gather_particles(Ctx *ctx, const double *d_pos_aos, const double *d_mom_aos, bool mixed,
                     const int *leafpos = nullptr);
// Traversal geometry (centre, radius, diameter, leaf flag) for the stretch in d_consts[3..5].
int compute_geom(Ctx *ctx, const double *d_consts);
// Chebyshev node coordinates (degree n) of every cluster into "nodes".
int compute_nodes(Ctx *ctx, int n);
int node_stride(int n);

// ---------------------------------------------------------------- traverse.cu
// Device buffer `name` of at least `need` bytes whose first `used` bytes survive a
// reallocation (which leaves headroom, so that similar later needs grow nothing).
int grow_keep(Ctx *ctx, const char *name, size_t used, size_t need, void **out);
int build_lists(Ctx *ctx, double eta, const double *d_consts);
// m2lu_* / p2pu_*: union of each list and its transpose with role flags
// (bit 0: (t,s) in the list, bit 1: (s,t) in the list), grouped by target.
int build_union_lists(Ctx *ctx);

// ---------------------------------------------------------------- backward.cu
// Adjoint of the saved FP64 forward; device AoS arrays in the caller's order.
int run_backward(Ctx *ctx, const double *d_ge, const double *d_gb, double *d_gx, double *d_gu);

// ---------------------------------------------------------------- interp.cu
// P2M of leaves (leaf_ids null: all leaves of the tree) into "mom"; accumulate
// adds to the existing moments instead of overwriting them.
int launch_p2m(Ctx *ctx, int n, bool mixed, const int *d_leaf_ids, int64_t nleaf, bool accumulate);
// M2M for all parents at parent level `plevel` (children at plevel+1).
int launch_m2m(Ctx *ctx, int n, bool mixed, int plevel, bool accumulate);
// L2L for all children at child level `clevel` (>= 1).
int launch_l2l(Ctx *ctx, int n, bool mixed, int clevel);
// The same two passes on a heap of clusters stored from cluster `off` on.
int launch_m2m_heap(Ctx *ctx, int n, bool mixed, int plevel, int off);
int launch_l2l_heap(Ctx *ctx, int n, bool mixed, int clevel, int off);
// L2L from parent d_pc[b].x into the single child d_pc[b].y, b < npc.
int launch_l2l_pairs(Ctx *ctx, int n, bool mixed, const int2 *d_pc, int npc);
// L2P of leaves.  mode 0: explicit (near += far at tree-order particles);
// mode 1: pipeline (out_aos[perm] = amp * (near + far)).
int launch_l2p(Ctx *ctx, int n, bool mixed, const int *d_leaf_ids, int64_t nleaf, int mode,
               double amp, double *d_out_e, double *d_out_b);

// ---------------------------------------------------------------- m2l.cu / p2p.cu
int launch_m2l(Ctx *ctx, int n, bool mixed, bool accumulate);
int launch_p2p(Ctx *ctx, bool mixed, const int *d_leaf_ids, int64_t nleaf, bool accumulate);

// ---------------------------------------------------------------- api.cu, for shard.cu
// Argument checks of a forward; consts[0..5] = (p_avg, stretch) from a host p_avg; the
// moment / local / near-field buffers of the context's tree.
int shard_check(Ctx *ctx, int64_t N, int n, int64_t N0, int precision);
int shard_consts(Ctx *ctx, const double *pavg_host, double **d_consts);
int shard_expansions(Ctx *ctx, int n, bool mixed);

}  // namespace fmmb200
