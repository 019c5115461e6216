/*
 * fmm_oracle.h -- CPU restatement (FP64) of the FMM4RBGPU.jl algorithms on the
 * space-charge field path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it.
 * The product (libfmmb200.so) never links, calls or falls back to it.
 *
 * Conventions (all 0-based; the reference is 1-based):
 *   positions / momenta / fields : AoS double[3*N]  (x,y,z per particle) -- the
 *                                  memory layout of Vector{SVector{3,Float64}}
 *   node k (0-based) == reference node k+1; children 2k+1, 2k+2; parent (k+1)/2-1
 *   parindices : int64[N]      (0-based particle ids, the permutation)
 *   levels     : int64[nc]
 *   parlohis   : int64[2*nc]   (inclusive lo, hi; 0-based)
 *   parents    : int64[nc]     (-1 for the root)
 *   children   : int64[2*nc]   (-1,-1 for a leaf)
 *   bboxes     : double[6*nc]  (xmin,ymin,zmin,xmax,ymax,zmax)
 *   moment / local arrays use the reference's (n+1,n+1,n+1,nc) column-major
 *   layout: gammas[i + m*(j + m*k) + m^3*c] with m = n+1, vector quantities
 *   interleaved as SVector: vec[3*(node + m^3*c) + comp].
 *   pair lists : int64[2*npairs] as (target, source).
 *
 * variant: ORC_VARIANT_CPU follows the serial `FMM` path (cheb2 node formula,
 * lgweight exact-node semantics, scatter M2M, DFS-ordered lists);
 * ORC_VARIANT_GPU follows the `FMMGPU` kernels (cheb2coord node formula,
 * last-flag exact-node semantics, per-thread partial sums, target-sorted lists)
 * without the shared-memory race of gpu_M2L!.
 */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_VARIANT_CPU 0
#define ORC_VARIANT_GPU 1

int64_t orc_maxlevel(int64_t N, int64_t N0);
int64_t orc_ncluster(int64_t N, int64_t N0);

/* sum(momenta)/N with Julia's pairwise reduction structure. */
void orc_pavg(int64_t N, const double *mom, double out[3]);
void orc_stretch(const double pavg[3], double stretch[3]);

int64_t orc_partition(int64_t *labels, int64_t lo, int64_t hi, const double *data,
                      int64_t stride, int64_t comp, int64_t pvtindex, int tiebreak);
int64_t orc_kpermute(int64_t *labels, int64_t lo, int64_t hi, const double *data,
                     int64_t stride, int64_t comp, int64_t k, uint64_t seed, int tiebreak);

/* Returns 0 if every node of the complete tree was filled, 1 if a leaf occurred
 * above the maximum level (unfilled nodes are left as level -1). */
int orc_cluster_tree(int64_t N, const double *pos, int64_t N0, const double stretch[3],
                     uint64_t seed, int canonical, int64_t *parindices, int64_t *levels,
                     int64_t *parlohis, int64_t *parents, int64_t *children, double *bboxes);

double orc_diameter(const double *bbox, const double stretch[3]);
int orc_admissible(const double *bbox1, const double *bbox2, const double stretch[3], double eta);

/* DFS dual traversal from (root, root).  Pass NULL buffers to count only.
 * Returns 0, or -1 when a capacity is too small (counts are still exact). */
int orc_interaction_lists(int64_t nc, const int64_t *children, const double *bboxes,
                          const double stretch[3], double eta, int64_t *p2p, int64_t cap_p2p,
                          int64_t *np2p, int64_t *m2l, int64_t cap_m2l, int64_t *nm2l);
/* Stable sort of pairs by target, then CSR group pointers (0-based, ngroup+1). */
void orc_sort_by_target(int64_t npairs, int64_t *pairs);
int64_t orc_ilistptrs(int64_t npairs, const int64_t *pairs, int64_t *ptrs);

void orc_cheb2(int n, double a, double b, double *out);
double orc_cheb2coord(int64_t i1, double a, double b, int D);
void orc_lgweight(double x, const double *nodes, int n, double *out);
void orc_lgweight_gpu(double x, const double *nodes, int n, double *out);

void orc_p2m(int variant, int n, const double *pos, const double *mom, const int64_t *parindices,
             const int64_t *parlohis, const double *bboxes, int64_t nleaf, const int64_t *leaf_ids,
             double *gammas, double *mmom);
void orc_m2m(int variant, int n, int64_t level, const int64_t *parents, const int64_t *children,
             const double *bboxes, double *gammas, double *mmom);
void orc_m2l(int variant, int n, const double *bboxes, const double *gammas, const double *mmom,
             int64_t npairs, const int64_t *pairs, const double pavg[3], double *mef, double *mbf);
void orc_p2p(int variant, const double *pos, const double *mom, const int64_t *parindices,
             const int64_t *parlohis, int64_t npairs, const int64_t *pairs, double *ef, double *bf);
void orc_l2l(int variant, int n, int64_t level, const int64_t *parents, const double *bboxes,
             double *mef, double *mbf);
void orc_l2p(int variant, int n, const double *pos, const int64_t *parindices,
             const int64_t *parlohis, const double *bboxes, int64_t nleaf, const int64_t *leaf_ids,
             const double *mef, const double *mbf, double *ef, double *bf);

/* Full field evaluation (update_particles_field! with FMM / FMMGPU), fields are
 * overwritten (they start from zero).  pavg may be NULL (then orc_pavg is used).
 * nthreads > 1 parallelises over independent targets with OpenMP; the result is
 * bit-identical to nthreads == 1.  stats (may be NULL) receives
 * {ml, nc, nm2l, np2p, t_tree, t_up, t_lists, t_m2l, t_p2p, t_down} (times in s).
 * Returns 0, 1 for a tree with a leaf above the maximum level, -2 on OOM. */
int orc_fmm(int variant, int64_t N, const double *pos, const double *mom, double charge,
            double lambda, int n, int64_t N0, double eta, const double *pavg, uint64_t seed,
            int nthreads, double *ef, double *bf, double *stats);

/* BruteForce (update_particles_field.jl:21-38) over all particles. */
void orc_bruteforce(int64_t N, const double *pos, const double *mom, double charge,
                    double lambda, int nthreads, double *ef, double *bf);
/* The same direct sum for a subset of targets (ef/bf are 3*ntarget). */
void orc_direct_targets(int64_t N, const double *pos, const double *mom, double charge,
                        double lambda, int64_t ntarget, const int64_t *targets, int nthreads,
                        double *ef, double *bf);

#ifdef __cplusplus
}
#endif
#endif
