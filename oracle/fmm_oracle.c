/*
 * fmm_oracle.c -- CPU restatement (FP64) of the FMM4RBGPU.jl space-charge path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU arms load this library;
 * the product path never does.
 *
 * Every function names the reference file:line it restates (paths inside the
 * FMM4RBGPU.jl project).  Arithmetic follows the reference's operation order
 * (no FMA contraction: build with -ffp-contract=off) so that tree shapes,
 * bounding boxes, admissibility decisions and interaction lists are bit-exact.
 *
 * Deliberate, documented differences from the reference:
 *  - kpermute! picks its pivot with rand(); here the pivot comes from a seeded
 *    xorshift generator and ties on the split coordinate are broken by particle
 *    id (tiebreak=1).  The SET of particles in each child is then deterministic
 *    and equal to the reference's whenever the split coordinate has no ties.
 *    With canonical=1 the ids inside each leaf are sorted ascending.
 *  - The serial FMM driver accumulates into particles.efields without zeroing
 *    them first (update_particles_field.jl:40-64 with interaction.jl:70-71);
 *    orc_fmm always starts from zero fields.
 *  - Empty pair lists give empty CSR pointers instead of the BoundsError of
 *    ilistptrs (gpu_interaction_lists.jl:16).
 */
#include "fmm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 2.220446049250313e-16   /* eps(Float64) == eps() */
#define ORC_RE 2.8179403699772166e-15   /* classical electron radius used for amp */

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------------- */
/* tree shape: cluster_tree/treeinfo.jl:6-26                                  */
/* ------------------------------------------------------------------------- */

/* treeinfo.jl:6-8: (N > N0) ? ceil(log(N/N0)/log(2)) : 0 */
int64_t orc_maxlevel(int64_t N, int64_t N0) {
    if (N > N0) return (int64_t)ceil(log((double)N / (double)N0) / log(2.0));
    return 0;
}

/* treeinfo.jl:10-13 */
int64_t orc_ncluster(int64_t N, int64_t N0) {
    int64_t ml = orc_maxlevel(N, N0);
    return ((int64_t)1 << (ml + 1)) - 1;
}

/* ------------------------------------------------------------------------- */
/* p_avg / stretch: update_particles_field.jl:45-47                           */
/* ------------------------------------------------------------------------- */

/* Base.mapreduce_impl sequential portion (first < last). */
static void vsum_seq(const double *a, int64_t first, int64_t last, double out[3]) {
    double s0 = a[3 * first + 0] + a[3 * (first + 1) + 0];
    double s1 = a[3 * first + 1] + a[3 * (first + 1) + 1];
    double s2 = a[3 * first + 2] + a[3 * (first + 1) + 2];
    for (int64_t i = first + 2; i <= last; ++i) {
        s0 = s0 + a[3 * i + 0];
        s1 = s1 + a[3 * i + 1];
        s2 = s2 + a[3 * i + 2];
    }
    out[0] = s0; out[1] = s1; out[2] = s2;
}

/* Base.mapreduce_impl with pairwise blocksize 1024. */
static void vsum_pairwise(const double *a, int64_t first, int64_t last, double out[3]) {
    if (first == last) {
        out[0] = a[3 * first]; out[1] = a[3 * first + 1]; out[2] = a[3 * first + 2];
    } else if (last - first < 1024) {
        vsum_seq(a, first, last, out);
    } else {
        int64_t mid = first + ((last - first) >> 1);
        double v1[3], v2[3];
        vsum_pairwise(a, first, mid, v1);
        vsum_pairwise(a, mid + 1, last, v2);
        out[0] = v1[0] + v2[0]; out[1] = v1[1] + v2[1]; out[2] = v1[2] + v2[2];
    }
}

/* sum(particles.momenta) / particles.npar (update_particles_field.jl:45);
 * Base._mapreduce: n==1 -> a1, n<16 -> sequential, else pairwise. */
void orc_pavg(int64_t N, const double *mom, double out[3]) {
    double s[3];
    if (N <= 0) { out[0] = out[1] = out[2] = 0.0; return; }
    if (N == 1) { s[0] = mom[0]; s[1] = mom[1]; s[2] = mom[2]; }
    else if (N < 16) vsum_seq(mom, 0, N - 1, s);
    else vsum_pairwise(mom, 0, N - 1, s);
    out[0] = s[0] / (double)N; out[1] = s[1] / (double)N; out[2] = s[2] / (double)N;
}

/* update_particles_field.jl:46-47: g_avg = sqrt(1 + dot(p,p)); stretch = (1,1,g_avg) */
void orc_stretch(const double p[3], double stretch[3]) {
    double pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    stretch[0] = 1.0; stretch[1] = 1.0; stretch[2] = sqrt(1.0 + pp);
}

/* ------------------------------------------------------------------------- */
/* partition / kpermute: utils/partition.jl:10-43                            */
/* ------------------------------------------------------------------------- */

static inline int key_less(const double *data, int64_t stride, int64_t comp, int64_t la,
                           int64_t lb, int tiebreak) {
    double va = data[la * stride + comp], vb = data[lb * stride + comp];
    if (va < vb) return 1;
    if (tiebreak && va == vb) return la < lb;
    return 0;
}

static uint64_t xorshift64(uint64_t *s) {
    uint64_t x = *s;
    x ^= x << 13; x ^= x >> 7; x ^= x << 17;
    *s = x;
    return x;
}

/* partition.jl:10-22 (Lomuto).  pvtval = data[labels[pvtindex]]. */
int64_t orc_partition(int64_t *labels, int64_t lo, int64_t hi, const double *data,
                      int64_t stride, int64_t comp, int64_t pvtindex, int tiebreak) {
    int64_t pl = labels[pvtindex], t;
    labels[pvtindex] = labels[hi]; labels[hi] = pl;
    int64_t j = lo;
    for (int64_t i = lo; i <= hi - 1; ++i) {
        if (key_less(data, stride, comp, labels[i], pl, tiebreak)) {
            t = labels[j]; labels[j] = labels[i]; labels[i] = t;
            j = j + 1;
        }
    }
    t = labels[hi]; labels[hi] = labels[j]; labels[j] = t;
    return j;
}

/* partition.jl:29-43 (quickselect); the pivot is drawn from a seeded generator. */
static int64_t kpermute_rng(int64_t *labels, int64_t lo, int64_t hi, const double *data,
                            int64_t stride, int64_t comp, int64_t k, uint64_t *rng, int tiebreak) {
    for (;;) {
        if (lo == hi) return lo;
        int64_t pvt = lo + (int64_t)(xorshift64(rng) % (uint64_t)(hi - lo + 1));
        int64_t p = orc_partition(labels, lo, hi, data, stride, comp, pvt, tiebreak);
        if (p == k) return k;
        else if (p > k) hi = p - 1;
        else lo = p + 1;
    }
}

int64_t orc_kpermute(int64_t *labels, int64_t lo, int64_t hi, const double *data,
                     int64_t stride, int64_t comp, int64_t k, uint64_t seed, int tiebreak) {
    uint64_t rng = seed ? seed : 0x9E3779B97F4A7C15ull;
    return kpermute_rng(labels, lo, hi, data, stride, comp, k, &rng, tiebreak);
}

/* ------------------------------------------------------------------------- */
/* cluster tree: cluster_tree/cluster_tree.jl:12-18, clusters.jl:21-70        */
/* ------------------------------------------------------------------------- */

typedef struct {
    const double *pos;
    int64_t N0;
    double stretch[3];
    uint64_t rng;
    int64_t *parindices, *levels, *parlohis, *parents, *children;
    double *bboxes;
    int64_t nc;
    int overflow;
} tree_ctx;

/* clusters.jl:51-70 */
static void bbox_of(const double *pos, const int64_t *parindices, int64_t lo, int64_t hi,
                    double *bb) {
    double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY;
    double zmin = INFINITY, zmax = -INFINITY;
    for (int64_t i = lo; i <= hi; ++i) {
        const double *p = pos + 3 * parindices[i];
        double x = p[0], y = p[1], z = p[2];
        xmin = x < xmin ? x : xmin;
        xmax = x > xmax ? x : xmax;
        ymin = y < ymin ? y : ymin;
        ymax = y > ymax ? y : ymax;
        zmin = z < zmin ? z : zmin;
        zmax = z > zmax ? z : zmax;
    }
    bb[0] = xmin; bb[1] = ymin; bb[2] = zmin; bb[3] = xmax; bb[4] = ymax; bb[5] = zmax;
}

/* clusters.jl:21-49 (node is 0-based; the reference's nodeindex is node+1) */
static void fill_clusters(tree_ctx *c, int64_t node, int64_t lo, int64_t hi, int64_t level) {
    if (node >= c->nc) { c->overflow = 1; return; }
    int64_t npar = hi - lo + 1;
    double *bb = c->bboxes + 6 * node;
    bbox_of(c->pos, c->parindices, lo, hi, bb);
    c->levels[node] = level;
    c->parlohis[2 * node] = lo;
    c->parlohis[2 * node + 1] = hi;
    c->parents[node] = (node + 1) / 2 - 1;
    if (npar <= c->N0) {
        c->children[2 * node] = -1;
        c->children[2 * node + 1] = -1;
    } else {
        /* splitdir = argmax(stretch .* (bbox[2] - bbox[1])), first maximum */
        double v0 = c->stretch[0] * (bb[3] - bb[0]);
        double v1 = c->stretch[1] * (bb[4] - bb[1]);
        double v2 = c->stretch[2] * (bb[5] - bb[2]);
        int64_t dir = 0;
        double best = v0;
        if (v1 > best) { best = v1; dir = 1; }
        if (v2 > best) { best = v2; dir = 2; }
        int64_t k = (lo + hi) >> 1; /* 1-based floor((lo+hi)/2) shifted to 0-based */
        int64_t pvt = kpermute_rng(c->parindices, lo, hi, c->pos, 3, dir, k, &c->rng, 1);
        int64_t c1 = 2 * node + 1, c2 = 2 * node + 2;
        c->children[2 * node] = c1;
        c->children[2 * node + 1] = c2;
        fill_clusters(c, c1, lo, pvt, level + 1);
        fill_clusters(c, c2, pvt + 1, hi, level + 1);
    }
}

static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

int orc_cluster_tree(int64_t N, const double *pos, int64_t N0, const double stretch[3],
                     uint64_t seed, int canonical, int64_t *parindices, int64_t *levels,
                     int64_t *parlohis, int64_t *parents, int64_t *children, double *bboxes) {
    tree_ctx c;
    c.pos = pos;
    c.N0 = N0;
    c.stretch[0] = stretch[0]; c.stretch[1] = stretch[1]; c.stretch[2] = stretch[2];
    c.rng = seed ? seed : 0x9E3779B97F4A7C15ull;
    c.parindices = parindices; c.levels = levels; c.parlohis = parlohis;
    c.parents = parents; c.children = children; c.bboxes = bboxes;
    c.nc = orc_ncluster(N, N0);
    c.overflow = 0;
    for (int64_t i = 0; i < N; ++i) parindices[i] = i;
    for (int64_t k = 0; k < c.nc; ++k) {
        levels[k] = -1; parents[k] = (k + 1) / 2 - 1;
        parlohis[2 * k] = parlohis[2 * k + 1] = -1;
        children[2 * k] = children[2 * k + 1] = -1;
        for (int d = 0; d < 6; ++d) bboxes[6 * k + d] = 0.0;
    }
    fill_clusters(&c, 0, 0, N - 1, 0);
    int64_t ml = orc_maxlevel(N, N0);
    int incomplete = c.overflow;
    for (int64_t k = 0; k < c.nc; ++k) {
        if (levels[k] < 0) { incomplete = 1; continue; }
        if (children[2 * k] < 0) {
            if (levels[k] != ml) incomplete = 1;
            if (canonical)
                qsort(parindices + parlohis[2 * k], (size_t)(parlohis[2 * k + 1] - parlohis[2 * k] + 1),
                      sizeof(int64_t), cmp_i64);
        }
    }
    return incomplete;
}

/* ------------------------------------------------------------------------- */
/* geometry: utils/bbox.jl:9-11, fmm/interaction_lists.jl:10-21               */
/* ------------------------------------------------------------------------- */

/* StaticArrays norm of a 3-vector: sqrt(abs2(a1) + abs2(a2) + abs2(a3)). */
static inline double norm3(double a, double b, double c) { return sqrt(a * a + b * b + c * c); }

/* bbox.jl:9-11: norm(stretch .* (bbox[2] - bbox[1]) ./ 2.0) */
double orc_diameter(const double *bb, const double s[3]) {
    return norm3(s[0] * (bb[3] - bb[0]) / 2.0, s[1] * (bb[4] - bb[1]) / 2.0,
                 s[2] * (bb[5] - bb[2]) / 2.0);
}

/* interaction_lists.jl:10-21 */
int orc_admissible(const double *b1, const double *b2, const double s[3], double eta) {
    double xc1[3], xc2[3];
    for (int d = 0; d < 3; ++d) {
        xc1[d] = (b1[d] + b1[3 + d]) / 2.0;
        xc2[d] = (b2[d] + b2[3 + d]) / 2.0;
    }
    double r1 = norm3(s[0] * (b1[3] - xc1[0]), s[1] * (b1[4] - xc1[1]), s[2] * (b1[5] - xc1[2]));
    double r2 = norm3(s[0] * (b2[3] - xc2[0]), s[1] * (b2[4] - xc2[1]), s[2] * (b2[5] - xc2[2]));
    double R = norm3(s[0] * (xc1[0] - xc2[0]), s[1] * (xc1[1] - xc2[1]), s[2] * (xc1[2] - xc2[2]));
    double m = (r2 > r1) ? r2 : r1;
    if (isnan(r1) || isnan(r2)) m = NAN;
    return (m / R) < eta;
}

/* ------------------------------------------------------------------------- */
/* dual traversal: fmm/interaction_lists.jl:23-58                             */
/* ------------------------------------------------------------------------- */

typedef struct {
    const int64_t *children;
    const double *bboxes;
    double stretch[3];
    double eta;
    int64_t *p2p, *m2l;
    int64_t cap_p2p, cap_m2l, np2p, nm2l;
} trav_ctx;

static void dualtraverse(trav_ctx *c, int64_t t, int64_t s) {
    const int64_t *tc = c->children + 2 * t, *sc = c->children + 2 * s;
    int tleaf = (tc[0] == -1 && tc[1] == -1), sleaf = (sc[0] == -1 && sc[1] == -1);
    if (tleaf && sleaf) {
        if (c->p2p && c->np2p < c->cap_p2p) {
            c->p2p[2 * c->np2p] = t; c->p2p[2 * c->np2p + 1] = s;
        }
        c->np2p++;
    } else if (orc_admissible(c->bboxes + 6 * t, c->bboxes + 6 * s, c->stretch, c->eta)) {
        if (c->m2l && c->nm2l < c->cap_m2l) {
            c->m2l[2 * c->nm2l] = t; c->m2l[2 * c->nm2l + 1] = s;
        }
        c->nm2l++;
    } else if (tleaf) {
        dualtraverse(c, t, sc[0]);
        dualtraverse(c, t, sc[1]);
    } else if (sleaf) {
        dualtraverse(c, tc[0], s);
        dualtraverse(c, tc[1], s);
    } else {
        if (orc_diameter(c->bboxes + 6 * t, c->stretch) > orc_diameter(c->bboxes + 6 * s, c->stretch)) {
            dualtraverse(c, tc[0], s);
            dualtraverse(c, tc[1], s);
        } else {
            dualtraverse(c, t, sc[0]);
            dualtraverse(c, t, sc[1]);
        }
    }
}

int orc_interaction_lists(int64_t nc, const int64_t *children, const double *bboxes,
                          const double stretch[3], double eta, int64_t *p2p, int64_t cap_p2p,
                          int64_t *np2p, int64_t *m2l, int64_t cap_m2l, int64_t *nm2l) {
    trav_ctx c;
    (void)nc;
    c.children = children; c.bboxes = bboxes;
    c.stretch[0] = stretch[0]; c.stretch[1] = stretch[1]; c.stretch[2] = stretch[2];
    c.eta = eta;
    c.p2p = p2p; c.m2l = m2l; c.cap_p2p = cap_p2p; c.cap_m2l = cap_m2l;
    c.np2p = 0; c.nm2l = 0;
    dualtraverse(&c, 0, 0);
    *np2p = c.np2p;
    *nm2l = c.nm2l;
    if ((p2p && c.np2p > cap_p2p) || (m2l && c.nm2l > cap_m2l)) return -1;
    return 0;
}

/* sort!(lists, by = x -> x[1]) -- stable (gpu_interaction_lists.jl:33-34) */
void orc_sort_by_target(int64_t npairs, int64_t *pairs) {
    if (npairs <= 1) return;
    int64_t tmax = 0;
    for (int64_t i = 0; i < npairs; ++i) if (pairs[2 * i] > tmax) tmax = pairs[2 * i];
    int64_t *cnt = (int64_t *)calloc((size_t)tmax + 2, sizeof(int64_t));
    int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)npairs);
    for (int64_t i = 0; i < npairs; ++i) cnt[pairs[2 * i] + 1]++;
    for (int64_t t = 0; t <= tmax; ++t) cnt[t + 1] += cnt[t];
    for (int64_t i = 0; i < npairs; ++i) {
        int64_t d = cnt[pairs[2 * i]]++;
        tmp[2 * d] = pairs[2 * i]; tmp[2 * d + 1] = pairs[2 * i + 1];
    }
    memcpy(pairs, tmp, sizeof(int64_t) * 2 * (size_t)npairs);
    free(tmp);
    free(cnt);
}

/* gpu_interaction_lists.jl:14-25 (0-based); returns the number of groups. */
int64_t orc_ilistptrs(int64_t npairs, const int64_t *pairs, int64_t *ptrs) {
    int64_t ng = 0;
    ptrs[0] = 0;
    if (npairs == 0) return 0;
    int64_t val = pairs[0];
    for (int64_t i = 0; i < npairs; ++i) {
        if (pairs[2 * i] != val) { val = pairs[2 * i]; ptrs[++ng] = i; }
    }
    ptrs[++ng] = npairs;
    return ng;
}

/* ------------------------------------------------------------------------- */
/* Chebyshev nodes and Lagrange weights                                       */
/* ------------------------------------------------------------------------- */

/* utils/cheb2.jl:3-5: [cos(pi*i/n) for i=0:n].*(b-a)/2.0 .+ (a+b)/2.0 */
void orc_cheb2(int n, double a, double b, double *out) {
    for (int i = 0; i <= n; ++i) out[i] = cos(M_PI * (double)i / (double)n) * (b - a) / 2.0 + (a + b) / 2.0;
}

/* utils/barylg.jl:25-27 (i1 is 1-based): a + (cos(pi*(i-1)/D) + 1.0)/2.0 * (b - a) */
double orc_cheb2coord(int64_t i1, double a, double b, int D) {
    return a + (cos(M_PI * (double)(i1 - 1) / (double)D) + 1.0) / 2.0 * (b - a);
}

static void cheb2coords_gpu(int n, double a, double b, double *out) {
    for (int i = 0; i < n + 1; ++i) out[i] = orc_cheb2coord(i + 1, a, b, n);
}

/* fmm/upwardpass.jl:4-15 */
void orc_lgweight(double x, const double *nodes, int n, double *out) {
    int any = 0;
    for (int i = 0; i <= n; ++i) if (fabs(x - nodes[i]) < ORC_EPS) any = 1;
    if (any) {
        for (int i = 0; i <= n; ++i) out[i] = (fabs(x - nodes[i]) < ORC_EPS) ? 1.0 : 0.0;
        return;
    }
    double ws[16], v[16];
    for (int j = 0; j <= n; ++j) ws[j] = (j % 2 == 0) ? 1.0 : -1.0;
    ws[0] = 0.5;
    ws[n] = 0.5 * ws[n];
    for (int j = 0; j <= n; ++j) v[j] = ws[j] / (x - nodes[j]);
    double s = v[0] + v[1];
    for (int j = 2; j <= n; ++j) s = s + v[j];
    for (int j = 0; j <= n; ++j) out[j] = v[j] / s;
}

/* utils/barylg.jl:14-23 (baryweights(Val(n+1))); n=1 keeps the table's (0.5,-1). */
static void baryweights_gpu(int n, double *ws) {
    for (int j = 0; j <= n; ++j) ws[j] = (j % 2 == 0) ? 1.0 : -1.0;
    ws[0] = 0.5;
    if (n >= 2) ws[n] = 0.5 * ws[n];
}

/* The per-axis weight computation of gpu_P2M!/gpu_M2M!/gpu_L2L!/gpu_L2P!
 * (gpu_upwardpass.jl:48-76): last node within eps wins; otherwise
 * (ws[i]/(x - node_i))/sum. */
void orc_lgweight_gpu(double x, const double *nodes, int n, double *out) {
    double ws[16];
    baryweights_gpu(n, ws);
    double sum = 0.0;
    int flag = -1;
    for (int i = 0; i <= n; ++i) {
        double dx = x - nodes[i];
        flag = fabs(dx) < ORC_EPS ? i : flag;
        sum += ws[i] / dx;
    }
    for (int i = 0; i <= n; ++i) {
        if (flag == -1) out[i] = (ws[i] / (x - nodes[i])) / sum;
        else out[i] = (i == flag) ? 1.0 : 0.0;
    }
}

static void node_coords(int variant, int n, const double *bb, double *xs, double *ys, double *zs) {
    if (variant == ORC_VARIANT_CPU) {
        orc_cheb2(n, bb[0], bb[3], xs);
        orc_cheb2(n, bb[1], bb[4], ys);
        orc_cheb2(n, bb[2], bb[5], zs);
    } else {
        cheb2coords_gpu(n, bb[0], bb[3], xs);
        cheb2coords_gpu(n, bb[1], bb[4], ys);
        cheb2coords_gpu(n, bb[2], bb[5], zs);
    }
}

static inline void weights(int variant, double x, const double *nodes, int n, double *out) {
    if (variant == ORC_VARIANT_CPU) orc_lgweight(x, nodes, n, out);
    else orc_lgweight_gpu(x, nodes, n, out);
}

/* K(R; p) = R / sqrt(dot(R,R) + dot(p,R)^2 + eps())^3  (interaction.jl:36,69) */
static inline void kernel_K(double r0, double r1, double r2, const double *p, double *K) {
    double rr = r0 * r0 + r1 * r1 + r2 * r2;
    double pr = p[0] * r0 + p[1] * r1 + p[2] * r2;
    double s = sqrt(rr + pr * pr + ORC_EPS);
    double s3 = s * s * s;
    K[0] = r0 / s3; K[1] = r1 / s3; K[2] = r2 / s3;
}

/* ------------------------------------------------------------------------- */
/* upward pass                                                                */
/* ------------------------------------------------------------------------- */

/* CPU: fmm/upwardpass.jl:17-52.  GPU: gpu_upwardpass.jl:3-85. */
static void p2m_leaf(int variant, int n, const double *pos, const double *mom,
                     const int64_t *parindices, const int64_t *parlohis, const double *bboxes,
                     int64_t node, double *gammas, double *mmom) {
    int m = n + 1, NN = m * m * m;
    double xs[16], ys[16], zs[16], wx[16], wy[16], wz[16];
    int64_t lo = parlohis[2 * node], hi = parlohis[2 * node + 1];
    node_coords(variant, n, bboxes + 6 * node, xs, ys, zs);
    double *G = gammas + (int64_t)NN * node;
    double *M = mmom + (int64_t)3 * NN * node;
    if (variant == ORC_VARIANT_CPU) {
        for (int64_t p = lo; p <= hi; ++p) {
            int64_t pi = parindices[p];
            const double *x = pos + 3 * pi, *u = mom + 3 * pi;
            double ga = sqrt(1.0 + (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
            weights(variant, x[0], xs, n, wx);
            weights(variant, x[1], ys, n, wy);
            weights(variant, x[2], zs, n, wz);
            for (int k = 0; k < m; ++k)
                for (int j = 0; j < m; ++j)
                    for (int i = 0; i < m; ++i) {
                        double w = wx[i] * wy[j] * wz[k];
                        int a = i + m * (j + m * k);
                        G[a] += ga * w;
                        M[3 * a + 0] += u[0] * w;
                        M[3 * a + 1] += u[1] * w;
                        M[3 * a + 2] += u[2] * w;
                    }
        }
    } else {
        /* one thread per grid node, partial sums over the leaf's particles */
        int64_t cnt = hi - lo + 1;
        double *W = (double *)malloc(sizeof(double) * 3 * m * (size_t)(cnt > 0 ? cnt : 1));
        for (int64_t p = lo; p <= hi; ++p) {
            const double *x = pos + 3 * parindices[p];
            double *w = W + 3 * m * (p - lo);
            weights(variant, x[0], xs, n, w);
            weights(variant, x[1], ys, n, w + m);
            weights(variant, x[2], zs, n, w + 2 * m);
        }
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < m; ++j)
                for (int i = 0; i < m; ++i) {
                    double g = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0;
                    for (int64_t p = lo; p <= hi; ++p) {
                        const double *u = mom + 3 * parindices[p];
                        const double *w = W + 3 * m * (p - lo);
                        double ga = sqrt(1.0 + (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
                        double wt = w[i] * w[m + j] * w[2 * m + k];
                        g += ga * wt;
                        s0 += u[0] * wt; s1 += u[1] * wt; s2 += u[2] * wt;
                    }
                    int a = i + m * (j + m * k);
                    G[a] += g;
                    M[3 * a + 0] += s0; M[3 * a + 1] += s1; M[3 * a + 2] += s2;
                }
        free(W);
    }
}

void orc_p2m(int variant, int n, const double *pos, const double *mom, const int64_t *parindices,
             const int64_t *parlohis, const double *bboxes, int64_t nleaf, const int64_t *leaf_ids,
             double *gammas, double *mmom) {
    for (int64_t l = 0; l < nleaf; ++l)
        p2m_leaf(variant, n, pos, mom, parindices, parlohis, bboxes, leaf_ids[l], gammas, mmom);
}

/* CPU: fmm/upwardpass.jl:56-99 (child scatters into parent).
 * GPU: gpu_upwardpass.jl:87-163 (parent gathers from both children).
 * Both are expressed per parent so that parents can run in parallel; for
 * the CPU variant the children are visited in increasing node order, which is
 * the order of the serial loop over nodeindexrangeat(level). */
static void m2m_parent(int variant, int n, int64_t parent, const int64_t *children,
                       const double *bboxes, double *gammas, double *mmom) {
    int m = n + 1, NN = m * m * m;
    double pxs[16], pys[16], pzs[16], cxs[16], cys[16], czs[16];
    double wx[16], wy[16], wz[16];
    node_coords(variant, n, bboxes + 6 * parent, pxs, pys, pzs);
    double *PG = gammas + (int64_t)NN * parent;
    double *PM = mmom + (int64_t)3 * NN * parent;
    if (variant == ORC_VARIANT_CPU) {
        for (int ci2 = 0; ci2 < 2; ++ci2) {
            int64_t child = children[2 * parent + ci2];
            node_coords(variant, n, bboxes + 6 * child, cxs, cys, czs);
            const double *CG = gammas + (int64_t)NN * child;
            const double *CM = mmom + (int64_t)3 * NN * child;
            for (int ck = 0; ck < m; ++ck) {
                weights(variant, czs[ck], pzs, n, wz);
                for (int cj = 0; cj < m; ++cj) {
                    weights(variant, cys[cj], pys, n, wy);
                    for (int ci = 0; ci < m; ++ci) {
                        weights(variant, cxs[ci], pxs, n, wx);
                        int c = ci + m * (cj + m * ck);
                        double cga = CG[c], cm0 = CM[3 * c], cm1 = CM[3 * c + 1], cm2 = CM[3 * c + 2];
                        for (int pk = 0; pk < m; ++pk)
                            for (int pj = 0; pj < m; ++pj)
                                for (int pi = 0; pi < m; ++pi) {
                                    double w = wx[pi] * wy[pj] * wz[pk];
                                    int a = pi + m * (pj + m * pk);
                                    PG[a] += cga * w;
                                    PM[3 * a + 0] += cm0 * w;
                                    PM[3 * a + 1] += cm1 * w;
                                    PM[3 * a + 2] += cm2 * w;
                                }
                    }
                }
            }
        }
    } else {
        double *W = (double *)malloc(sizeof(double) * 2 * NN * 3 * m);
        for (int ci2 = 0; ci2 < 2; ++ci2) {
            int64_t child = children[2 * parent + ci2];
            node_coords(variant, n, bboxes + 6 * child, cxs, cys, czs);
            for (int c = 0; c < NN; ++c) {
                int ci = c % m, cj = (c / m) % m, ck = c / (m * m);
                double *w = W + ((int64_t)ci2 * NN + c) * 3 * m;
                weights(variant, cxs[ci], pxs, n, w);
                weights(variant, cys[cj], pys, n, w + m);
                weights(variant, czs[ck], pzs, n, w + 2 * m);
            }
        }
        for (int a = 0; a < NN; ++a) {
            int pi = a % m, pj = (a / m) % m, pk = a / (m * m);
            double g = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0;
            for (int ci2 = 0; ci2 < 2; ++ci2) {
                int64_t child = children[2 * parent + ci2];
                const double *CG = gammas + (int64_t)NN * child;
                const double *CM = mmom + (int64_t)3 * NN * child;
                for (int c = 0; c < NN; ++c) {
                    const double *w = W + ((int64_t)ci2 * NN + c) * 3 * m;
                    double wt = w[pi] * w[m + pj] * w[2 * m + pk];
                    g += CG[c] * wt;
                    s0 += CM[3 * c] * wt; s1 += CM[3 * c + 1] * wt; s2 += CM[3 * c + 2] * wt;
                }
            }
            PG[a] += g;
            PM[3 * a] += s0; PM[3 * a + 1] += s1; PM[3 * a + 2] += s2;
        }
        free(W);
    }
}

/* level = the CHILD level (upwardpass.jl:104-107 calls M2M! for l = ml..1). */
void orc_m2m(int variant, int n, int64_t level, const int64_t *parents, const int64_t *children,
             const double *bboxes, double *gammas, double *mmom) {
    (void)parents;
    int64_t p0 = ((int64_t)1 << (level - 1)) - 1, p1 = ((int64_t)1 << level) - 1;
    for (int64_t p = p0; p < p1; ++p) {
        if (children[2 * p] < 0) continue;
        m2m_parent(variant, n, p, children, bboxes, gammas, mmom);
    }
}

/* ------------------------------------------------------------------------- */
/* interactions                                                               */
/* ------------------------------------------------------------------------- */

/* CPU: fmm/interaction.jl:3-46.  GPU: gpu_interaction.jl:3-41 (per target node
 * partial sum over the source grid, then +=). */
static void m2l_pair(int variant, int n, const double *bboxes, const double *gammas,
                     const double *mmom, int64_t t, int64_t s, const double *pavg, double *mef,
                     double *mbf) {
    int m = n + 1, NN = m * m * m;
    double sxs[16], sys[16], szs[16], txs[16], tys[16], tzs[16], K[3];
    node_coords(variant, n, bboxes + 6 * s, sxs, sys, szs);
    node_coords(variant, n, bboxes + 6 * t, txs, tys, tzs);
    const double *SG = gammas + (int64_t)NN * s;
    const double *SM = mmom + (int64_t)3 * NN * s;
    double *TE = mef + (int64_t)3 * NN * t;
    double *TB = mbf + (int64_t)3 * NN * t;
    for (int tk = 0; tk < m; ++tk)
        for (int tj = 0; tj < m; ++tj)
            for (int ti = 0; ti < m; ++ti) {
                int a = ti + m * (tj + m * tk);
                double tx = txs[ti], ty = tys[tj], tz = tzs[tk];
                double e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
                double *E = TE + 3 * a, *B = TB + 3 * a;
                for (int sk = 0; sk < m; ++sk)
                    for (int sj = 0; sj < m; ++sj)
                        for (int si = 0; si < m; ++si) {
                            int b = si + m * (sj + m * sk);
                            kernel_K(tx - sxs[si], ty - sys[sj], tz - szs[sk], pavg, K);
                            double g = SG[b];
                            const double *M = SM + 3 * b;
                            double c0 = M[1] * K[2] - M[2] * K[1];
                            double c1 = M[2] * K[0] - M[0] * K[2];
                            double c2 = M[0] * K[1] - M[1] * K[0];
                            if (variant == ORC_VARIANT_CPU) {
                                E[0] += g * K[0]; E[1] += g * K[1]; E[2] += g * K[2];
                                B[0] += c0; B[1] += c1; B[2] += c2;
                            } else {
                                e0 += g * K[0]; e1 += g * K[1]; e2 += g * K[2];
                                b0 += c0; b1 += c1; b2 += c2;
                            }
                        }
                if (variant != ORC_VARIANT_CPU) {
                    E[0] += e0; E[1] += e1; E[2] += e2;
                    B[0] += b0; B[1] += b1; B[2] += b2;
                }
            }
}

void orc_m2l(int variant, int n, const double *bboxes, const double *gammas, const double *mmom,
             int64_t npairs, const int64_t *pairs, const double pavg[3], double *mef, double *mbf) {
    for (int64_t i = 0; i < npairs; ++i)
        m2l_pair(variant, n, bboxes, gammas, mmom, pairs[2 * i], pairs[2 * i + 1], pavg, mef, mbf);
}

/* CPU: fmm/interaction.jl:49-75.  GPU: gpu_interaction.jl:43-86. */
static void p2p_pair(int variant, const double *pos, const double *mom, const int64_t *parindices,
                     const int64_t *parlohis, int64_t t, int64_t s, double *ef, double *bf) {
    int64_t tlo = parlohis[2 * t], thi = parlohis[2 * t + 1];
    int64_t slo = parlohis[2 * s], shi = parlohis[2 * s + 1];
    double K[3];
    for (int64_t i = tlo; i <= thi; ++i) {
        int64_t pi = parindices[i];
        const double *xi = pos + 3 * pi;
        double *E = ef + 3 * pi, *B = bf + 3 * pi;
        double e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
        for (int64_t j = slo; j <= shi; ++j) {
            int64_t pj = parindices[j];
            const double *xj = pos + 3 * pj, *u = mom + 3 * pj;
            double gj = sqrt(1.0 + (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
            kernel_K(xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2], u, K);
            double c0 = u[1] * K[2] - u[2] * K[1];
            double c1 = u[2] * K[0] - u[0] * K[2];
            double c2 = u[0] * K[1] - u[1] * K[0];
            if (variant == ORC_VARIANT_CPU) {
                E[0] += gj * K[0]; E[1] += gj * K[1]; E[2] += gj * K[2];
                B[0] += c0; B[1] += c1; B[2] += c2;
            } else {
                e0 += gj * K[0]; e1 += gj * K[1]; e2 += gj * K[2];
                b0 += c0; b1 += c1; b2 += c2;
            }
        }
        if (variant != ORC_VARIANT_CPU) {
            E[0] += e0; E[1] += e1; E[2] += e2;
            B[0] += b0; B[1] += b1; B[2] += b2;
        }
    }
}

void orc_p2p(int variant, const double *pos, const double *mom, const int64_t *parindices,
             const int64_t *parlohis, int64_t npairs, const int64_t *pairs, double *ef, double *bf) {
    for (int64_t i = 0; i < npairs; ++i)
        p2p_pair(variant, pos, mom, parindices, parlohis, pairs[2 * i], pairs[2 * i + 1], ef, bf);
}

/* ------------------------------------------------------------------------- */
/* downward pass                                                              */
/* ------------------------------------------------------------------------- */

/* CPU: fmm/downwardpass.jl:3-45.  GPU: gpu_downwardpass.jl:4-74. */
static void l2l_child(int variant, int n, int64_t child, const int64_t *parents,
                      const double *bboxes, double *mef, double *mbf) {
    int m = n + 1, NN = m * m * m;
    int64_t parent = parents[child];
    double cxs[16], cys[16], czs[16], pxs[16], pys[16], pzs[16], wx[16], wy[16], wz[16];
    node_coords(variant, n, bboxes + 6 * child, cxs, cys, czs);
    node_coords(variant, n, bboxes + 6 * parent, pxs, pys, pzs);
    double *CE = mef + (int64_t)3 * NN * child, *CB = mbf + (int64_t)3 * NN * child;
    const double *PE = mef + (int64_t)3 * NN * parent, *PB = mbf + (int64_t)3 * NN * parent;
    for (int ck = 0; ck < m; ++ck) {
        weights(variant, czs[ck], pzs, n, wz);
        for (int cj = 0; cj < m; ++cj) {
            weights(variant, cys[cj], pys, n, wy);
            for (int ci = 0; ci < m; ++ci) {
                weights(variant, cxs[ci], pxs, n, wx);
                int c = ci + m * (cj + m * ck);
                double *E = CE + 3 * c, *B = CB + 3 * c;
                double e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
                for (int pk = 0; pk < m; ++pk)
                    for (int pj = 0; pj < m; ++pj)
                        for (int pi = 0; pi < m; ++pi) {
                            double w = wx[pi] * wy[pj] * wz[pk];
                            int a = pi + m * (pj + m * pk);
                            if (variant == ORC_VARIANT_CPU) {
                                E[0] += PE[3 * a] * w; E[1] += PE[3 * a + 1] * w; E[2] += PE[3 * a + 2] * w;
                                B[0] += PB[3 * a] * w; B[1] += PB[3 * a + 1] * w; B[2] += PB[3 * a + 2] * w;
                            } else {
                                e0 += PE[3 * a] * w; e1 += PE[3 * a + 1] * w; e2 += PE[3 * a + 2] * w;
                                b0 += PB[3 * a] * w; b1 += PB[3 * a + 1] * w; b2 += PB[3 * a + 2] * w;
                            }
                        }
                if (variant != ORC_VARIANT_CPU) {
                    E[0] += e0; E[1] += e1; E[2] += e2;
                    B[0] += b0; B[1] += b1; B[2] += b2;
                }
            }
        }
    }
}

void orc_l2l(int variant, int n, int64_t level, const int64_t *parents, const double *bboxes,
             double *mef, double *mbf) {
    int64_t c0 = ((int64_t)1 << level) - 1, c1 = ((int64_t)1 << (level + 1)) - 1;
    for (int64_t c = c0; c < c1; ++c) l2l_child(variant, n, c, parents, bboxes, mef, mbf);
}

/* CPU: fmm/downwardpass.jl:47-80.  GPU: gpu_downwardpass.jl:76-145. */
static void l2p_leaf(int variant, int n, const double *pos, const int64_t *parindices,
                     const int64_t *parlohis, const double *bboxes, int64_t node,
                     const double *mef, const double *mbf, double *ef, double *bf) {
    int m = n + 1, NN = m * m * m;
    double xs[16], ys[16], zs[16], wx[16], wy[16], wz[16];
    int64_t lo = parlohis[2 * node], hi = parlohis[2 * node + 1];
    node_coords(variant, n, bboxes + 6 * node, xs, ys, zs);
    const double *LE = mef + (int64_t)3 * NN * node, *LB = mbf + (int64_t)3 * NN * node;
    for (int64_t p = lo; p <= hi; ++p) {
        int64_t pi = parindices[p];
        const double *x = pos + 3 * pi;
        weights(variant, x[0], xs, n, wx);
        weights(variant, x[1], ys, n, wy);
        weights(variant, x[2], zs, n, wz);
        double *E = ef + 3 * pi, *B = bf + 3 * pi;
        double e0 = 0, e1 = 0, e2 = 0, b0 = 0, b1 = 0, b2 = 0;
        for (int k = 0; k < m; ++k)
            for (int j = 0; j < m; ++j)
                for (int i = 0; i < m; ++i) {
                    double w = wx[i] * wy[j] * wz[k];
                    int a = i + m * (j + m * k);
                    if (variant == ORC_VARIANT_CPU) {
                        E[0] += LE[3 * a] * w; E[1] += LE[3 * a + 1] * w; E[2] += LE[3 * a + 2] * w;
                        B[0] += LB[3 * a] * w; B[1] += LB[3 * a + 1] * w; B[2] += LB[3 * a + 2] * w;
                    } else {
                        e0 += LE[3 * a] * w; e1 += LE[3 * a + 1] * w; e2 += LE[3 * a + 2] * w;
                        b0 += LB[3 * a] * w; b1 += LB[3 * a + 1] * w; b2 += LB[3 * a + 2] * w;
                    }
                }
        if (variant != ORC_VARIANT_CPU) {
            E[0] += e0; E[1] += e1; E[2] += e2;
            B[0] += b0; B[1] += b1; B[2] += b2;
        }
    }
}

void orc_l2p(int variant, int n, const double *pos, const int64_t *parindices,
             const int64_t *parlohis, const double *bboxes, int64_t nleaf, const int64_t *leaf_ids,
             const double *mef, const double *mbf, double *ef, double *bf) {
    for (int64_t l = 0; l < nleaf; ++l)
        l2p_leaf(variant, n, pos, parindices, parlohis, bboxes, leaf_ids[l], mef, mbf, ef, bf);
}

/* ------------------------------------------------------------------------- */
/* drivers                                                                    */
/* ------------------------------------------------------------------------- */

/* Group pairs by target keeping list order (a stable counting sort of the
 * pair indices).  order[] lists pair indices; gptr[t]..gptr[t+1] are target t's. */
static void group_by_target(int64_t nc, int64_t npairs, const int64_t *pairs, int64_t *gptr,
                            int64_t *order) {
    memset(gptr, 0, sizeof(int64_t) * (size_t)(nc + 1));
    for (int64_t i = 0; i < npairs; ++i) gptr[pairs[2 * i] + 1]++;
    for (int64_t t = 0; t < nc; ++t) gptr[t + 1] += gptr[t];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
    memcpy(fill, gptr, sizeof(int64_t) * (size_t)(nc + 1));
    for (int64_t i = 0; i < npairs; ++i) order[fill[pairs[2 * i]]++] = i;
    free(fill);
}

/* update_particles_field.jl:40-64 (FMM) and :66-148 (FMMGPU). */
int orc_fmm(int variant, int64_t N, const double *pos, const double *mom, double charge,
            double lambda, int n, int64_t N0, double eta, const double *pavg_in, uint64_t seed,
            int nthreads, double *ef, double *bf, double *stats) {
    if (nthreads < 1) nthreads = 1;
    double t0 = now_s(), t1, t2, t3, t4, t5, t6;
    double pavg[3], stretch[3];
    if (pavg_in) { pavg[0] = pavg_in[0]; pavg[1] = pavg_in[1]; pavg[2] = pavg_in[2]; }
    else orc_pavg(N, mom, pavg);
    orc_stretch(pavg, stretch);

    int64_t ml = orc_maxlevel(N, N0);
    int64_t nc = orc_ncluster(N, N0);
    int m = n + 1, NN = m * m * m;
    int64_t *parindices = (int64_t *)malloc(sizeof(int64_t) * (size_t)N);
    int64_t *levels = (int64_t *)malloc(sizeof(int64_t) * (size_t)nc);
    int64_t *parlohis = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)nc);
    int64_t *parents = (int64_t *)malloc(sizeof(int64_t) * (size_t)nc);
    int64_t *children = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)nc);
    double *bboxes = (double *)malloc(sizeof(double) * 6 * (size_t)nc);
    double *gam = (double *)calloc((size_t)NN * (size_t)nc, sizeof(double));
    double *mmo = (double *)calloc((size_t)3 * NN * (size_t)nc, sizeof(double));
    double *mef = (double *)calloc((size_t)3 * NN * (size_t)nc, sizeof(double));
    double *mbf = (double *)calloc((size_t)3 * NN * (size_t)nc, sizeof(double));
    if (!parindices || !levels || !parlohis || !parents || !children || !bboxes || !gam || !mmo ||
        !mef || !mbf) {
        free(parindices); free(levels); free(parlohis); free(parents); free(children);
        free(bboxes); free(gam); free(mmo); free(mef); free(mbf);
        return -2;
    }
    int rc = orc_cluster_tree(N, pos, N0, stretch, seed, 1, parindices, levels, parlohis, parents,
                              children, bboxes);
    if (rc != 0) {
        free(parindices); free(levels); free(parlohis); free(parents); free(children);
        free(bboxes); free(gam); free(mmo); free(mef); free(mbf);
        return 1;
    }
    t1 = now_s();

    /* upward pass (upwardpass.jl:101-108 / update_particles_field.jl:100-110) */
    int64_t leaf0 = ((int64_t)1 << ml) - 1, nleaf = (int64_t)1 << ml;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) if (nthreads > 1)
    for (int64_t l = 0; l < nleaf; ++l)
        p2m_leaf(variant, n, pos, mom, parindices, parlohis, bboxes, leaf0 + l, gam, mmo);
    for (int64_t lev = ml; lev >= 1; --lev) {
        int64_t p0 = ((int64_t)1 << (lev - 1)) - 1, np = (int64_t)1 << (lev - 1);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) if (nthreads > 1)
        for (int64_t q = 0; q < np; ++q) m2m_parent(variant, n, p0 + q, children, bboxes, gam, mmo);
    }
    t2 = now_s();

    /* interaction lists */
    int64_t np2p = 0, nm2l = 0;
    orc_interaction_lists(nc, children, bboxes, stretch, eta, NULL, 0, &np2p, NULL, 0, &nm2l);
    int64_t *p2p = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(np2p > 0 ? np2p : 1));
    int64_t *m2l = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(nm2l > 0 ? nm2l : 1));
    orc_interaction_lists(nc, children, bboxes, stretch, eta, p2p, np2p, &np2p, m2l, nm2l, &nm2l);
    if (variant == ORC_VARIANT_GPU) {
        orc_sort_by_target(np2p, p2p);
        orc_sort_by_target(nm2l, m2l);
    }
    int64_t *gptr = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
    int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)((np2p > nm2l ? np2p : nm2l) + 1));
    t3 = now_s();

    for (int64_t i = 0; i < 3 * N; ++i) { ef[i] = 0.0; bf[i] = 0.0; }
    /* M2L (interaction.jl:3-46), grouped by target, list order kept per target */
    group_by_target(nc, nm2l, m2l, gptr, order);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) if (nthreads > 1)
    for (int64_t t = 0; t < nc; ++t)
        for (int64_t q = gptr[t]; q < gptr[t + 1]; ++q) {
            int64_t i = order[q];
            m2l_pair(variant, n, bboxes, gam, mmo, m2l[2 * i], m2l[2 * i + 1], pavg, mef, mbf);
        }
    t4 = now_s();
    /* P2P (interaction.jl:49-75) */
    group_by_target(nc, np2p, p2p, gptr, order);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) if (nthreads > 1)
    for (int64_t t = 0; t < nc; ++t)
        for (int64_t q = gptr[t]; q < gptr[t + 1]; ++q) {
            int64_t i = order[q];
            p2p_pair(variant, pos, mom, parindices, parlohis, p2p[2 * i], p2p[2 * i + 1], ef, bf);
        }
    t5 = now_s();

    /* downward pass (downwardpass.jl:82-89) */
    for (int64_t lev = 1; lev <= ml; ++lev) {
        int64_t c0 = ((int64_t)1 << lev) - 1, ncl = (int64_t)1 << lev;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) if (nthreads > 1)
        for (int64_t q = 0; q < ncl; ++q) l2l_child(variant, n, c0 + q, parents, bboxes, mef, mbf);
    }
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) if (nthreads > 1)
    for (int64_t l = 0; l < nleaf; ++l)
        l2p_leaf(variant, n, pos, parindices, parlohis, bboxes, leaf0 + l, mef, mbf, ef, bf);

    /* update_particles_field.jl:57-63 */
    double amp = ORC_RE * charge / lambda;
    for (int64_t i = 0; i < 3 * N; ++i) { ef[i] *= amp; bf[i] *= amp; }
    t6 = now_s();

    if (stats) {
        stats[0] = (double)ml; stats[1] = (double)nc; stats[2] = (double)nm2l; stats[3] = (double)np2p;
        stats[4] = t1 - t0; stats[5] = t2 - t1; stats[6] = t3 - t2; stats[7] = t4 - t3;
        stats[8] = t5 - t4; stats[9] = t6 - t5;
    }
    free(parindices); free(levels); free(parlohis); free(parents); free(children); free(bboxes);
    free(gam); free(mmo); free(mef); free(mbf); free(p2p); free(m2l); free(gptr); free(order);
    return 0;
}

/* update_particles_field.jl:21-38, for target particle i */
static void direct_one(int64_t N, const double *pos, const double *mom, double amp, int64_t i,
                       double *E, double *B) {
    const double *xi = pos + 3 * i;
    double K[3];
    E[0] = E[1] = E[2] = 0.0;
    B[0] = B[1] = B[2] = 0.0;
    for (int64_t j = 0; j < N; ++j) {
        const double *xj = pos + 3 * j, *u = mom + 3 * j;
        kernel_K(xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2], u, K);
        double ag = amp * sqrt(1.0 + (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        E[0] += ag * K[0]; E[1] += ag * K[1]; E[2] += ag * K[2];
        B[0] += amp * (u[1] * K[2] - u[2] * K[1]);
        B[1] += amp * (u[2] * K[0] - u[0] * K[2]);
        B[2] += amp * (u[0] * K[1] - u[1] * K[0]);
    }
}

void orc_bruteforce(int64_t N, const double *pos, const double *mom, double charge,
                    double lambda, int nthreads, double *ef, double *bf) {
    double amp = ORC_RE * charge / lambda;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) if (nthreads > 1)
    for (int64_t i = 0; i < N; ++i) direct_one(N, pos, mom, amp, i, ef + 3 * i, bf + 3 * i);
}

void orc_direct_targets(int64_t N, const double *pos, const double *mom, double charge,
                        double lambda, int64_t ntarget, const int64_t *targets, int nthreads,
                        double *ef, double *bf) {
    double amp = ORC_RE * charge / lambda;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
    for (int64_t q = 0; q < ntarget; ++q)
        direct_one(N, pos, mom, amp, targets[q], ef + 3 * q, bf + 3 * q);
}
