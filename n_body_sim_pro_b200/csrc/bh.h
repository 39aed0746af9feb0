/*
 * GPU Barnes-Hut: host orchestration (bh_host.c, C17) and kernel launchers
 * (bh.cu).  Internal; hidden visibility.
 *
 * Pipeline per force evaluation (all on one stream, no host synchronisation):
 *   bounds      FP64 bbox -> root cube (barnes_hut.c:453-483) + centre of mass
 *   keys        63-bit Morton keys, bit-exact with barnes_hut.c:286-305
 *   sort        stable LSD radix sort, 8 x 8-bit digits (same permutation as
 *               the reference's 3 x 21-bit LSD sort, barnes_hut.c:312-339)
 *   gather      float4 (x - com, m) in Morton order
 *   build       binary radix tree over the sorted keys (one thread per
 *               internal node), collapsed to a path-compressed octree with
 *               leaf buckets, laid out in depth-first order with skip links
 *   moments     bottom-up monopole + trace-free quadrupole in FP64
 *   walk        warp-cooperative stackless walk, opening test
 *               (2h)^2 < theta^2 d^2 to the cell centre of mass
 *   scatter     a[perm[s]] = G * a_sorted[s] in FP64
 */
#ifndef NBSP_BH_H
#define NBSP_BH_H

#include "n_body_sim_pro_cuda.h"
#include "internal.h"

#ifdef __cplusplus
extern "C" {
#endif

#define NBSP_BH_MAX_LEAF 64

typedef struct NbspBarnesHut NbspBarnesHut;

typedef struct NbspBarnesHutParams {
    double theta;
    double gravitational_constant;
    double softening_squared;
    int multipole_order;
    int leaf_capacity;
    int walk_mode;
    int opening;            /* NBSP_BH_OPENING_* */
    double tolerance;       /* alpha of the relative opening test; 0: geometric test alone */
    const void* correction; /* device network (mlp.cuh Net) or NULL */
    int quadrupoles;        /* the cells' quadrupoles and spread even for the monopole walk
                               (the correction's training reads them) */
} NbspBarnesHutParams;

/* The leapfrog of a device-resident step fused into an evaluation's first and
 * last passes, with kick_drift_kernel's arithmetic (integrator.c:64-83): with
 * vx set, the bounds pass first kicks v by half_dt * a (a: the accelerations in
 * the state, the previous evaluation's) and drifts x by dt * v, and the pass
 * that writes the new accelerations kicks v by half_dt * a.  vx NULL: none. */
typedef struct NbspLeapfrogFusion {
    double *vx, *vy, *vz;
    double half_dt, dt;
} NbspLeapfrogFusion;

typedef struct NbspBarnesHutState {
    double *x, *y, *z;  /* written only by a fused drift */
    const double* m;
    double *ax, *ay, *az;
    size_t n;
    NbspLeapfrogFusion leapfrog;
} NbspBarnesHutState;

/* Enqueue one full Barnes-Hut force evaluation; accelerations into s->ax/ay/az.
 * Statistics and phase timings of the evaluation are copied into *stats and
 * *timings by nbsp_bh_collect after the stream has been synchronised. */
NBSP_HIDDEN NBodySimProStatus nbsp_bh_accelerations(NbspBarnesHut** bh,
                                                    const NbspBarnesHutState* s,
                                                    const NbspBarnesHutParams* p, int* status,
                                                    cudaStream_t stream,
                                                    NBodySimProBarnesHutStats* stats,
                                                    NBodySimProCudaTimings* timings,
                                                    NBodySimProError* error);

/* After a stream synchronisation: fill stats / timings of the last evaluation
 * and the number of 32-target groups the interaction-list walk restarted. */
NBSP_HIDDEN void nbsp_bh_collect(NbspBarnesHut* bh, NBodySimProBarnesHutStats* stats,
                                 NBodySimProCudaTimings* timings, size_t* walk_restarts,
                                 size_t* corrected_cells);

/* Keys + sort only; copies the sorted keys / permutation / root to the host (synchronises). */
NBSP_HIDDEN NBodySimProStatus nbsp_bh_morton(NbspBarnesHut** bh, const NbspBarnesHutState* s,
                                             int* status, cudaStream_t stream,
                                             uint64_t* keys_sorted, uint64_t* permutation,
                                             double* root, NBodySimProError* error);

NBSP_HIDDEN void nbsp_bh_destroy(NbspBarnesHut* bh);

/* ---- kernel launchers (bh.cu) -------------------------------------------- */

/* bbox + centre of mass: geometry[0..3] = root centre xyz + half size (bit-exact
 * with the reference), geometry[4..6] = centre of mass.  partial >= 1024*10 doubles. */
NBSP_HIDDEN void nbsp_bh_bounds(double* x, double* y, double* z, const double* m, size_t n,
                                double* partial, double* geometry, int* status, const double* ax,
                                const double* ay, const double* az, int rms_of_a,
                                const NbspLeapfrogFusion* leapfrog, cudaStream_t stream);
/* geometry: root centre [0..2], half side [3], centre of mass [4..6], and with
 * rms_of_a the rms |a| [7] of (ax, ay, az) (the relative test's floor); with a
 * leapfrog fusion (NULL: none) the kick and drift come first and the rest is of
 * the drifted positions */

/* Morton keys, the identity index, the 8 digit histograms (into sort_scratch)
 * and the walk's float4 (x - c, y - c, z - c, m) with c the centre of mass, in
 * input order (`unsorted`, n entries). */
NBSP_HIDDEN void nbsp_bh_keys(const double* x, const double* y, const double* z, const double* m,
                              size_t n, const double* geometry, uint64_t* keys, uint32_t* index,
                              void* unsorted, uint32_t* sort_scratch, const double* ax,
                              const double* ay, const double* az, double tol_scale,
                              float* unsorted_tol, cudaStream_t stream);
/* (with unsorted_tol != NULL also the relative opening test's tolerance of each
 * particle, tol_scale |a| from the previous accelerations, +inf where |a| = 0) */

/* 32-bit words of sort scratch for n keys (digit histograms, pass bases, tile
 * tickets and look-back status words). */
NBSP_HIDDEN size_t nbsp_bh_sort_scratch_words(size_t n);

/* Stable LSD radix sort of (keys, index) by all 64 key bits, after nbsp_bh_keys
 * filled `sort_scratch` (nbsp_bh_sort_scratch_words(n) words) on the same stream.
 * `keys`/`index` are ping-ponged with `keys_alt`/`index_alt`; the sorted result
 * ends in the first pair. */
NBSP_HIDDEN void nbsp_bh_sort(uint64_t* keys, uint32_t* index, uint64_t* keys_alt,
                              uint32_t* index_alt, size_t n, uint32_t* sort_scratch, int* status,
                              cudaStream_t stream);

/* Flag NBSP_DEVICE_ERROR_DUPLICATE_POSITION when two particles share a position. */
NBSP_HIDDEN void nbsp_bh_duplicates(const uint64_t* keys, const uint32_t* perm, const double* x,
                                    const double* y, const double* z, size_t n, int* status,
                                    cudaStream_t stream);

/* pos4[s] = unsorted[perm[s]] (Morton order), tol[s] = unsorted_tol[perm[s]]. */
NBSP_HIDDEN void nbsp_bh_gather(const void* unsorted, const uint32_t* perm, size_t n, void* pos4,
                                const float* unsorted_tol, float* tol, int* status,
                                cudaStream_t stream);

/* Device-side layout of the tree build scratch; sized by nbsp_bh_tree_bytes. */
NBSP_HIDDEN size_t nbsp_bh_tree_bytes(size_t n);

/* Build the octree from the sorted keys. `tree` is nbsp_bh_tree_bytes(n) bytes. */
NBSP_HIDDEN void nbsp_bh_build(const uint64_t* keys, size_t n, int leaf_capacity, void* tree,
                               int* status, cudaStream_t stream);

/* Moments + walk-format node records.  order 1 or 2. */
/* Opening tests: the reference's (2h)^2 < theta^2 d^2 (barnes_hut.c:596-599), or
 * with the cell's centre-of-mass offset added, 2h / theta + shift < d. */
enum { NBSP_BH_OPENING_REFERENCE = 0, NBSP_BH_OPENING_OFFSET = 1 };

/* start_theta > 0 (the relative opening test is on): when the state has no
 * previous accelerations (rms |a_old| zero or not finite) the opening radii are
 * those of start_theta instead of theta.  The relative test then passes for
 * every target and the geometric test decides alone, so a fresh state is
 * opened at an ordinary angle rather than at the loose geometric bound the
 * relative test is run under. */
#define NBSP_BH_START_THETA 0.5

NBSP_HIDDEN void nbsp_bh_moments(const void* pos4, const uint64_t* keys, size_t n,
                                 const double* geometry, double theta, double start_theta,
                                 int opening, int quadrupoles, void* tree, int* status,
                                 cudaStream_t stream);

enum { NBSP_BH_WALK_STACKLESS = 0, NBSP_BH_WALK_LISTS = 1, NBSP_BH_WALK_SHARED = 2 };

/* Walk: a_sorted / G (double4 per target: the compensated sums combined in
 * FP64) and interaction counters.
 * mode NBSP_BH_WALK_STACKLESS: warp-coherent skip-link walk, per-target test;
 * mode NBSP_BH_WALK_LISTS: lane-parallel node tests against the warp's group
 * box, dense evaluation of gathered interaction lists. */
/* Per 32-target group, the cells a corrected walk lists for the network, and
 * the pipeline's rows: row r = offset[g] + k is cell k of group g. */
typedef struct NbspCorrectionLists {
    int* cells;     /* [groups * capacity] node ids, in the walk's order */
    int* count;     /* [groups] listed cells kept (<= capacity) */
    int* offset;    /* [groups + 1] exclusive prefix of count */
    float* centre;  /* [groups * 4] group centre x, y, z and group radius^2 */
    float* y;       /* [groups * capacity * 3] network outputs per row */
    int* row;       /* [groups * capacity * 2] (group, cell) of each row */
    int capacity;   /* cells per group; more are left to the plain monopole and counted */
} NbspCorrectionLists;

NBSP_HIDDEN void nbsp_bh_walk(const void* pos4, const float* tol, size_t n, const void* tree,
                              int order, int mode, const void* correction,
                              const NbspCorrectionLists* lists, float softening_squared,
                              const uint32_t* perm, void* acc, unsigned long long* counters,
                              int* status, cudaStream_t stream);
/* (acc: one double4 per particle, stored at the target's input index perm[s];
 * tol != NULL: every opening test also takes the relative test with the
 * per-target tolerances tol, Morton order; correction != NULL: the monopole
 * walk lists cells into `lists` for nbsp_bh_correct) */

/* After a corrected walk: the network on every listed (cell, group) row on the
 * tcgen05 tensor cores and the corrections added to the walk's result acc. */
NBSP_HIDDEN void nbsp_bh_correct(const void* pos4, size_t n, const void* tree,
                                 const void* correction, const NbspCorrectionLists* lists,
                                 const uint32_t* perm, void* acc, unsigned long long* counters,
                                 int* status, cudaStream_t stream);

/* Learned correction: training pairs (target, accepted cell) sampled with the
 * opening criterion `opening` at theta, their features and exact-sum labels, and
 * the column statistics written into the network's scaling tables (`net`). */
NBSP_HIDDEN void nbsp_bh_mlp_pairs(const void* pos4, size_t n, const void* tree, float theta,
                                   int opening, unsigned long long seed, int samples, int* target, int* cell,
                                   int* status, cudaStream_t stream);
NBSP_HIDDEN void nbsp_bh_mlp_labels(const void* pos4, size_t n, const void* tree,
                                    const int* target, const int* cell, int samples,
                                    float softening_squared, float* feat, float* lab, int* ok,
                                    cudaStream_t stream);
NBSP_HIDDEN void nbsp_bh_mlp_stats(const float* feat, const float* lab, const int* ok, int rows,
                                   void* net, cudaStream_t stream);

/* A context's freshly built Barnes-Hut tree, for training-pair generation. */
typedef struct NbspTreeRef {
    const void* pos4;
    const void* tree;
    size_t n;
    cudaStream_t stream;
    int* status;
    int opening; /* the criterion the tree's opening radii were built with */
} NbspTreeRef;

/* Build the tree of the context's resident state (one Barnes-Hut evaluation,
 * synchronised and checked) and describe it. */
NBSP_HIDDEN NBodySimProStatus nbsp_context_tree(NBodySimProCudaContext* ctx,
                                                const NBodySimProGravity* gravity,
                                                NbspTreeRef* out, NBodySimProError* error);

/* The device network of a correction object (NULL-safe). */
NBSP_HIDDEN const void* nbsp_correction_net(const NBodySimProCudaCorrection* correction);

/* The last evaluation's Morton-ordered float4 positions and tree scratch. */
NBSP_HIDDEN const void* nbsp_bh_positions(const NbspBarnesHut* bh);
NBSP_HIDDEN const void* nbsp_bh_tree(const NbspBarnesHut* bh);

/* a[i] = G * acc[i] (acc: double4 per particle in input order, as the walk
 * stores it) */
NBSP_HIDDEN void nbsp_bh_unsort(const void* acc, size_t n, double gravitational_constant,
                                double* ax, double* ay, double* az,
                                const NbspLeapfrogFusion* leapfrog, cudaStream_t stream);
/* (with a leapfrog fusion, NULL: none, v is then kicked by half_dt * a) */

/* Copy node_count, leaf_count and depth of the tree to counters[2..4]. */
NBSP_HIDDEN void nbsp_bh_tree_counts(const void* tree, size_t n, unsigned long long* counters,
                                     cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif
