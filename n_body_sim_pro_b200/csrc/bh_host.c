/*
 * Host orchestration of the GPU Barnes-Hut force evaluation (C17).
 * Buffer management and the order of the kernel launches of bh.cu; replaces
 * n_body_sim_pro_barnes_hut_compute_acceleration (src/c/barnes_hut/barnes_hut.c:638-690)
 * and its timing/statistics bookkeeping (:648-688, :255-283).
 */
#include "bh.h"

#include <cuda_runtime_api.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { BH_EVENTS = 8, BH_COUNTERS = 8 };
/* cells a corrected walk lists per 32-target group for the network; further
 * ones keep the plain monopole (counted in counters[7]) */
enum { BH_CORRECTION_CAPACITY = 512 };

struct NbspBarnesHut {
    size_t capacity;
    double* partial;    /* 1024 * 12 */
    double* geometry;   /* 8 */
    uint64_t* keys;
    uint64_t* keys_alt;
    uint32_t* index;
    uint32_t* index_alt;
    uint32_t* hist;
    void* pos4;
    void* tree;
    void* acc;          /* double4 per target, input order (the walk stores at perm[s]) */
    void* unsorted;     /* float4 positions in input order */
    float* tol_unsorted; /* relative opening test: tolerance per particle, input order */
    float* tol;          /* the same in Morton order */
    NbspCorrectionLists lists;          /* corrected walk (allocated on first use) */
    size_t lists_groups;
    unsigned long long* counters;       /* device */
    unsigned long long* host_counters;  /* pinned */
    cudaEvent_t events[BH_EVENTS];
    int timed;                          /* events hold a full evaluation */
};

static NBodySimProStatus bh_fail(NBodySimProError* error, NBodySimProStatus status,
                                 const char* file, int line, const char* message) {
    if (error != NULL) {
        error->status = status;
        error->source_file = file;
        error->source_line = line;
        snprintf(error->message, sizeof(error->message), "%s", message);
    }
    return status;
}

static NBodySimProStatus bh_cuda(NBodySimProError* error, cudaError_t code, const char* what,
                                 int line) {
    char text[256];
    snprintf(text, sizeof(text), "%s: %s", what, cudaGetErrorString(code));
    return bh_fail(error,
                   code == cudaErrorMemoryAllocation ? N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY
                                                     : N_BODY_SIM_PRO_STATUS_INVALID_STATE,
                   __FILE__, line, text);
}

#define BH_TRY(call)                                                     \
    do {                                                                 \
        cudaError_t bh_try_code = (call);                                \
        if (bh_try_code != cudaSuccess)                                  \
            return bh_cuda(error, bh_try_code, #call, __LINE__);         \
    } while (0)

static void release_lists(NbspBarnesHut* b) {
    cudaFree(b->lists.cells);
    cudaFree(b->lists.count);
    cudaFree(b->lists.offset);
    cudaFree(b->lists.centre);
    cudaFree(b->lists.y);
    cudaFree(b->lists.row);
    memset(&b->lists, 0, sizeof(b->lists));
    b->lists_groups = 0;
}

static NBodySimProStatus ensure_lists(NbspBarnesHut* b, size_t n, NBodySimProError* error) {
    const size_t groups = (n + 31) / 32;
    if (groups <= b->lists_groups) return N_BODY_SIM_PRO_STATUS_OK;
    release_lists(b);
    const size_t cap = BH_CORRECTION_CAPACITY;
    BH_TRY(cudaMalloc((void**)&b->lists.cells, groups * cap * sizeof(int)));
    BH_TRY(cudaMalloc((void**)&b->lists.count, groups * sizeof(int)));
    BH_TRY(cudaMalloc((void**)&b->lists.offset, (groups + 1) * sizeof(int)));
    BH_TRY(cudaMalloc((void**)&b->lists.centre, groups * 4 * sizeof(float)));
    BH_TRY(cudaMalloc((void**)&b->lists.y, groups * cap * 3 * sizeof(float)));
    BH_TRY(cudaMalloc((void**)&b->lists.row, groups * cap * 2 * sizeof(int)));
    b->lists.capacity = (int)cap;
    b->lists_groups = groups;
    return N_BODY_SIM_PRO_STATUS_OK;
}

static void release_buffers(NbspBarnesHut* b) {
    void* buffers[] = {b->partial, b->geometry, b->keys, b->keys_alt, b->index, b->index_alt,
                       b->hist, b->pos4, b->tree, b->acc, b->unsorted, b->tol_unsorted,
                       b->tol};
    for (size_t k = 0; k < sizeof(buffers) / sizeof(buffers[0]); ++k) cudaFree(buffers[k]);
    b->partial = b->geometry = NULL;
    b->keys = b->keys_alt = NULL;
    b->index = b->index_alt = NULL;
    b->hist = NULL;
    b->pos4 = b->tree = b->acc = b->unsorted = NULL;
    b->tol_unsorted = b->tol = NULL;
    b->capacity = 0;
}

void nbsp_bh_destroy(NbspBarnesHut* b) {
    if (b == NULL) return;
    release_buffers(b);
    release_lists(b);
    cudaFree(b->counters);
    cudaFreeHost(b->host_counters);
    for (int k = 0; k < BH_EVENTS; ++k)
        if (b->events[k] != NULL) cudaEventDestroy(b->events[k]);
    free(b);
}

static NBodySimProStatus ensure(NbspBarnesHut** handle, size_t n, NBodySimProError* error) {
    NbspBarnesHut* b = *handle;
    if (b == NULL) {
        b = (NbspBarnesHut*)calloc(1, sizeof(*b));
        if (b == NULL)
            return bh_fail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __FILE__, __LINE__,
                           "failed to allocate Barnes-Hut context");
        *handle = b;
        for (int k = 0; k < BH_EVENTS; ++k) BH_TRY(cudaEventCreate(&b->events[k]));
        BH_TRY(cudaMalloc((void**)&b->counters, BH_COUNTERS * sizeof(unsigned long long)));
        BH_TRY(cudaMallocHost((void**)&b->host_counters, BH_COUNTERS * sizeof(unsigned long long)));
        memset(b->host_counters, 0, BH_COUNTERS * sizeof(unsigned long long));
    }
    if (n <= b->capacity) return N_BODY_SIM_PRO_STATUS_OK;
    release_buffers(b);
    const size_t cap = n < 1024 ? 1024 : n;
    BH_TRY(cudaMalloc((void**)&b->partial, 1024 * 12 * sizeof(double)));
    BH_TRY(cudaMalloc((void**)&b->geometry, 8 * sizeof(double)));
    BH_TRY(cudaMalloc((void**)&b->keys, cap * sizeof(uint64_t)));
    BH_TRY(cudaMalloc((void**)&b->keys_alt, cap * sizeof(uint64_t)));
    BH_TRY(cudaMalloc((void**)&b->index, cap * sizeof(uint32_t)));
    BH_TRY(cudaMalloc((void**)&b->index_alt, cap * sizeof(uint32_t)));
    BH_TRY(cudaMalloc((void**)&b->hist, nbsp_bh_sort_scratch_words(cap) * sizeof(uint32_t)));
    BH_TRY(cudaMalloc(&b->pos4, cap * 16));
    BH_TRY(cudaMalloc(&b->tree, nbsp_bh_tree_bytes(cap)));
    BH_TRY(cudaMalloc(&b->acc, cap * 32));
    BH_TRY(cudaMalloc(&b->unsorted, cap * 16));
    BH_TRY(cudaMalloc((void**)&b->tol_unsorted, cap * sizeof(float)));
    BH_TRY(cudaMalloc((void**)&b->tol, cap * sizeof(float)));
    b->capacity = cap;
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* tol_scale > 0: also the relative opening test's tolerances (alpha / G). */
static NBodySimProStatus morton(NbspBarnesHut* b, const NbspBarnesHutState* s, double tol_scale,
                                int* status, cudaStream_t stream) {
    const int rel = tol_scale > 0.0;
    const NbspLeapfrogFusion* lf = s->leapfrog.vx != NULL ? &s->leapfrog : NULL;
    const int with_a = rel || lf != NULL;
    nbsp_bh_bounds(s->x, s->y, s->z, s->m, s->n, b->partial, b->geometry, status,
                   with_a ? s->ax : NULL, with_a ? s->ay : NULL, with_a ? s->az : NULL, rel, lf,
                   stream);
    cudaEventRecord(b->events[1], stream);
    nbsp_bh_keys(s->x, s->y, s->z, s->m, s->n, b->geometry, b->keys, b->index, b->unsorted,
                 b->hist, s->ax, s->ay, s->az, tol_scale, rel ? b->tol_unsorted : NULL, stream);
    cudaEventRecord(b->events[2], stream);
    nbsp_bh_sort(b->keys, b->index, b->keys_alt, b->index_alt, s->n, b->hist, status, stream);
    cudaEventRecord(b->events[3], stream);
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus nbsp_bh_accelerations(NbspBarnesHut** handle, const NbspBarnesHutState* s,
                                        const NbspBarnesHutParams* p, int* status,
                                        cudaStream_t stream, NBodySimProBarnesHutStats* stats,
                                        NBodySimProCudaTimings* timings,
                                        NBodySimProError* error) {
    NBodySimProStatus st = ensure(handle, s->n, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    NbspBarnesHut* b = *handle;
    const size_t n = s->n;
    if (n == 1) { /* a lone particle feels nothing; no tree to walk */
        BH_TRY(cudaMemsetAsync(s->ax, 0, sizeof(double), stream));
        BH_TRY(cudaMemsetAsync(s->ay, 0, sizeof(double), stream));
        BH_TRY(cudaMemsetAsync(s->az, 0, sizeof(double), stream));
        memset(stats, 0, sizeof(*stats));
        stats->node_count = stats->leaf_count = stats->maximum_depth = 1;
        b->timed = 0;
        return N_BODY_SIM_PRO_STATUS_OK;
    }
    BH_TRY(cudaMemsetAsync(b->counters, 0, BH_COUNTERS * sizeof(unsigned long long), stream));
    cudaEventRecord(b->events[0], stream);
    /* relative opening test: tolerance alpha |a_old| / G */
    const double g = fabs(p->gravitational_constant);
    const double tol_scale = p->tolerance > 0.0 ? (g > 0.0 ? p->tolerance / g : INFINITY) : 0.0;
    if (p->correction != NULL && (st = ensure_lists(b, n, error)) != N_BODY_SIM_PRO_STATUS_OK)
        return st;
    const int rel = tol_scale > 0.0;
    morton(b, s, tol_scale, status, stream);
    nbsp_bh_duplicates(b->keys, b->index, s->x, s->y, s->z, n, status, stream);
    nbsp_bh_gather(b->unsorted, b->index, n, b->pos4, rel ? b->tol_unsorted : NULL,
                   rel ? b->tol : NULL, status, stream);
    nbsp_bh_build(b->keys, n, p->leaf_capacity, b->tree, status, stream);
    cudaEventRecord(b->events[4], stream);
    nbsp_bh_moments(b->pos4, b->keys, n, b->geometry, p->theta,
                    rel ? fmin(p->theta, NBSP_BH_START_THETA) : 0.0, p->opening,
                    p->multipole_order == 2 || p->correction != NULL || p->quadrupoles, b->tree,
                    status, stream);
    cudaEventRecord(b->events[5], stream);
    nbsp_bh_walk(b->pos4, rel ? b->tol : NULL, n, b->tree, p->multipole_order, p->walk_mode,
                 p->correction, p->correction != NULL ? &b->lists : NULL,
                 (float)p->softening_squared, b->index, b->acc, b->counters, status, stream);
    if (p->correction != NULL)
        nbsp_bh_correct(b->pos4, n, b->tree, p->correction, &b->lists, b->index, b->acc,
                        b->counters, status, stream);
    cudaEventRecord(b->events[6], stream);
    nbsp_bh_unsort(b->acc, n, p->gravitational_constant, s->ax, s->ay, s->az,
                   s->leapfrog.vx != NULL ? &s->leapfrog : NULL, stream);
    nbsp_bh_tree_counts(b->tree, n, b->counters, stream);
    cudaEventRecord(b->events[7], stream);
    BH_TRY(cudaGetLastError());
    BH_TRY(cudaMemcpyAsync(b->host_counters, b->counters, BH_COUNTERS * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, stream));
    b->timed = 1;
    /* stats/timings are read after the caller synchronises */
    (void)stats;
    (void)timings;
    return N_BODY_SIM_PRO_STATUS_OK;
}

const void* nbsp_bh_positions(const NbspBarnesHut* b) { return b != NULL ? b->pos4 : NULL; }
const void* nbsp_bh_tree(const NbspBarnesHut* b) { return b != NULL ? b->tree : NULL; }

static double elapsed(const NbspBarnesHut* b, int from, int to) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, b->events[from], b->events[to]) != cudaSuccess) return 0.0;
    return (double)ms;
}

void nbsp_bh_collect(NbspBarnesHut* b, NBodySimProBarnesHutStats* stats,
                     NBodySimProCudaTimings* timings, size_t* walk_restarts,
                     size_t* corrected_cells) {
    if (b == NULL || !b->timed) return;
    const unsigned long long* c = b->host_counters;
    stats->accepted_approximations = (size_t)c[0];
    stats->exact_interactions = (size_t)c[1];
    stats->node_count = (size_t)c[2];
    stats->leaf_count = (size_t)c[3];
    stats->internal_node_count = (size_t)(c[2] - c[3]);
    stats->maximum_depth = (size_t)c[4];
    *walk_restarts = (size_t)c[5];
    *corrected_cells = (size_t)c[6];
    timings->bounds_ms = elapsed(b, 0, 1);
    timings->keys_ms = elapsed(b, 1, 2);
    timings->sort_ms = elapsed(b, 2, 3);
    timings->build_ms = elapsed(b, 3, 4);
    timings->moments_ms = elapsed(b, 4, 5);
    timings->walk_ms = elapsed(b, 5, 6);
    timings->integrate_ms = elapsed(b, 6, 7);
    timings->total_ms = elapsed(b, 0, 7);
    stats->build_time_seconds = (timings->total_ms - timings->walk_ms - timings->integrate_ms) * 1e-3;
    stats->evaluation_time_seconds = timings->walk_ms * 1e-3;
}

NBodySimProStatus nbsp_bh_morton(NbspBarnesHut** handle, const NbspBarnesHutState* s,
                                 int* status, cudaStream_t stream, uint64_t* keys_sorted,
                                 uint64_t* permutation, double* root, NBodySimProError* error) {
    NBodySimProStatus st = ensure(handle, s->n, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    NbspBarnesHut* b = *handle;
    const size_t n = s->n;
    cudaEventRecord(b->events[0], stream);
    morton(b, s, 0.0, status, stream);
    BH_TRY(cudaGetLastError());
    uint32_t* perm32 = NULL;
    if (permutation != NULL) {
        perm32 = (uint32_t*)malloc(n * sizeof(uint32_t));
        if (perm32 == NULL)
            return bh_fail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __FILE__, __LINE__,
                           "failed to allocate permutation copy");
    }
    cudaError_t code = cudaSuccess;
    if (keys_sorted != NULL)
        code = cudaMemcpyAsync(keys_sorted, b->keys, n * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                               stream);
    if (code == cudaSuccess && perm32 != NULL)
        code = cudaMemcpyAsync(perm32, b->index, n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               stream);
    if (code == cudaSuccess && root != NULL)
        code = cudaMemcpyAsync(root, b->geometry, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                               stream);
    if (code == cudaSuccess) code = cudaStreamSynchronize(stream);
    if (code == cudaSuccess && perm32 != NULL)
        for (size_t i = 0; i < n; ++i) permutation[i] = perm32[i];
    free(perm32);
    if (code != cudaSuccess) return bh_cuda(error, code, "morton order copy", __LINE__);
    b->timed = 0;
    return N_BODY_SIM_PRO_STATUS_OK;
}
