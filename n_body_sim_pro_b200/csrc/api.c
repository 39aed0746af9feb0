/*
 * C17 host layer of libn_body_sim_pro_cuda: argument checking and error
 * reporting with the reference engine's conventions, device memory and stream
 * management, the integrator loops, the all-pairs tile autotuner, and the
 * plugin entry points.  All GPU work is enqueued through the launchers of
 * internal.h on the context's stream.
 *
 * Reference behaviour followed here:
 *   error reporting       src/c/core/status.c:29-46 (n_body_sim_pro_error_set)
 *   argument checks       src/c/physics/gravity.c:19-23, integrator.c:145-156,
 *                         barnes_hut.c:446-451, :642-646
 *   integrator semantics  src/c/physics/integrator.c:15-172
 */
#include "n_body_sim_pro_cuda.h"

#include "bh.h"
#include "internal.h"

#include <cuda_runtime_api.h>
#include <math.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* errors                                                                     */
/* ------------------------------------------------------------------------- */

static NBodySimProStatus fail(NBodySimProError* error, NBodySimProStatus status, const char* file,
                              int line, const char* message) {
    if (error != NULL) {
        error->status = status;
        error->source_file = file;
        error->source_line = line;
        size_t length = message != NULL ? strlen(message) : 0;
        if (length >= sizeof(error->message)) length = sizeof(error->message) - 1;
        if (length > 0) memcpy(error->message, message, length);
        error->message[length] = '\0';
    }
    return status;
}

#define FAIL(status, message) fail(error, (status), __FILE__, __LINE__, (message))

static NBodySimProStatus cuda_fail(NBodySimProError* error, cudaError_t code, const char* what,
                                   const char* file, int line) {
    char text[256];
    snprintf(text, sizeof(text), "%s: %s", what, cudaGetErrorString(code));
    NBodySimProStatus status = N_BODY_SIM_PRO_STATUS_INVALID_STATE;
    if (code == cudaErrorMemoryAllocation) {
        status = N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY;
    } else if (code == cudaErrorNoDevice || code == cudaErrorInsufficientDriver ||
               code == cudaErrorNoKernelImageForDevice || code == cudaErrorInvalidDevice) {
        status = N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM;
    }
    return fail(error, status, file, line, text);
}

#define CUDA_TRY(call)                                                              \
    do {                                                                            \
        cudaError_t cuda_try_code = (call);                                         \
        if (cuda_try_code != cudaSuccess)                                           \
            return cuda_fail(error, cuda_try_code, #call, __FILE__, __LINE__);      \
    } while (0)

/* ------------------------------------------------------------------------- */
/* context                                                                    */
/* ------------------------------------------------------------------------- */

enum { TUNE_SLOTS = 16, EVENT_COUNT = 10 };

typedef struct TuneEntry {
    size_t n;       /* targets */
    size_t sources; /* padded sources */
    int zero_softening;
    NbspAllPairsShape shape;
} TuneEntry;

struct NBodySimProCudaContext {
    int device;
    int sm_count;
    cudaStream_t stream;
    cudaEvent_t events[EVENT_COUNT];

    size_t capacity;  /* particles the state buffers hold */
    size_t n;         /* resident particle count */
    size_t n_padded;  /* n rounded up to 256 (all-pairs source tiles) */
    int resident;     /* a state was uploaded */

    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
    void* packed;     /* float4[capacity_padded] */
    void* partial_hi; /* float4[partial_elems] */
    void* partial_lo;
    size_t partial_elems;
    double* centre;   /* device double[3] */
    double* scratch;  /* device doubles */
    size_t scratch_elems;
    double* out;      /* device double[16] */
    int* status;      /* device status bits */
    double* host_out; /* pinned double[16] */
    int* host_status; /* pinned int */

    double theta;
    int multipole_order;
    int leaf_capacity;
    int walk_mode;
    int opening;
    double tolerance; /* alpha of the relative opening test; 0: off */
    int relative_source; /* NBodySimProCudaRelativeSource */
    /* the last plugin call's result, still in ax/ay/az: its particle count and
     * the view's acceleration array it was copied to (0 / NULL: none) */
    size_t history_n;
    const double* history_ax;
    const void* correction; /* device network of the learned correction, or NULL */
    int tree_quadrupoles; /* the next build keeps every cell's quadrupole (training reads them) */
    NbspBarnesHut* bh;
    int bh_pending; /* a Barnes-Hut evaluation's stats await collection */

    NBodySimProBarnesHutStats stats;
    NBodySimProCudaTimings timings;
    size_t walk_restarts; /* groups the interaction-list walk handed to the stackless walk */
    size_t corrected_cells; /* (cell, group) pairs the correction network evaluated */

    TuneEntry tune[TUNE_SLOTS];
    int tune_count;
    int autotune;
};

static void release_state(NBodySimProCudaContext* c) {
    double** arrays[] = {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->ax, &c->ay, &c->az, &c->m};
    for (size_t k = 0; k < sizeof(arrays) / sizeof(arrays[0]); ++k) {
        cudaFree(*arrays[k]);
        *arrays[k] = NULL;
    }
    cudaFree(c->packed);
    c->packed = NULL;
    c->capacity = 0;
}

NBodySimProCudaContext* n_body_sim_pro_cuda_context_create(NBodySimProError* error) {
    int count = 0;
    cudaError_t code = cudaGetDeviceCount(&count);
    if (code != cudaSuccess || count == 0) {
        fail(error, N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM, __FILE__, __LINE__,
             code != cudaSuccess ? cudaGetErrorString(code) : "no CUDA device");
        return NULL;
    }
    NBodySimProCudaContext* c = (NBodySimProCudaContext*)calloc(1, sizeof(*c));
    if (c == NULL) {
        fail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __FILE__, __LINE__,
             "failed to allocate CUDA context");
        return NULL;
    }
    c->theta = 0.7;
    c->multipole_order = 1;
    c->leaf_capacity = 16;
    c->walk_mode = NBSP_BH_WALK_LISTS;
    c->opening = NBSP_BH_OPENING_REFERENCE;
    const char* tune = getenv("NBSP_AUTOTUNE");
    c->autotune = !(tune != NULL && tune[0] == '0');
    struct cudaDeviceProp prop;
    if ((code = cudaGetDevice(&c->device)) != cudaSuccess ||
        (code = cudaGetDeviceProperties(&prop, c->device)) != cudaSuccess) {
        free(c);
        cuda_fail(error, code, "cudaGetDeviceProperties", __FILE__, __LINE__);
        return NULL;
    }
    if (prop.major < 10) {
        free(c);
        fail(error, N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM, __FILE__, __LINE__,
             "this library is built for sm_100a (B200)");
        return NULL;
    }
    c->sm_count = prop.multiProcessorCount;
    code = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    for (int k = 0; k < EVENT_COUNT && code == cudaSuccess; ++k) code = cudaEventCreate(&c->events[k]);
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->centre, 3 * sizeof(double));
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->out, 16 * sizeof(double));
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->status, sizeof(int));
    if (code == cudaSuccess) code = cudaMallocHost((void**)&c->host_out, 16 * sizeof(double));
    if (code == cudaSuccess) code = cudaMallocHost((void**)&c->host_status, sizeof(int));
    if (code == cudaSuccess) code = cudaMemset(c->status, 0, sizeof(int));
    if (code != cudaSuccess) {
        cuda_fail(error, code, "context allocation", __FILE__, __LINE__);
        n_body_sim_pro_cuda_context_destroy(c);
        return NULL;
    }
    return c;
}

void n_body_sim_pro_cuda_context_destroy(NBodySimProCudaContext* c) {
    if (c == NULL) return;
    cudaSetDevice(c->device);
    if (c->stream != NULL) cudaStreamSynchronize(c->stream);
    nbsp_bh_destroy(c->bh);
    release_state(c);
    cudaFree(c->partial_hi);
    cudaFree(c->partial_lo);
    cudaFree(c->scratch);
    cudaFree(c->centre);
    cudaFree(c->out);
    cudaFree(c->status);
    cudaFreeHost(c->host_out);
    cudaFreeHost(c->host_status);
    for (int k = 0; k < EVENT_COUNT; ++k)
        if (c->events[k] != NULL) cudaEventDestroy(c->events[k]);
    if (c->stream != NULL) cudaStreamDestroy(c->stream);
    free(c);
}

void n_body_sim_pro_cuda_context_set_theta(NBodySimProCudaContext* c, double theta) {
    if (c != NULL) c->theta = theta;
}

double n_body_sim_pro_cuda_context_theta(const NBodySimProCudaContext* c) {
    return c != NULL ? c->theta : 0.0;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_multipole_order(NBodySimProCudaContext* c,
                                                                  int order,
                                                                  NBodySimProError* error) {
    if (c == NULL || (order != 1 && order != 2))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "multipole order must be 1 or 2");
    c->multipole_order = order;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_leaf_capacity(NBodySimProCudaContext* c,
                                                                int capacity,
                                                                NBodySimProError* error) {
    if (c == NULL || capacity < 1 || capacity > NBSP_BH_MAX_LEAF)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "leaf capacity must be in 1..64");
    c->leaf_capacity = capacity;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_walk(NBodySimProCudaContext* c, int walk,
                                                       NBodySimProError* error) {
    if (c == NULL || (walk != N_BODY_SIM_PRO_CUDA_WALK_STACKLESS &&
                      walk != N_BODY_SIM_PRO_CUDA_WALK_INTERACTION_LISTS &&
                      walk != N_BODY_SIM_PRO_CUDA_WALK_SHARED_TOP))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "unknown Barnes-Hut walk");
    c->walk_mode = walk == N_BODY_SIM_PRO_CUDA_WALK_STACKLESS   ? NBSP_BH_WALK_STACKLESS
                   : walk == N_BODY_SIM_PRO_CUDA_WALK_SHARED_TOP ? NBSP_BH_WALK_SHARED
                                                                 : NBSP_BH_WALK_LISTS;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_opening(NBodySimProCudaContext* c, int opening,
                                                          NBodySimProError* error) {
    if (c == NULL || (opening != N_BODY_SIM_PRO_CUDA_OPENING_REFERENCE &&
                      opening != N_BODY_SIM_PRO_CUDA_OPENING_OFFSET))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "unknown opening criterion");
    c->opening = opening == N_BODY_SIM_PRO_CUDA_OPENING_OFFSET ? NBSP_BH_OPENING_OFFSET
                                                              : NBSP_BH_OPENING_REFERENCE;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_relative_opening(NBodySimProCudaContext* c,
                                                                  double alpha,
                                                                  NBodySimProError* error) {
    if (c == NULL || !(alpha >= 0.0) || !isfinite(alpha))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "relative opening tolerance must be finite and >= 0");
    c->tolerance = alpha;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_relative_source(NBodySimProCudaContext* c,
                                                                 int source,
                                                                 NBodySimProError* error) {
    if (c == NULL) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context must not be null");
    if (source != N_BODY_SIM_PRO_CUDA_RELATIVE_FROM_VIEW &&
        source != N_BODY_SIM_PRO_CUDA_RELATIVE_FROM_CONTEXT)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "unknown relative-test source");
    c->relative_source = source;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_context_set_correction(
    NBodySimProCudaContext* c, const NBodySimProCudaCorrection* correction,
    NBodySimProError* error) {
    if (c == NULL) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context must not be null");
    c->correction = nbsp_correction_net(correction);
    return N_BODY_SIM_PRO_STATUS_OK;
}

int n_body_sim_pro_cuda_context_stats(const NBodySimProCudaContext* c,
                                      NBodySimProBarnesHutStats* stats) {
    if (c == NULL || stats == NULL) return 1;
    *stats = c->stats;
    return 0;
}

int n_body_sim_pro_cuda_context_timings(const NBodySimProCudaContext* c,
                                        NBodySimProCudaTimings* timings) {
    if (c == NULL || timings == NULL) return 1;
    *timings = c->timings;
    return 0;
}

size_t n_body_sim_pro_cuda_context_walk_restarts(const NBodySimProCudaContext* c) {
    return c == NULL ? 0 : c->walk_restarts;
}

size_t n_body_sim_pro_cuda_context_corrected_cells(const NBodySimProCudaContext* c) {
    return c == NULL ? 0 : c->corrected_cells;
}

const char* n_body_sim_pro_cuda_architecture(void) { return "sm_100a"; }

unsigned long long nbsp_kernel_launch_count = 0;

unsigned long long n_body_sim_pro_cuda_kernel_launches(void) {
    return __atomic_load_n(&nbsp_kernel_launch_count, __ATOMIC_RELAXED);
}

static size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

static NBodySimProStatus ensure_capacity(NBodySimProCudaContext* c, size_t n,
                                         NBodySimProError* error) {
    if (n > N_BODY_SIM_PRO_CUDA_MAX_PARTICLES)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "more particles than N_BODY_SIM_PRO_CUDA_MAX_PARTICLES");
    if (n <= c->capacity && c->packed != NULL) return N_BODY_SIM_PRO_STATUS_OK;
    release_state(c);
    const size_t cap = n < 256 ? 256 : n;
    double** arrays[] = {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->ax, &c->ay, &c->az, &c->m};
    for (size_t k = 0; k < sizeof(arrays) / sizeof(arrays[0]); ++k) {
        CUDA_TRY(cudaMalloc((void**)arrays[k], cap * sizeof(double)));
    }
    CUDA_TRY(cudaMalloc(&c->packed, round_up(cap, 256) * 16));
    c->capacity = cap;
    return N_BODY_SIM_PRO_STATUS_OK;
}

static NBodySimProStatus ensure_scratch(NBodySimProCudaContext* c, size_t doubles,
                                        NBodySimProError* error) {
    if (doubles <= c->scratch_elems) return N_BODY_SIM_PRO_STATUS_OK;
    cudaFree(c->scratch);
    c->scratch = NULL;
    c->scratch_elems = 0;
    CUDA_TRY(cudaMalloc((void**)&c->scratch, doubles * sizeof(double)));
    c->scratch_elems = doubles;
    return N_BODY_SIM_PRO_STATUS_OK;
}

static NBodySimProStatus ensure_partials(NBodySimProCudaContext* c, size_t elems,
                                         NBodySimProError* error) {
    if (elems <= c->partial_elems) return N_BODY_SIM_PRO_STATUS_OK;
    cudaFree(c->partial_hi);
    cudaFree(c->partial_lo);
    c->partial_hi = c->partial_lo = NULL;
    c->partial_elems = 0;
    CUDA_TRY(cudaMalloc(&c->partial_hi, elems * 16));
    CUDA_TRY(cudaMalloc(&c->partial_lo, elems * 16));
    c->partial_elems = elems;
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* Read and clear the device status word; map it to a status code. */
static NBodySimProStatus check_device_status(NBodySimProCudaContext* c, NBodySimProError* error) {
    CUDA_TRY(cudaMemcpyAsync(c->host_status, c->status, sizeof(int), cudaMemcpyDeviceToHost,
                             c->stream));
    CUDA_TRY(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->bh_pending) {
        nbsp_bh_collect(c->bh, &c->stats, &c->timings, &c->walk_restarts, &c->corrected_cells);
        c->bh_pending = 0;
    }
    const int bits = *c->host_status;
    if (bits & NBSP_DEVICE_ERROR_NONFINITE_POSITION)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "non-finite particle position");
    if (bits & NBSP_DEVICE_ERROR_DUPLICATE_POSITION) /* barnes_hut.c:149-153 */
        return FAIL(N_BODY_SIM_PRO_STATUS_OVERFLOW,
                    "Barnes-Hut tree exceeded maximum depth (duplicate positions?)");
    if (bits & NBSP_DEVICE_ERROR_TREE_INCONSISTENT)
        return FAIL(N_BODY_SIM_PRO_STATUS_OVERFLOW, "Barnes-Hut tree build exceeded its bounds");
    if (bits & NBSP_DEVICE_ERROR_WALK_LIMIT)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "Barnes-Hut walk exceeded its step limit");
    if (bits & NBSP_DEVICE_ERROR_ENSEMBLE_LIMIT)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "ensemble kernel exceeded its limits");
    if (bits & NBSP_DEVICE_ERROR_MMA_TIMEOUT)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE,
                    "correction network: a tensor-core product did not complete in time");
    if (bits != 0) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "unknown device status");
    return N_BODY_SIM_PRO_STATUS_OK;
}

static NBodySimProStatus check_gravity(const NBodySimProGravity* g, NBodySimProError* error) {
    if (!isfinite(g->gravitational_constant) || !isfinite(g->softening_squared) ||
        g->softening_squared < 0.0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "gravity parameters must be finite with non-negative softening");
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* ------------------------------------------------------------------------- */
/* all-pairs tile autotuner                                                   */
/* ------------------------------------------------------------------------- */

static const NbspAllPairsShape kShapes[] = {
    {128, 4, 1, 0, 0}, {128, 2, 1, 0, 0}, {256, 2, 1, 0, 0}, {64, 8, 1, 0, 0},
    {128, 8, 1, 0, 0}, {64, 4, 1, 0, 0},  {256, 4, 1, 0, 0}, {64, 8, 1, 1, 0},
    {128, 4, 1, 1, 0}, {128, 8, 1, 1, 0}, {256, 4, 1, 1, 0}, {64, 4, 1, 1, 0},
    {128, 2, 1, 1, 0}, {256, 2, 1, 1, 0}, {256, 2, 1, 1, 4}, {128, 4, 1, 1, 6},
};

/* Source chunks so that (target blocks x chunks) fills whole waves of resident
 * CTAs: the busiest CTA slot's sources (chunks end on 8-source boundaries) against
 * the average, less a small cost per chunk (one more partial per target). */
static NbspAllPairsShape fit_chunks(const NBodySimProCudaContext* c, NbspAllPairsShape s,
                                    size_t n_targets, size_t n_sources_padded) {
    const size_t per_cta = (size_t)s.block * (size_t)s.per_thread;
    const size_t target_blocks = (n_targets + per_cta - 1) / per_cta;
    int resident = nbsp_allpairs_resident_ctas(s);
    if (resident < 1) resident = 1;
    const size_t slots = (size_t)c->sm_count * (size_t)resident;
    size_t best_chunks = 1;
    double best_eff = 0.0;
    for (size_t chunks = 1; chunks <= 64; ++chunks) {
        const size_t len = nbsp_allpairs_chunk_len(n_sources_padded, (int)chunks);
        if (chunks > 1 && len < 2 * (size_t)s.block) break;
        const size_t ctas = target_blocks * chunks;
        const size_t waves = (ctas + slots - 1) / slots;
        const double work = (double)target_blocks * (double)n_sources_padded;
        const double span = (double)waves * (double)len * (double)slots;
        const double eff = work / span - 0.002 * (double)chunks;
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best_chunks = chunks;
        }
    }
    s.chunks = (int)best_chunks;
    return s;
}

/* The fastest kernel shape for n_targets targets (`targets`) against
 * n_sources_padded packed sources (`sources`), timed once per size pair on
 * the live buffers and cached. */
static NbspAllPairsShape choose_shape_for(NBodySimProCudaContext* c, const void* sources,
                                          size_t n_sources_padded, const void* targets,
                                          size_t n_targets, float eps2) {
    const int zero = eps2 == 0.f;
    for (int k = 0; k < c->tune_count; ++k)
        if (c->tune[k].n == n_targets && c->tune[k].sources == n_sources_padded &&
            c->tune[k].zero_softening == zero)
            return c->tune[k].shape;
    NbspAllPairsShape best = fit_chunks(c, kShapes[0], n_targets, n_sources_padded);
    if (c->autotune && n_targets >= 2048) {
        float best_ms = 1e30f;
        const int shapes = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
        for (int k = 0; k < shapes; ++k) {
            if (!nbsp_allpairs_shape_supported(kShapes[k])) continue;
            NbspAllPairsShape s = fit_chunks(c, kShapes[k], n_targets, n_sources_padded);
            if ((size_t)s.chunks * n_targets > c->partial_elems) continue;
            float fastest = 1e30f; /* best of 4 timed launches after one warm-up */
            for (int rep = 0; rep < 5; ++rep) {
                cudaEventRecord(c->events[8], c->stream);
                nbsp_allpairs_force_targets(sources, n_sources_padded, targets, n_targets, eps2,
                                            s, c->partial_hi, c->partial_lo, c->stream);
                cudaEventRecord(c->events[9], c->stream);
                cudaEventSynchronize(c->events[9]);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, c->events[8], c->events[9]);
                if (rep > 0 && ms < fastest) fastest = ms;
            }
            if (fastest < best_ms) {
                best_ms = fastest;
                best = s;
            }
        }
    }
    const int slot = c->tune_count < TUNE_SLOTS ? c->tune_count++ : (int)(n_targets % TUNE_SLOTS);
    c->tune[slot].n = n_targets;
    c->tune[slot].sources = n_sources_padded;
    c->tune[slot].zero_softening = zero;
    c->tune[slot].shape = best;
    return best;
}

static NbspAllPairsShape choose_shape(NBodySimProCudaContext* c, size_t n, float eps2) {
    return choose_shape_for(c, c->packed, c->n_padded, c->packed, n, eps2);
}

/* Partial buffers big enough for any candidate shape at n (<= 64 chunks). */
static NBodySimProStatus prepare_allpairs(NBodySimProCudaContext* c, size_t n,
                                          NBodySimProError* error) {
    const size_t want = n * 64;
    const size_t cap_bytes = (size_t)1 << 30; /* at most 2 x 1 GiB of partials */
    size_t elems = want * 16 > cap_bytes ? cap_bytes / 16 : want;
    if (elems < n) elems = n;
    return ensure_partials(c, elems, error);
}

/* forces of the resident, already packed state -> c->ax/ay/az (FP64) */
static NBodySimProStatus allpairs_accelerations(NBodySimProCudaContext* c,
                                                const NBodySimProGravity* g,
                                                NBodySimProError* error) {
    const size_t n = c->n;
    NBodySimProStatus st = prepare_allpairs(c, n, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    const float eps2 = (float)g->softening_squared;
    NbspAllPairsShape s = choose_shape(c, n, eps2);
    if ((size_t)s.chunks * n > c->partial_elems) s.chunks = (int)(c->partial_elems / n);
    nbsp_allpairs_force(c->packed, n, c->n_padded, eps2, s, c->partial_hi, c->partial_lo,
                        c->stream);
    nbsp_allpairs_finalize(c->partial_hi, c->partial_lo, n, s.chunks, g->gravitational_constant,
                           c->ax, c->ay, c->az, c->stream);
    CUDA_TRY(cudaGetLastError());
    return N_BODY_SIM_PRO_STATUS_OK;
}

static NBodySimProStatus pack_state(NBodySimProCudaContext* c, NBodySimProError* error) {
    NBodySimProStatus st = ensure_scratch(c, 11 * 1024, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    nbsp_centre_of_mass(c->x, c->y, c->z, c->m, c->n, c->scratch, c->centre, c->stream);
    nbsp_pack_relative(c->x, c->y, c->z, c->m, c->n, c->n_padded, c->centre, c->packed, c->status,
                       c->stream);
    CUDA_TRY(cudaGetLastError());
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* One force evaluation of the resident state with `algorithm`; with a
 * leapfrog fusion (Barnes-Hut only; NULL: none) the step's opening kick and
 * drift and its closing kick run inside the evaluation's first and last passes. */
static NBodySimProStatus resident_accelerations_fused(NBodySimProCudaContext* c,
                                                      const NBodySimProGravity* g,
                                                      NBodySimProCudaAlgorithm algorithm,
                                                      const NbspLeapfrogFusion* leapfrog,
                                                      NBodySimProError* error) {
    if (c->n == 0) return N_BODY_SIM_PRO_STATUS_OK;
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT) {
        NbspBarnesHutParams p;
        p.theta = c->theta;
        p.gravitational_constant = g->gravitational_constant;
        p.softening_squared = g->softening_squared;
        p.multipole_order = c->multipole_order;
        p.leaf_capacity = c->leaf_capacity;
        p.walk_mode = c->walk_mode;
        p.opening = c->opening;
        p.tolerance = c->tolerance;
        p.correction = c->correction;
        p.quadrupoles = c->tree_quadrupoles;
        NbspBarnesHutState s = {c->x, c->y, c->z, c->m, c->ax, c->ay, c->az, c->n,
                                {NULL, NULL, NULL, 0.0, 0.0}};
        if (leapfrog != NULL) s.leapfrog = *leapfrog;
        c->bh_pending = 1;
        return nbsp_bh_accelerations(&c->bh, &s, &p, c->status, c->stream, &c->stats,
                                     &c->timings, error);
    }
    NBodySimProStatus st = pack_state(c, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    return allpairs_accelerations(c, g, error);
}

/* One force evaluation of the resident state with `algorithm`. */
static NBodySimProStatus resident_accelerations(NBodySimProCudaContext* c,
                                                const NBodySimProGravity* g,
                                                NBodySimProCudaAlgorithm algorithm,
                                                NBodySimProError* error) {
    return resident_accelerations_fused(c, g, algorithm, NULL, error);
}

/* ------------------------------------------------------------------------- */
/* plugin force functions                                                     */
/* ------------------------------------------------------------------------- */

static _Atomic(NBodySimProCudaContext*) g_default_context = NULL;

/* The context of a NULL `context` argument, created by the first such call;
 * when two threads make that call at once, one creation wins and the other
 * is destroyed. */
static NBodySimProCudaContext* context_or_default(void* context, NBodySimProError* error) {
    if (context != NULL) return (NBodySimProCudaContext*)context;
    NBodySimProCudaContext* c = atomic_load(&g_default_context);
    if (c != NULL) return c;
    NBodySimProCudaContext* made = n_body_sim_pro_cuda_context_create(error);
    if (made == NULL) return NULL;
    NBodySimProCudaContext* expected = NULL;
    if (atomic_compare_exchange_strong(&g_default_context, &expected, made)) return made;
    n_body_sim_pro_cuda_context_destroy(made);
    return expected;
}

static NBodySimProStatus copy_in(NBodySimProCudaContext* c, const NBodySimProParticleSystemView* v,
                                 int everything, NBodySimProError* error) {
    const size_t n = v->particle_count;
    const size_t bytes = n * sizeof(double);
    struct {
        double* dst;
        const double* src;
        int always;
    } copies[] = {
        {c->x, v->positions_x, 1},      {c->y, v->positions_y, 1},
        {c->z, v->positions_z, 1},      {c->m, v->masses, 1},
        {c->vx, v->velocities_x, 0},    {c->vy, v->velocities_y, 0},
        {c->vz, v->velocities_z, 0},    {c->ax, v->accelerations_x, 0},
        {c->ay, v->accelerations_y, 0}, {c->az, v->accelerations_z, 0},
    };
    for (size_t k = 0; k < sizeof(copies) / sizeof(copies[0]); ++k) {
        if (!copies[k].always && !everything) continue;
        if (copies[k].src == NULL) {
            if (copies[k].always) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                                              "view position and mass arrays must not be null");
            CUDA_TRY(cudaMemsetAsync(copies[k].dst, 0, bytes, c->stream));
            continue;
        }
        CUDA_TRY(cudaMemcpyAsync(copies[k].dst, copies[k].src, bytes, cudaMemcpyHostToDevice,
                                 c->stream));
    }
    return N_BODY_SIM_PRO_STATUS_OK;
}

static NBodySimProStatus copy_accelerations_out(NBodySimProCudaContext* c,
                                                const NBodySimProParticleSystemView* v,
                                                NBodySimProError* error) {
    const size_t bytes = v->particle_count * sizeof(double);
    if (v->accelerations_x == NULL || v->accelerations_y == NULL || v->accelerations_z == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "view acceleration arrays must not be null");
    CUDA_TRY(cudaMemcpyAsync(v->accelerations_x, c->ax, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(v->accelerations_y, c->ay, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(v->accelerations_z, c->az, bytes, cudaMemcpyDeviceToHost, c->stream));
    return N_BODY_SIM_PRO_STATUS_OK;
}

static NBodySimProStatus view_force(const NBodySimProParticleSystemView* view,
                                    const NBodySimProGravity* gravity, void* context,
                                    NBodySimProCudaAlgorithm algorithm, NBodySimProError* error) {
    if (view == NULL || gravity == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "view and gravity parameters must not be null");
    NBodySimProStatus st = check_gravity(gravity, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT && view->particle_count == 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "cannot build a Barnes-Hut tree for an empty system");
    NBodySimProCudaContext* c = context_or_default(context, error);
    if (c == NULL) return error != NULL ? error->status : N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM;
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t n = view->particle_count;
    if (n == 0) return N_BODY_SIM_PRO_STATUS_OK;
    /* Every other call that writes ax/ay/az needs or makes a resident state,
     * so with none since the last plugin call its result is still there. */
    const int reuse = algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT &&
                      c->tolerance > 0.0 &&
                      c->relative_source == N_BODY_SIM_PRO_CUDA_RELATIVE_FROM_CONTEXT &&
                      !c->resident && c->history_n == n &&
                      c->history_ax == view->accelerations_x;
    c->history_n = 0;
    c->history_ax = NULL;
    if ((st = ensure_capacity(c, n, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    c->n = n;
    c->n_padded = round_up(n, 256);
    c->resident = 0; /* the plugin path only stages positions and masses */
    if ((st = copy_in(c, view, 0, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT && c->tolerance > 0.0 && !reuse) {
        /* the relative opening test reads the view's previous accelerations */
        const size_t bytes = n * sizeof(double);
        double* dst[3] = {c->ax, c->ay, c->az};
        const double* src[3] = {view->accelerations_x, view->accelerations_y,
                                view->accelerations_z};
        for (int k = 0; k < 3; ++k) {
            if (src[k] != NULL)
                CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], bytes, cudaMemcpyHostToDevice,
                                         c->stream));
            else
                CUDA_TRY(cudaMemsetAsync(dst[k], 0, bytes, c->stream));
        }
    }
    CUDA_TRY(cudaEventRecord(c->events[0], c->stream));
    if ((st = resident_accelerations(c, gravity, algorithm, error)) != N_BODY_SIM_PRO_STATUS_OK)
        return st;
    CUDA_TRY(cudaEventRecord(c->events[1], c->stream));
    if ((st = copy_accelerations_out(c, view, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    if ((st = check_device_status(c, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    c->history_n = n;
    c->history_ax = view->accelerations_x;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->events[0], c->events[1]);
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS) {
        memset(&c->timings, 0, sizeof(c->timings));
        c->timings.walk_ms = ms;
    }
    c->timings.total_ms = ms;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_gravity_compute_acceleration_cuda(
    const NBodySimProParticleSystemView* view, const NBodySimProGravity* gravity, void* context,
    NBodySimProError* error) {
    return view_force(view, gravity, context, N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS, error);
}

NBodySimProStatus n_body_sim_pro_barnes_hut_compute_acceleration_cuda(
    const NBodySimProParticleSystemView* view, const NBodySimProGravity* gravity, void* context,
    NBodySimProError* error) {
    return view_force(view, gravity, context, N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT, error);
}

/* ------------------------------------------------------------------------- */
/* device-resident API                                                        */
/* ------------------------------------------------------------------------- */

NBodySimProStatus n_body_sim_pro_cuda_upload(NBodySimProCudaContext* c,
                                             const NBodySimProParticleSystemView* view,
                                             NBodySimProError* error) {
    if (c == NULL || view == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context and view must not be null");
    CUDA_TRY(cudaSetDevice(c->device));
    NBodySimProStatus st = ensure_capacity(c, view->particle_count, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    c->n = view->particle_count;
    c->n_padded = round_up(c->n, 256);
    if (c->n > 0 && (st = copy_in(c, view, 1, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->resident = 1;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_preset_generate_parallel(
    NBodySimProCudaContext* c, NBodySimProSimulationPreset preset,
    const NBodySimProPresetParameters* parameters, NBodySimProError* error) {
    /* presets_parallel.c:314-326 argument checks */
    if (c == NULL || parameters == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "particle system and parameters must not be null");
    const size_t n = parameters->particle_count;
    if ((int)preset < 0 || (int)preset >= (int)N_BODY_SIM_PRO_PRESET_COUNT)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "unknown preset");
    if (preset == N_BODY_SIM_PRO_PRESET_TWO_BODY && n != 2) /* :343-347 */
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "two_body preset requires exactly 2 particles");
    if (n == 0 || (preset == N_BODY_SIM_PRO_PRESET_GALAXY_COLLISION && n < 2) ||
        (preset == N_BODY_SIM_PRO_PRESET_TRIPLE_GALAXY && n < 3))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "too few particles for the preset");
    CUDA_TRY(cudaSetDevice(c->device));
    NBodySimProStatus st = ensure_capacity(c, n, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if ((st = ensure_scratch(c, nbsp_preset_scratch_doubles(n), error)) != N_BODY_SIM_PRO_STATUS_OK)
        return st;
    c->n = n;
    c->n_padded = round_up(n, 256);
    /* unfilled tails (collision, triple) and accelerations start at zero */
    double* arrays[] = {c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, c->m};
    for (size_t k = 0; k < sizeof(arrays) / sizeof(arrays[0]); ++k)
        CUDA_TRY(cudaMemsetAsync(arrays[k], 0, n * sizeof(double), c->stream));
    if (nbsp_preset_generate((int)preset, n, parameters->random_seed, c->x, c->y, c->z, c->vx,
                             c->vy, c->vz, c->m, c->scratch, c->stream) != 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "too few particles for the preset");
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->resident = 1;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_plummer_collision_generate(
    NBodySimProCudaContext* c, size_t count, uint64_t seed, double scale_radius,
    double separation, double relative_speed, NBodySimProError* error) {
    if (c == NULL) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context must not be null");
    if (count < 2) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "too few particles for the preset");
    if (!(scale_radius > 0.0) || !isfinite(scale_radius) || !isfinite(separation) ||
        !isfinite(relative_speed))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "scale radius must be positive, separation and speed finite");
    CUDA_TRY(cudaSetDevice(c->device));
    NBodySimProStatus st = ensure_capacity(c, count, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if ((st = ensure_scratch(c, nbsp_preset_scratch_doubles(count), error)) != N_BODY_SIM_PRO_STATUS_OK)
        return st;
    c->n = count;
    c->n_padded = round_up(count, 256);
    double* acc[] = {c->ax, c->ay, c->az};
    for (size_t k = 0; k < 3; ++k)
        CUDA_TRY(cudaMemsetAsync(acc[k], 0, count * sizeof(double), c->stream));
    if (nbsp_plummer_collision_generate(count, seed, scale_radius, separation, relative_speed,
                                        c->x, c->y, c->z, c->vx, c->vy, c->vz, c->m, c->scratch,
                                        c->stream) != 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "too few particles for the preset");
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->resident = 1;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_download(NBodySimProCudaContext* c,
                                               const NBodySimProParticleSystemView* view,
                                               NBodySimProError* error) {
    if (c == NULL || view == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context and view must not be null");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    if (view->particle_count != c->n)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "view particle count differs from the resident state");
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t bytes = c->n * sizeof(double);
    struct {
        double* dst;
        const double* src;
    } copies[] = {
        {view->positions_x, c->x},      {view->positions_y, c->y},
        {view->positions_z, c->z},      {view->velocities_x, c->vx},
        {view->velocities_y, c->vy},    {view->velocities_z, c->vz},
        {view->accelerations_x, c->ax}, {view->accelerations_y, c->ay},
        {view->accelerations_z, c->az}, {view->masses, c->m},
    };
    for (size_t k = 0; k < sizeof(copies) / sizeof(copies[0]); ++k) {
        if (copies[k].dst == NULL || bytes == 0) continue;
        CUDA_TRY(cudaMemcpyAsync(copies[k].dst, copies[k].src, bytes, cudaMemcpyDeviceToHost,
                                 c->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_compute_acceleration(NBodySimProCudaContext* c,
                                                           const NBodySimProGravity* gravity,
                                                           NBodySimProCudaAlgorithm algorithm,
                                                           NBodySimProError* error) {
    if (c == NULL || gravity == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context and gravity must not be null");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    NBodySimProStatus st = check_gravity(gravity, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT && c->n == 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "cannot build a Barnes-Hut tree for an empty system");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaEventRecord(c->events[0], c->stream));
    if ((st = resident_accelerations(c, gravity, algorithm, error)) != N_BODY_SIM_PRO_STATUS_OK)
        return st;
    CUDA_TRY(cudaEventRecord(c->events[1], c->stream));
    if ((st = check_device_status(c, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->events[0], c->events[1]);
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS) {
        memset(&c->timings, 0, sizeof(c->timings));
        c->timings.walk_ms = ms;
    }
    c->timings.total_ms = ms;
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* Leapfrog / Verlet on all-pairs: opening kick+drift, then per step one force
 * pass and one fused epilogue (closing kick of this step + opening kick and
 * drift of the next + repack). */
static NBodySimProStatus advance_allpairs_kdk(NBodySimProCudaContext* c,
                                              const NBodySimProGravity* g, double dt, int steps,
                                              NBodySimProError* error) {
    const size_t n = c->n;
    const double h = 0.5 * dt;
    NBodySimProStatus st = prepare_allpairs(c, n, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if ((st = ensure_scratch(c, 11 * 1024, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    nbsp_kick_drift(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, n, h, dt,
                    c->stream);
    nbsp_centre_of_mass(c->x, c->y, c->z, c->m, n, c->scratch, c->centre, c->stream);
    nbsp_pack_relative(c->x, c->y, c->z, c->m, n, c->n_padded, c->centre, c->packed, c->status,
                       c->stream);
    const float eps2 = (float)g->softening_squared;
    NbspAllPairsShape s = choose_shape(c, n, eps2);
    if ((size_t)s.chunks * n > c->partial_elems) s.chunks = (int)(c->partial_elems / n);
    for (int step = 0; step < steps; ++step) {
        const int last = step + 1 == steps;
        if (last) cudaEventRecord(c->events[2], c->stream);
        nbsp_allpairs_force(c->packed, n, c->n_padded, eps2, s, c->partial_hi, c->partial_lo,
                            c->stream);
        if (last) cudaEventRecord(c->events[3], c->stream);
        if (step + 1 < steps) {
            nbsp_allpairs_finalize_kick_kick_drift_pack(
                c->partial_hi, c->partial_lo, n, c->n_padded, s.chunks, g->gravitational_constant,
                c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, c->m, h, dt, c->centre,
                c->packed, c->status, c->stream);
        } else {
            nbsp_allpairs_finalize_kick(c->partial_hi, c->partial_lo, n, s.chunks,
                                        g->gravitational_constant, c->ax, c->ay, c->az, c->vx,
                                        c->vy, c->vz, h, c->stream);
        }
    }
    CUDA_TRY(cudaGetLastError());
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_advance(NBodySimProCudaContext* c,
                                              const NBodySimProGravity* gravity,
                                              NBodySimProIntegratorType integrator,
                                              double timestep, int steps,
                                              NBodySimProCudaAlgorithm algorithm,
                                              NBodySimProError* error) {
    if (c == NULL || gravity == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "view, gravity, and force function must not be null");
    if (!(timestep > 0.0)) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "timestep must be positive");
    if (steps < 0) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "steps must be non-negative");
    if (integrator != N_BODY_SIM_PRO_INTEGRATOR_EULER &&
        integrator != N_BODY_SIM_PRO_INTEGRATOR_LEAPFROG &&
        integrator != N_BODY_SIM_PRO_INTEGRATOR_VELOCITY_VERLET)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "unknown integrator type");
    if (algorithm != N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS &&
        algorithm != N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "unknown algorithm");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    NBodySimProStatus st = check_gravity(gravity, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT && c->n == 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "cannot build a Barnes-Hut tree for an empty system");
    if (c->n == 0 || steps == 0) return N_BODY_SIM_PRO_STATUS_OK;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaEventRecord(c->events[0], c->stream));
    const size_t n = c->n;
    const double dt = timestep, h = 0.5 * timestep;
    if (integrator == N_BODY_SIM_PRO_INTEGRATOR_EULER) {
        for (int step = 0; step < steps; ++step) {
            if ((st = resident_accelerations(c, gravity, algorithm, error)) != N_BODY_SIM_PRO_STATUS_OK)
                return st;
            nbsp_euler_update(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, n, dt,
                              c->stream);
        }
    } else if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS) {
        if ((st = advance_allpairs_kdk(c, gravity, dt, steps, error)) != N_BODY_SIM_PRO_STATUS_OK)
            return st;
    } else {
        /* Barnes-Hut: the kicks and the drift ride in the evaluation's bounds
         * pass and its last pass (a lone particle has no tree: plain kicks) */
        const NbspLeapfrogFusion lf = {c->vx, c->vy, c->vz, h, dt};
        for (int step = 0; step < steps; ++step) {
            if (n >= 2) {
                if ((st = resident_accelerations_fused(c, gravity, algorithm, &lf, error)) !=
                    N_BODY_SIM_PRO_STATUS_OK)
                    return st;
                continue;
            }
            nbsp_kick_drift(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, n, h, dt,
                            c->stream);
            if ((st = resident_accelerations(c, gravity, algorithm, error)) != N_BODY_SIM_PRO_STATUS_OK)
                return st;
            nbsp_kick_drift(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, n, h, 0.0,
                            c->stream);
        }
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(c->events[1], c->stream));
    if ((st = check_device_status(c, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->events[0], c->events[1]);
    if (algorithm == N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS &&
        integrator != N_BODY_SIM_PRO_INTEGRATOR_EULER) {
        float force_ms = 0.f; /* the last step's force kernel alone */
        cudaEventElapsedTime(&force_ms, c->events[2], c->events[3]);
        memset(&c->timings, 0, sizeof(c->timings));
        c->timings.walk_ms = force_ms;
        c->timings.integrate_ms = ms - force_ms * steps;
    }
    c->timings.total_ms = ms;
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* ---- all-pairs sharded by targets (one process per GPU) ------------------ */

NBodySimProStatus n_body_sim_pro_cuda_shard_begin(NBodySimProCudaContext* c, double timestep,
                                                  const double centre[3], void* slice,
                                                  size_t slice_capacity, NBodySimProError* error) {
    if (c == NULL || centre == NULL || slice == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "context, centre and slice must not be null");
    if (!(timestep >= 0.0) || !isfinite(timestep))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "timestep must be finite and >= 0");
    if (!isfinite(centre[0]) || !isfinite(centre[1]) || !isfinite(centre[2]))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "centre must be finite");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    if (slice_capacity < c->n || slice_capacity % NBSP_ALLPAIRS_CHUNK_ALIGN != 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "slice capacity must hold the resident particles and be a multiple of 8");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaEventRecord(c->events[0], c->stream));
    if (timestep > 0.0 && c->n > 0)
        nbsp_kick_drift(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->ax, c->ay, c->az, c->n,
                        0.5 * timestep, timestep, c->stream);
    CUDA_TRY(cudaMemcpyAsync(c->centre, centre, 3 * sizeof(double), cudaMemcpyHostToDevice,
                             c->stream));
    if (slice_capacity > 0)
        nbsp_pack_relative(c->x, c->y, c->z, c->m, c->n, slice_capacity, c->centre, slice,
                           c->status, c->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(c->events[1], c->stream));
    NBodySimProStatus st = check_device_status(c, error); /* synchronises */
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->events[0], c->events[1]);
    memset(&c->timings, 0, sizeof(c->timings));
    c->timings.integrate_ms = ms;
    c->timings.total_ms = ms;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_shard_end(NBodySimProCudaContext* c,
                                                const NBodySimProGravity* gravity,
                                                double timestep, const void* sources,
                                                size_t source_count, size_t slice_offset,
                                                NBodySimProError* error) {
    if (c == NULL || gravity == NULL || sources == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "context, gravity and sources must not be null");
    if (!(timestep >= 0.0) || !isfinite(timestep))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "timestep must be finite and >= 0");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    if (source_count % NBSP_ALLPAIRS_CHUNK_ALIGN != 0 || slice_offset > source_count ||
        c->n > source_count - slice_offset || source_count > (size_t)INT32_MAX)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "sources must be a multiple of 8 entries holding this rank's slice at "
                    "slice_offset");
    NBodySimProStatus st = check_gravity(gravity, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    const size_t n = c->n;
    if (n == 0) return N_BODY_SIM_PRO_STATUS_OK;
    CUDA_TRY(cudaSetDevice(c->device));
    if ((st = prepare_allpairs(c, n, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    const float eps2 = (float)gravity->softening_squared;
    const void* targets = (const char*)sources + slice_offset * 16;
    NbspAllPairsShape s = choose_shape_for(c, sources, source_count, targets, n, eps2);
    if ((size_t)s.chunks * n > c->partial_elems) s.chunks = (int)(c->partial_elems / n);
    CUDA_TRY(cudaEventRecord(c->events[2], c->stream));
    nbsp_allpairs_force_targets(sources, source_count, targets, n, eps2, s, c->partial_hi,
                                c->partial_lo, c->stream);
    CUDA_TRY(cudaEventRecord(c->events[3], c->stream));
    nbsp_allpairs_finalize_kick(c->partial_hi, c->partial_lo, n, s.chunks,
                                gravity->gravitational_constant, c->ax, c->ay, c->az, c->vx,
                                c->vy, c->vz, 0.5 * timestep, c->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(c->events[1], c->stream));
    if ((st = check_device_status(c, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    float ms = 0.f, force_ms = 0.f;
    cudaEventElapsedTime(&ms, c->events[2], c->events[1]);
    cudaEventElapsedTime(&force_ms, c->events[2], c->events[3]);
    memset(&c->timings, 0, sizeof(c->timings));
    c->timings.walk_ms = force_ms;
    c->timings.integrate_ms = ms - force_ms;
    c->timings.total_ms = ms;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_diagnostics(NBodySimProCudaContext* c,
                                                  const NBodySimProGravity* gravity,
                                                  NBodySimProDiagnosticsQuantities* q,
                                                  double* potential_energy,
                                                  NBodySimProError* error) {
    if (c == NULL || q == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "view and quantities must not be null");
    if (potential_energy != NULL && gravity == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "view, gravity, and output must not be null");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    CUDA_TRY(cudaSetDevice(c->device));
    memset(q, 0, sizeof(*q));
    if (potential_energy != NULL) *potential_energy = 0.0;
    if (c->n == 0) return N_BODY_SIM_PRO_STATUS_OK;
    NBodySimProStatus st = ensure_scratch(c, c->n > 11 * 1024 ? c->n : 11 * 1024, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    nbsp_global_sums(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->m, c->n, c->scratch, c->out,
                     c->stream);
    if (potential_energy != NULL)
        nbsp_potential_energy(c->x, c->y, c->z, c->m, c->n, gravity->gravitational_constant,
                              gravity->softening_squared, c->scratch, c->out + 11, c->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c->host_out, c->out, 12 * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const double* r = c->host_out;
    q->kinetic_energy = r[0];
    q->total_mass = r[1];
    q->total_momentum_x = r[2];
    q->total_momentum_y = r[3];
    q->total_momentum_z = r[4];
    q->total_angular_momentum_x = r[5];
    q->total_angular_momentum_y = r[6];
    q->total_angular_momentum_z = r[7];
    if (r[1] != 0.0) {
        q->center_of_mass_x = r[8] / r[1];
        q->center_of_mass_y = r[9] / r[1];
        q->center_of_mass_z = r[10] / r[1];
    }
    if (potential_energy != NULL) *potential_energy = r[11];
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_reference_acceleration(NBodySimProCudaContext* c,
                                                             const NBodySimProGravity* gravity,
                                                             const int64_t* targets, size_t count,
                                                             double* out,
                                                             NBodySimProError* error) {
    if (c == NULL || gravity == NULL || (count > 0 && (targets == NULL || out == NULL)))
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "arguments must not be null");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    for (size_t t = 0; t < count; ++t)
        if (targets[t] < 0 || (size_t)targets[t] >= c->n)
            return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "target index out of range");
    if (count == 0) return N_BODY_SIM_PRO_STATUS_OK;
    CUDA_TRY(cudaSetDevice(c->device));
    int chunks = (int)(4 * c->sm_count * 4 / ((count + 127) / 128));
    if (chunks < 1) chunks = 1;
    if ((size_t)chunks > c->n / 256 + 1) chunks = (int)(c->n / 256 + 1);
    NBodySimProStatus st = ensure_scratch(c, 3 * count * (size_t)chunks, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    int64_t* d_targets = NULL;
    double* d_out = NULL;
    CUDA_TRY(cudaMallocAsync((void**)&d_targets, count * sizeof(int64_t), c->stream));
    cudaError_t code = cudaMallocAsync((void**)&d_out, 3 * count * sizeof(double), c->stream);
    if (code == cudaSuccess)
        code = cudaMemcpyAsync(d_targets, targets, count * sizeof(int64_t), cudaMemcpyHostToDevice,
                               c->stream);
    if (code == cudaSuccess) {
        nbsp_reference_subset(c->x, c->y, c->z, c->m, c->n, d_targets, count,
                              gravity->gravitational_constant, gravity->softening_squared,
                              c->scratch, chunks, d_out, c->stream);
        code = cudaGetLastError();
    }
    if (code == cudaSuccess)
        code = cudaMemcpyAsync(out, d_out, 3 * count * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream);
    cudaFreeAsync(d_targets, c->stream);
    if (d_out != NULL) cudaFreeAsync(d_out, c->stream);
    if (code == cudaSuccess) code = cudaStreamSynchronize(c->stream);
    if (code != cudaSuccess) return cuda_fail(error, code, "reference acceleration", __FILE__, __LINE__);
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_morton_order(NBodySimProCudaContext* c, uint64_t* keys_sorted,
                                                   uint64_t* permutation, double* root,
                                                   NBodySimProError* error) {
    if (c == NULL) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context must not be null");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    if (c->n == 0)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "cannot build a Barnes-Hut tree for an empty system");
    CUDA_TRY(cudaSetDevice(c->device));
    NbspBarnesHutState s = {c->x, c->y, c->z, c->m, c->ax, c->ay, c->az, c->n,
                                {NULL, NULL, NULL, 0.0, 0.0}};
    NBodySimProStatus st =
        nbsp_bh_morton(&c->bh, &s, c->status, c->stream, keys_sorted, permutation, root, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    return check_device_status(c, error);
}

NBodySimProStatus nbsp_context_tree(NBodySimProCudaContext* c, const NBodySimProGravity* gravity,
                                    NbspTreeRef* out, NBodySimProError* error) {
    if (c == NULL || gravity == NULL || out == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context and gravity must not be null");
    if (!c->resident || c->n < 2)
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "need a resident system of >= 2 particles");
    NBodySimProStatus st = check_gravity(gravity, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    CUDA_TRY(cudaSetDevice(c->device));
    const void* saved = c->correction;
    c->correction = NULL; /* the plain tree and walk, with the features' moments */
    c->tree_quadrupoles = 1;
    st = resident_accelerations(c, gravity, N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT, error);
    c->correction = saved;
    c->tree_quadrupoles = 0;
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if ((st = check_device_status(c, error)) != N_BODY_SIM_PRO_STATUS_OK) return st;
    out->pos4 = nbsp_bh_positions(c->bh);
    out->tree = nbsp_bh_tree(c->bh);
    out->n = c->n;
    out->stream = c->stream;
    out->status = c->status;
    out->opening = c->opening;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_synchronize(NBodySimProCudaContext* c,
                                                  NBodySimProError* error) {
    if (c == NULL) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, "context must not be null");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* ---- checkpoints (checkpoint/checkpoint.h, src/c/checkpoint/checkpoint.c) ---------- */

enum { CHECKPOINT_ARRAYS = 10, CHECKPOINT_CHUNK = 8 << 20 /* bytes per staging buffer */ };

/* Two pinned staging buffers and their events; released by staging_free. */
typedef struct Staging {
    void* buffer[2];
    cudaEvent_t done[2];
} Staging;

static void staging_free(Staging* s) {
    for (int k = 0; k < 2; ++k) {
        if (s->buffer[k] != NULL) cudaFreeHost(s->buffer[k]);
        if (s->done[k] != NULL) cudaEventDestroy(s->done[k]);
        s->buffer[k] = NULL;
        s->done[k] = NULL;
    }
}

static NBodySimProStatus staging_alloc(Staging* s, NBodySimProError* error) {
    memset(s, 0, sizeof(*s));
    for (int k = 0; k < 2; ++k) {
        cudaError_t code = cudaMallocHost(&s->buffer[k], CHECKPOINT_CHUNK);
        if (code == cudaSuccess) code = cudaEventCreateWithFlags(&s->done[k], cudaEventDisableTiming);
        if (code != cudaSuccess) {
            staging_free(s);
            return cuda_fail(error, code, "checkpoint staging", __FILE__, __LINE__);
        }
    }
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* The state arrays in file order (checkpoint.c:49-53). */
static void checkpoint_arrays(NBodySimProCudaContext* c, double* out[CHECKPOINT_ARRAYS]) {
    double* const a[CHECKPOINT_ARRAYS] = {c->x, c->y, c->z, c->vx, c->vy, c->vz,
                                          c->ax, c->ay, c->az, c->m};
    memcpy(out, a, sizeof(a));
}

NBodySimProStatus n_body_sim_pro_cuda_checkpoint_write(NBodySimProCudaContext* c,
                                                       const char* path,
                                                       const NBodySimProCheckpointHeader* header,
                                                       NBodySimProError* error) {
    if (c == NULL || path == NULL || header == NULL) /* checkpoint.c:13-17 */
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "path, view, and header must not be null");
    if (!c->resident) return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "no resident state");
    if (header->particle_count != c->n) /* :18-22 */
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "checkpoint particle count does not match the view");
    CUDA_TRY(cudaSetDevice(c->device));
    Staging st;
    NBodySimProStatus s = staging_alloc(&st, error);
    if (s != N_BODY_SIM_PRO_STATUS_OK) return s;
    FILE* file = fopen(path, "wb");
    if (file == NULL) {
        staging_free(&st);
        return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to open checkpoint file for writing");
    }
    const uint32_t magic = N_BODY_SIM_PRO_CHECKPOINT_MAGIC;
    const uint32_t version = N_BODY_SIM_PRO_CHECKPOINT_VERSION;
    const NBodySimProCheckpointHeader stored = *header;
    int ok = fwrite(&magic, sizeof(magic), 1, file) == 1 &&
             fwrite(&version, sizeof(version), 1, file) == 1 &&
             fwrite(&stored, sizeof(stored), 1, file) == 1;
    double* arrays[CHECKPOINT_ARRAYS];
    checkpoint_arrays(c, arrays);
    const size_t bytes = c->n * sizeof(double);
    const size_t per_array = (bytes + CHECKPOINT_CHUNK - 1) / CHECKPOINT_CHUNK;
    const size_t chunks = per_array * CHECKPOINT_ARRAYS;
    cudaError_t code = cudaSuccess;
    /* chunk j: array j / per_array, bytes [o, o + len) of it; copy j + 1 is in
     * flight while chunk j is written */
#define CHUNK_SPAN(j, arr, off, len)                                                 \
    const size_t arr = (j) / per_array;                                             \
    const size_t off = ((j) % per_array) * (size_t)CHECKPOINT_CHUNK;                \
    const size_t len = bytes - off < (size_t)CHECKPOINT_CHUNK ? bytes - off : (size_t)CHECKPOINT_CHUNK
    if (ok && chunks > 0) {
        CHUNK_SPAN(0, a0, o0, l0);
        code = cudaMemcpyAsync(st.buffer[0], (const char*)arrays[a0] + o0, l0,
                               cudaMemcpyDeviceToHost, c->stream);
        if (code == cudaSuccess) code = cudaEventRecord(st.done[0], c->stream);
    }
    for (size_t j = 0; ok && code == cudaSuccess && j < chunks; ++j) {
        if (j + 1 < chunks) {
            CHUNK_SPAN(j + 1, an, on, ln);
            const int b = (int)((j + 1) & 1);
            code = cudaMemcpyAsync(st.buffer[b], (const char*)arrays[an] + on, ln,
                                   cudaMemcpyDeviceToHost, c->stream);
            if (code == cudaSuccess) code = cudaEventRecord(st.done[b], c->stream);
            if (code != cudaSuccess) break;
        }
        CHUNK_SPAN(j, aj, oj, lj);
        (void)aj;
        (void)oj;
        code = cudaEventSynchronize(st.done[j & 1]);
        if (code != cudaSuccess) break;
        ok = fwrite(st.buffer[j & 1], lj, 1, file) == 1;
    }
#undef CHUNK_SPAN
    cudaStreamSynchronize(c->stream);
    staging_free(&st);
    const int closed = fclose(file) == 0;
    if (code != cudaSuccess) return cuda_fail(error, code, "checkpoint copy", __FILE__, __LINE__);
    if (!ok) return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to write checkpoint array");
    if (!closed) return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to close checkpoint file");
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_checkpoint_read(NBodySimProCudaContext* c, const char* path,
                                                      NBodySimProCheckpointHeader* header,
                                                      NBodySimProError* error) {
    if (c == NULL || path == NULL || header == NULL) /* checkpoint.c:134-138 */
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
                    "path, header, and particle system must not be null");
    CUDA_TRY(cudaSetDevice(c->device));
    FILE* file = fopen(path, "rb");
    if (file == NULL)
        return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to open checkpoint file for reading");
    uint32_t magic = 0, version = 0;
    if (fread(&magic, sizeof(magic), 1, file) != 1 || fread(&version, sizeof(version), 1, file) != 1) {
        fclose(file);
        return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to read checkpoint magic");
    }
    if (magic != N_BODY_SIM_PRO_CHECKPOINT_MAGIC) { /* :88-92 */
        fclose(file);
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "not an N-Body Sim Pro checkpoint file");
    }
    if (version != N_BODY_SIM_PRO_CHECKPOINT_VERSION) {
        fclose(file);
        return FAIL(N_BODY_SIM_PRO_STATUS_INVALID_STATE, "unsupported checkpoint version");
    }
    NBodySimProCheckpointHeader stored;
    if (fread(&stored, sizeof(stored), 1, file) != 1) {
        fclose(file);
        return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to read checkpoint metadata");
    }
    NBodySimProStatus s = ensure_capacity(c, stored.particle_count, error);
    if (s != N_BODY_SIM_PRO_STATUS_OK) {
        fclose(file);
        return s;
    }
    Staging st;
    if ((s = staging_alloc(&st, error)) != N_BODY_SIM_PRO_STATUS_OK) {
        fclose(file);
        return s;
    }
    double* arrays[CHECKPOINT_ARRAYS];
    checkpoint_arrays(c, arrays);
    const size_t bytes = stored.particle_count * sizeof(double);
    const size_t per_array = (bytes + CHECKPOINT_CHUNK - 1) / CHECKPOINT_CHUNK;
    const size_t chunks = per_array * CHECKPOINT_ARRAYS;
    cudaError_t code = cudaSuccess;
    int ok = 1;
    for (size_t j = 0; j < chunks; ++j) {
        const size_t arr = j / per_array;
        const size_t off = (j % per_array) * (size_t)CHECKPOINT_CHUNK;
        const size_t len = bytes - off < (size_t)CHECKPOINT_CHUNK ? bytes - off : (size_t)CHECKPOINT_CHUNK;
        const int b = (int)(j & 1);
        if (j >= 2 && (code = cudaEventSynchronize(st.done[b])) != cudaSuccess) break;
        if (fread(st.buffer[b], len, 1, file) != 1) { /* the copy of chunk j - 1 runs meanwhile */
            ok = 0;
            break;
        }
        code = cudaMemcpyAsync((char*)arrays[arr] + off, st.buffer[b], len, cudaMemcpyHostToDevice,
                               c->stream);
        if (code == cudaSuccess) code = cudaEventRecord(st.done[b], c->stream);
        if (code != cudaSuccess) break;
    }
    cudaStreamSynchronize(c->stream);
    staging_free(&st);
    const int closed = fclose(file) == 0;
    if (code != cudaSuccess) return cuda_fail(error, code, "checkpoint copy", __FILE__, __LINE__);
    if (!ok) return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to read checkpoint array");
    if (!closed) return FAIL(N_BODY_SIM_PRO_STATUS_IO_ERROR, "failed to close checkpoint file");
    c->n = stored.particle_count;
    c->n_padded = round_up(c->n, 256);
    c->resident = 1;
    *header = stored;
    return N_BODY_SIM_PRO_STATUS_OK;
}
