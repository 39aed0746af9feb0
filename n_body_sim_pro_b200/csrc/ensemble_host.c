/*
 * Batched ensembles of independent small systems (C17 host side).
 *
 * Upload: systems are concatenated SoA ranges [offsets[k], offsets[k+1]).
 * Advance, persistent mode: one CUDA-graph launch of ensemble.cu's persistent
 * kernel runs `steps` leapfrog steps of every system; the tile shape (threads
 * per CTA x targets per thread) is chosen by a measuring autotuner on the
 * uploaded ensemble, and the work items are ordered longest-first.
 * Advance, per-system mode (the baseline): the single-system all-pairs path,
 * launched system by system and step by step.
 */
#include "n_body_sim_pro_cuda.h"

#include "internal.h"

#include <cuda_runtime_api.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ensemble.cu launchers */
NBSP_HIDDEN int nbsp_ensemble_shape_supported(int block, int per_thread);
NBSP_HIDDEN int nbsp_ensemble_resident_ctas(int block, int per_thread);
NBSP_HIDDEN void nbsp_ensemble_advance(int block, int per_thread, int grid, double* x, double* y,
                                       double* z, double* vx, double* vy, double* vz, double* ax,
                                       double* ay, double* az, const double* m,
                                       const long long* offset, const double* centre,
                                       const int* item_start, const int* item_systems,
                                       const int* item_group, int items, int* counter,
                                       int* status, double g, float eps2, double dt, int steps,
                                       int guard, cudaStream_t stream);

enum { ENS_MAX_SYSTEM = 4096, ENS_SHAPES = 3, ENS_TILE = 64 /* = kTile in ensemble.cu */ };

static const int kEnsShapes[ENS_SHAPES][2] = {{512, 8}, {1024, 4}, {256, 16}};

typedef struct Items {
    int* start;    /* host [items + 1] */
    int* systems;  /* host [systems] */
    int* group;    /* host [items] */
    int count;
} Items;

struct NBodySimProCudaEnsemble {
    int device, sm_count;
    cudaStream_t stream;
    cudaEvent_t ev[2];
    size_t systems, particles;
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m, *centre;
    double max_mass; /* largest |m|: decides whether the self pair needs a guard */
    long long* offset;      /* device */
    long long* host_offset; /* host */
    int *d_item_start, *d_item_systems, *d_item_group;
    int items;
    int *counter, *status, *host_status;
    int block, per_thread, grid, tuned;
    /* per-system baseline scratch */
    void *packed, *hi, *lo;
    /* captured graph of the persistent launch */
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    int graph_steps;
    double graph_dt, graph_g, graph_eps2;
    double last_ms;
    float tune_ms[ENS_SHAPES];
};

static NBodySimProStatus efail(NBodySimProError* error, NBodySimProStatus status, int line,
                               const char* message) {
    if (error != NULL) {
        error->status = status;
        error->source_file = __FILE__;
        error->source_line = line;
        snprintf(error->message, sizeof(error->message), "%s", message);
    }
    return status;
}

static NBodySimProStatus ecuda(NBodySimProError* error, cudaError_t code, int line,
                               const char* what) {
    char text[256];
    snprintf(text, sizeof(text), "%s: %s", what, cudaGetErrorString(code));
    NBodySimProStatus st = code == cudaErrorMemoryAllocation ? N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY
                                                             : N_BODY_SIM_PRO_STATUS_INVALID_STATE;
    if (code == cudaErrorNoDevice || code == cudaErrorInsufficientDriver)
        st = N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM;
    return efail(error, st, line, text);
}

#define ETRY(call)                                                          \
    do {                                                                    \
        cudaError_t etry_code = (call);                                     \
        if (etry_code != cudaSuccess) return ecuda(error, etry_code, __LINE__, #call); \
    } while (0)

static void release_graph(NBodySimProCudaEnsemble* e) {
    if (e->exec != NULL) cudaGraphExecDestroy(e->exec);
    if (e->graph != NULL) cudaGraphDestroy(e->graph);
    e->exec = NULL;
    e->graph = NULL;
}

static void release_data(NBodySimProCudaEnsemble* e) {
    void* p[] = {e->x, e->y, e->z, e->vx, e->vy, e->vz, e->ax, e->ay, e->az, e->m, e->centre,
                 e->offset, e->d_item_start, e->d_item_systems, e->d_item_group, e->packed,
                 e->hi, e->lo};
    for (size_t k = 0; k < sizeof(p) / sizeof(p[0]); ++k) cudaFree(p[k]);
    e->x = e->y = e->z = e->vx = e->vy = e->vz = e->ax = e->ay = e->az = e->m = e->centre = NULL;
    e->offset = NULL;
    e->d_item_start = e->d_item_systems = e->d_item_group = NULL;
    e->packed = e->hi = e->lo = NULL;
    free(e->host_offset);
    e->host_offset = NULL;
    e->systems = e->particles = 0;
    e->items = 0;
    e->tuned = 0;
    release_graph(e);
}

NBodySimProCudaEnsemble* n_body_sim_pro_cuda_ensemble_create(NBodySimProError* error) {
    int count = 0;
    cudaError_t code = cudaGetDeviceCount(&count);
    if (code != cudaSuccess || count == 0) {
        efail(error, N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM, __LINE__,
              code != cudaSuccess ? cudaGetErrorString(code) : "no CUDA device");
        return NULL;
    }
    NBodySimProCudaEnsemble* e = (NBodySimProCudaEnsemble*)calloc(1, sizeof(*e));
    if (e == NULL) {
        efail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "ensemble allocation");
        return NULL;
    }
    struct cudaDeviceProp prop;
    code = cudaGetDevice(&e->device);
    if (code == cudaSuccess) code = cudaGetDeviceProperties(&prop, e->device);
    if (code == cudaSuccess && prop.major < 10) {
        free(e);
        efail(error, N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM, __LINE__,
              "this library is built for sm_100a (B200)");
        return NULL;
    }
    if (code == cudaSuccess) {
        e->sm_count = prop.multiProcessorCount;
        code = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    }
    if (code == cudaSuccess) code = cudaEventCreate(&e->ev[0]);
    if (code == cudaSuccess) code = cudaEventCreate(&e->ev[1]);
    if (code == cudaSuccess) code = cudaMalloc((void**)&e->counter, sizeof(int));
    if (code == cudaSuccess) code = cudaMalloc((void**)&e->status, sizeof(int));
    if (code == cudaSuccess) code = cudaMallocHost((void**)&e->host_status, sizeof(int));
    if (code == cudaSuccess) code = cudaMemset(e->status, 0, sizeof(int));
    if (code != cudaSuccess) {
        ecuda(error, code, __LINE__, "ensemble set-up");
        n_body_sim_pro_cuda_ensemble_destroy(e);
        return NULL;
    }
    e->block = kEnsShapes[0][0];
    e->per_thread = kEnsShapes[0][1];
    return e;
}

void n_body_sim_pro_cuda_ensemble_destroy(NBodySimProCudaEnsemble* e) {
    if (e == NULL) return;
    cudaSetDevice(e->device);
    if (e->stream != NULL) cudaStreamSynchronize(e->stream);
    release_data(e);
    cudaFree(e->counter);
    cudaFree(e->status);
    cudaFreeHost(e->host_status);
    if (e->ev[0] != NULL) cudaEventDestroy(e->ev[0]);
    if (e->ev[1] != NULL) cudaEventDestroy(e->ev[1]);
    if (e->stream != NULL) cudaStreamDestroy(e->stream);
    free(e);
}

static unsigned next_pow2(unsigned v) {
    unsigned p = 32;
    while (p < v) p <<= 1;
    return p;
}

typedef struct SortKey {
    long long cost;
    int index;
} SortKey;

static int by_cost_desc(const void* a, const void* b) {
    const SortKey* x = (const SortKey*)a;
    const SortKey* y = (const SortKey*)b;
    if (x->cost != y->cost) return x->cost > y->cost ? -1 : 1;
    return x->index - y->index;
}

/* Threads of the subgroup that owns a system of n particles: the kernel pads
 * each system to whole tiles of ENS_TILE sources (ensemble.cu kTile), and the
 * subgroup's G * k shared-memory slots must hold the padded system.  G is the
 * smallest whole number of warps that does (a power of two below one warp, so
 * subgroups never straddle a warp boundary): every thread slot beyond the
 * system's particles still runs the force loop, so a power-of-two G would
 * waste up to half of the work of the largest systems. */
static int group_threads(long long n, int k) {
    const long long padded = (n + ENS_TILE - 1) / ENS_TILE * ENS_TILE;
    const long long need = (padded + k - 1) / k;
    if (need < 32) return (int)next_pow2((unsigned)need);
    return (int)((need + 31) / 32 * 32);
}

/* Bundle systems into work items for threads-per-CTA `block` and `k` targets
 * per thread; items ordered by cost (sum n^2), largest first. */
static int build_items(const long long* off, size_t systems, int block, int k, Items* out) {
    SortKey* order = (SortKey*)malloc(systems * sizeof(SortKey));
    int* start = (int*)malloc((systems + 1) * sizeof(int));
    int* list = (int*)malloc(systems * sizeof(int));
    int* group = (int*)malloc(systems * sizeof(int));
    long long* cost = (long long*)malloc(systems * sizeof(long long));
    int* tmp_start = (int*)malloc((systems + 1) * sizeof(int));
    int* tmp_group = (int*)malloc(systems * sizeof(int));
    if (!order || !start || !list || !group || !cost || !tmp_start || !tmp_group) {
        free(order); free(start); free(list); free(group); free(cost); free(tmp_start); free(tmp_group);
        return 1;
    }
    for (size_t s = 0; s < systems; ++s) {
        order[s].cost = off[s + 1] - off[s];
        order[s].index = (int)s;
    }
    qsort(order, systems, sizeof(SortKey), by_cost_desc); /* largest systems first */
    /* greedy bundling: consecutive systems of one size class share an item */
    int items = 0;
    size_t s = 0;
    int* cursor = list;
    while (s < systems) {
        const long long n = order[s].cost;
        const int g = group_threads(n, k);
        const int per_item = block / g;
        tmp_start[items] = (int)(cursor - list);
        tmp_group[items] = g;
        long long c = 0;
        int taken = 0;
        while (s < systems && taken < per_item) {
            const long long m = order[s].cost;
            if (group_threads(m, k) != g) break;
            *cursor++ = order[s].index;
            c += m * m;
            ++taken;
            ++s;
        }
        cost[items] = c;
        ++items;
    }
    tmp_start[items] = (int)(cursor - list);
    /* order items by cost (longest processing time first) */
    SortKey* io = (SortKey*)malloc((size_t)items * sizeof(SortKey));
    int* list2 = (int*)malloc(systems * sizeof(int));
    if (!io || !list2) {
        free(io); free(list2); free(order); free(start); free(list); free(group); free(cost);
        free(tmp_start); free(tmp_group);
        return 1;
    }
    for (int i = 0; i < items; ++i) {
        io[i].cost = cost[i];
        io[i].index = i;
    }
    qsort(io, (size_t)items, sizeof(SortKey), by_cost_desc);
    int pos = 0;
    for (int i = 0; i < items; ++i) {
        const int src = io[i].index;
        start[i] = pos;
        group[i] = tmp_group[src];
        for (int q = tmp_start[src]; q < tmp_start[src + 1]; ++q) list2[pos++] = list[q];
    }
    start[items] = pos;
    free(io); free(order); free(list); free(cost); free(tmp_start); free(tmp_group);
    out->start = start;
    out->systems = list2;
    out->group = group;
    out->count = items;
    return 0;
}

static void free_items(Items* it) {
    free(it->start);
    free(it->systems);
    free(it->group);
    memset(it, 0, sizeof(*it));
}

static NBodySimProStatus load_items(NBodySimProCudaEnsemble* e, int block, int k,
                                    NBodySimProError* error) {
    Items it;
    if (build_items(e->host_offset, e->systems, block, k, &it))
        return efail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "work items");
    cudaFree(e->d_item_start);
    cudaFree(e->d_item_systems);
    cudaFree(e->d_item_group);
    e->d_item_start = e->d_item_systems = e->d_item_group = NULL;
    cudaError_t code = cudaMalloc((void**)&e->d_item_start, (size_t)(it.count + 1) * sizeof(int));
    if (code == cudaSuccess) code = cudaMalloc((void**)&e->d_item_systems, e->systems * sizeof(int));
    if (code == cudaSuccess) code = cudaMalloc((void**)&e->d_item_group, (size_t)it.count * sizeof(int));
    if (code == cudaSuccess)
        code = cudaMemcpy(e->d_item_start, it.start, (size_t)(it.count + 1) * sizeof(int),
                          cudaMemcpyHostToDevice);
    if (code == cudaSuccess)
        code = cudaMemcpy(e->d_item_systems, it.systems, e->systems * sizeof(int),
                          cudaMemcpyHostToDevice);
    if (code == cudaSuccess)
        code = cudaMemcpy(e->d_item_group, it.group, (size_t)it.count * sizeof(int),
                          cudaMemcpyHostToDevice);
    e->items = it.count;
    free_items(&it);
    if (code != cudaSuccess) return ecuda(error, code, __LINE__, "work item upload");
    const int resident = nbsp_ensemble_resident_ctas(block, k);
    e->block = block;
    e->per_thread = k;
    e->grid = e->sm_count * (resident > 0 ? resident : 1);
    if (e->grid > e->items) e->grid = e->items;
    if (e->grid < 1) e->grid = 1;
    release_graph(e);
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_ensemble_upload(NBodySimProCudaEnsemble* e,
                                                      const NBodySimProParticleSystemView* view,
                                                      const uint64_t* offsets, size_t systems,
                                                      NBodySimProError* error) {
    if (e == NULL || view == NULL || offsets == NULL || systems == 0)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "ensemble, view and offsets must not be null; at least one system");
    if (offsets[0] != 0 || offsets[systems] != view->particle_count)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "offsets must start at 0 and end at the view's particle count");
    for (size_t s = 0; s < systems; ++s) {
        const uint64_t n = offsets[s + 1] - offsets[s];
        if (offsets[s + 1] < offsets[s] || n == 0 || n > ENS_MAX_SYSTEM)
            return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                         "every system must hold 1..4096 particles");
    }
    const double* src[] = {view->positions_x, view->positions_y, view->positions_z,
                           view->velocities_x, view->velocities_y, view->velocities_z,
                           view->masses};
    for (int k = 0; k < 7; ++k)
        if (src[k] == NULL)
            return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                         "view positions, velocities and masses must not be null");
    ETRY(cudaSetDevice(e->device));
    ETRY(cudaStreamSynchronize(e->stream));
    release_data(e);
    const size_t n = view->particle_count;
    double** dst[] = {&e->x, &e->y, &e->z, &e->vx, &e->vy, &e->vz, &e->m, &e->ax, &e->ay, &e->az};
    for (int k = 0; k < 10; ++k) ETRY(cudaMalloc((void**)dst[k], n * sizeof(double)));
    for (int k = 0; k < 7; ++k)
        ETRY(cudaMemcpy(*dst[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice));
    ETRY(cudaMemset(e->ax, 0, n * sizeof(double)));
    ETRY(cudaMemset(e->ay, 0, n * sizeof(double)));
    ETRY(cudaMemset(e->az, 0, n * sizeof(double)));
    e->host_offset = (long long*)malloc((systems + 1) * sizeof(long long));
    double* centre = (double*)malloc(3 * systems * sizeof(double));
    if (e->host_offset == NULL || centre == NULL) {
        free(centre);
        return efail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "ensemble tables");
    }
    for (size_t s = 0; s <= systems; ++s) e->host_offset[s] = (long long)offsets[s];
    e->max_mass = 0.0;
    for (size_t i = 0; i < n; ++i) e->max_mass = fmax(e->max_mass, fabs(view->masses[i]));
    /* FP64 centre of mass of every system: the origin of its FP32 coordinates */
    for (size_t s = 0; s < systems; ++s) {
        double mt = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
        for (uint64_t i = offsets[s]; i < offsets[s + 1]; ++i) {
            const double mi = view->masses[i];
            mt += mi;
            cx += mi * view->positions_x[i];
            cy += mi * view->positions_y[i];
            cz += mi * view->positions_z[i];
        }
        centre[3 * s] = mt != 0.0 ? cx / mt : 0.0;
        centre[3 * s + 1] = mt != 0.0 ? cy / mt : 0.0;
        centre[3 * s + 2] = mt != 0.0 ? cz / mt : 0.0;
    }
    cudaError_t code = cudaMalloc((void**)&e->centre, 3 * systems * sizeof(double));
    if (code == cudaSuccess)
        code = cudaMemcpy(e->centre, centre, 3 * systems * sizeof(double), cudaMemcpyHostToDevice);
    free(centre);
    if (code != cudaSuccess) return ecuda(error, code, __LINE__, "centres");
    ETRY(cudaMalloc((void**)&e->offset, (systems + 1) * sizeof(long long)));
    ETRY(cudaMemcpy(e->offset, e->host_offset, (systems + 1) * sizeof(long long),
                    cudaMemcpyHostToDevice));
    /* per-system baseline scratch: the largest system */
    ETRY(cudaMalloc(&e->packed, ENS_MAX_SYSTEM * 16));
    ETRY(cudaMalloc(&e->hi, ENS_MAX_SYSTEM * 16));
    ETRY(cudaMalloc(&e->lo, ENS_MAX_SYSTEM * 16));
    e->systems = systems;
    e->particles = n;
    return load_items(e, kEnsShapes[0][0], kEnsShapes[0][1], error);
}

NBodySimProStatus n_body_sim_pro_cuda_ensemble_download(NBodySimProCudaEnsemble* e,
                                                        const NBodySimProParticleSystemView* view,
                                                        NBodySimProError* error) {
    if (e == NULL || view == NULL)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "null argument");
    if (view->particle_count != e->particles)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "view particle count differs from the uploaded ensemble");
    ETRY(cudaSetDevice(e->device));
    ETRY(cudaStreamSynchronize(e->stream));
    double* dst[] = {view->positions_x, view->positions_y, view->positions_z, view->velocities_x,
                     view->velocities_y, view->velocities_z, view->accelerations_x,
                     view->accelerations_y, view->accelerations_z, view->masses};
    const double* src[] = {e->x, e->y, e->z, e->vx, e->vy, e->vz, e->ax, e->ay, e->az, e->m};
    for (int k = 0; k < 10; ++k)
        if (dst[k] != NULL && e->particles > 0)
            ETRY(cudaMemcpy(dst[k], src[k], e->particles * sizeof(double), cudaMemcpyDeviceToHost));
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* The unguarded kernel relies on the self pair adding W * 0 = 0: eps^2 a
 * normal float and m / eps^3 far from overflow. */
static int self_pair_needs_guard(const NBodySimProCudaEnsemble* e, float eps2) {
    if (!(eps2 >= FLT_MIN)) return 1;
    const double inv_eps3 = 1.0 / ((double)eps2 * sqrt((double)eps2));
    return !(e->max_mass * inv_eps3 < 1e30);
}

static void enqueue_persistent(NBodySimProCudaEnsemble* e, double g, float eps2, double dt,
                               int steps) {
    cudaMemsetAsync(e->counter, 0, sizeof(int), e->stream);
    nbsp_ensemble_advance(e->block, e->per_thread, e->grid, e->x, e->y, e->z, e->vx, e->vy, e->vz,
                          e->ax, e->ay, e->az, e->m, e->offset, e->centre, e->d_item_start,
                          e->d_item_systems, e->d_item_group, e->items, e->counter, e->status, g,
                          eps2, dt, steps, self_pair_needs_guard(e, eps2), e->stream);
}

/* One launch per system per phase (the baseline the persistent launch replaces). */
static void enqueue_per_system(NBodySimProCudaEnsemble* e, double g, float eps2, double dt,
                               int steps) {
    const NbspAllPairsShape shape = {128, 4, 1, 0, 0};
    const double h = 0.5 * dt;
    for (int step = 0; step < steps; ++step) {
        for (size_t s = 0; s < e->systems; ++s) {
            const long long o = e->host_offset[s];
            const size_t n = (size_t)(e->host_offset[s + 1] - o);
            const size_t np = (n + 255) / 256 * 256;
            const double* c = e->centre + 3 * s;
            if (step == 0) {
                nbsp_pack_relative(e->x + o, e->y + o, e->z + o, e->m + o, n, np, c, e->packed,
                                   e->status, e->stream);
                nbsp_allpairs_force(e->packed, n, np, eps2, shape, e->hi, e->lo, e->stream);
                nbsp_allpairs_finalize(e->hi, e->lo, n, 1, g, e->ax + o, e->ay + o, e->az + o,
                                       e->stream);
            }
            nbsp_kick_drift(e->x + o, e->y + o, e->z + o, e->vx + o, e->vy + o, e->vz + o,
                            e->ax + o, e->ay + o, e->az + o, n, h, dt, e->stream);
            nbsp_pack_relative(e->x + o, e->y + o, e->z + o, e->m + o, n, np, c, e->packed,
                               e->status, e->stream);
            nbsp_allpairs_force(e->packed, n, np, eps2, shape, e->hi, e->lo, e->stream);
            nbsp_allpairs_finalize_kick(e->hi, e->lo, n, 1, g, e->ax + o, e->ay + o, e->az + o,
                                        e->vx + o, e->vy + o, e->vz + o, h, e->stream);
        }
    }
}

static NBodySimProStatus finish(NBodySimProCudaEnsemble* e, NBodySimProError* error) {
    ETRY(cudaEventRecord(e->ev[1], e->stream));
    ETRY(cudaMemcpyAsync(e->host_status, e->status, sizeof(int), cudaMemcpyDeviceToHost,
                         e->stream));
    ETRY(cudaMemsetAsync(e->status, 0, sizeof(int), e->stream));
    ETRY(cudaStreamSynchronize(e->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    e->last_ms = ms;
    if (*e->host_status & NBSP_DEVICE_ERROR_NONFINITE_POSITION)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "non-finite particle position");
    if (*e->host_status != 0)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__,
                     "ensemble kernel exceeded its limits");
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_ensemble_autotune(NBodySimProCudaEnsemble* e,
                                                        const NBodySimProGravity* gravity,
                                                        double timestep,
                                                        NBodySimProError* error) {
    if (e == NULL || gravity == NULL || e->systems == 0)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "ensemble and gravity must not be null; upload first");
    ETRY(cudaSetDevice(e->device));
    /* measure on a copy of the state so tuning does not advance the ensemble */
    const size_t bytes = e->particles * sizeof(double);
    double* save[9] = {0};
    double* live[9] = {e->x, e->y, e->z, e->vx, e->vy, e->vz, e->ax, e->ay, e->az};
    for (int k = 0; k < 9; ++k) {
        ETRY(cudaMalloc((void**)&save[k], bytes));
        ETRY(cudaMemcpyAsync(save[k], live[k], bytes, cudaMemcpyDeviceToDevice, e->stream));
    }
    int best = -1;
    float best_ms = 0.f;
    NBodySimProStatus st = N_BODY_SIM_PRO_STATUS_OK;
    for (int s = 0; s < ENS_SHAPES && st == N_BODY_SIM_PRO_STATUS_OK; ++s) {
        if (!nbsp_ensemble_shape_supported(kEnsShapes[s][0], kEnsShapes[s][1])) continue;
        st = load_items(e, kEnsShapes[s][0], kEnsShapes[s][1], error);
        if (st != N_BODY_SIM_PRO_STATUS_OK) break;
        cudaEventRecord(e->ev[0], e->stream);
        enqueue_persistent(e, gravity->gravitational_constant, (float)gravity->softening_squared,
                           timestep, 2);
        st = finish(e, error);
        e->tune_ms[s] = (float)e->last_ms;
        if (st == N_BODY_SIM_PRO_STATUS_OK && (best < 0 || e->last_ms < best_ms)) {
            best = s;
            best_ms = (float)e->last_ms;
        }
        for (int k = 0; k < 9; ++k)
            cudaMemcpyAsync(live[k], save[k], bytes, cudaMemcpyDeviceToDevice, e->stream);
    }
    cudaStreamSynchronize(e->stream);
    for (int k = 0; k < 9; ++k) cudaFree(save[k]);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    if (best < 0) return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__, "no tile shape");
    st = load_items(e, kEnsShapes[best][0], kEnsShapes[best][1], error);
    e->tuned = 1;
    return st;
}

NBodySimProStatus n_body_sim_pro_cuda_ensemble_advance(NBodySimProCudaEnsemble* e,
                                                       const NBodySimProGravity* gravity,
                                                       double timestep, int steps,
                                                       int one_launch_per_system,
                                                       NBodySimProError* error) {
    if (e == NULL || gravity == NULL)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "ensemble and gravity must not be null");
    if (!(timestep > 0.0))
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "timestep must be positive");
    if (steps < 0 || !isfinite(gravity->softening_squared) || gravity->softening_squared < 0.0)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "invalid steps or gravity");
    if (e->systems == 0)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__, "no ensemble uploaded");
    if (steps == 0) return N_BODY_SIM_PRO_STATUS_OK;
    ETRY(cudaSetDevice(e->device));
    const double g = gravity->gravitational_constant;
    const float eps2 = (float)gravity->softening_squared;
    if (one_launch_per_system) {
        ETRY(cudaEventRecord(e->ev[0], e->stream));
        enqueue_per_system(e, g, eps2, timestep, steps);
        ETRY(cudaGetLastError());
        return finish(e, error);
    }
    if (!e->tuned) {
        NBodySimProStatus st = n_body_sim_pro_cuda_ensemble_autotune(e, gravity, timestep, error);
        if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    }
    if (e->exec == NULL || e->graph_steps != steps || e->graph_dt != timestep || e->graph_g != g ||
        e->graph_eps2 != (double)eps2) {
        release_graph(e);
        ETRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
        enqueue_persistent(e, g, eps2, timestep, steps);
        cudaGraph_t graph = NULL;
        cudaError_t code = cudaStreamEndCapture(e->stream, &graph);
        if (code != cudaSuccess) return ecuda(error, code, __LINE__, "graph capture");
        e->graph = graph;
        ETRY(cudaGraphInstantiate(&e->exec, e->graph, 0));
        e->graph_steps = steps;
        e->graph_dt = timestep;
        e->graph_g = g;
        e->graph_eps2 = (double)eps2;
    }
    ETRY(cudaEventRecord(e->ev[0], e->stream));
    ETRY(cudaGraphLaunch(e->exec, e->stream));
    return finish(e, error);
}

NBodySimProStatus n_body_sim_pro_cuda_ensemble_info(const NBodySimProCudaEnsemble* e,
                                                    NBodySimProCudaEnsembleInfo* info,
                                                    NBodySimProError* error) {
    if (e == NULL || info == NULL)
        return efail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "null argument");
    memset(info, 0, sizeof(*info));
    info->systems = e->systems;
    info->particles = e->particles;
    info->threads_per_block = e->block;
    info->targets_per_thread = e->per_thread;
    info->grid = e->grid;
    info->work_items = e->items;
    info->last_advance_ms = e->last_ms;
    for (int s = 0; s < ENS_SHAPES; ++s) info->autotune_ms[s] = e->tune_ms[s];
    return N_BODY_SIM_PRO_STATUS_OK;
}
