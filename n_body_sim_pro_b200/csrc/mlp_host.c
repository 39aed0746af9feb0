/*
 * Learned far-field correction (C17 host side): training-pair generation from a
 * resident system's tree, minibatch Adam training on the GPU, parameter
 * exchange, and the single-batch gradient used to check the tensor-core
 * backward pass against an FP64 CPU computation.
 *
 * No counterpart in the reference engine (its Barnes-Hut is monopole-only,
 * src/c/barnes_hut/barnes_hut.c:600-612); the correction targets exactly that
 * monopole's residual against the exact cell sum.
 */
#include "n_body_sim_pro_cuda.h"

#include "bh.h"
#include "internal.h"

#include <cuda_runtime_api.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* mlp.cu launchers */
NBSP_HIDDEN size_t nbsp_mlp_net_bytes(void);
NBSP_HIDDEN size_t nbsp_mlp_frags_bytes(void);
NBSP_HIDDEN int nbsp_mlp_param_count(void);
NBSP_HIDDEN int nbsp_mlp_rows_per_cta(void);
NBSP_HIDDEN void nbsp_mlp_build_frags(const float* params, void* frags, void* net,
                                      cudaStream_t stream);
NBSP_HIDDEN void nbsp_mlp_standardise(const float* feat, const float* lab, int rows,
                                      const void* net, uint32_t* x, float* y, cudaStream_t stream);
NBSP_HIDDEN void nbsp_mlp_train_step(const uint32_t* x, const float* y, const int* order,
                                     int first_row, int rows_total, int ctas, float inv_batch3,
                                     const void* frags, float* partial, float* loss,
                                     cudaStream_t stream);
NBSP_HIDDEN void nbsp_mlp_reduce_adam(const float* partial, int slots, float* grad_out,
                                      float* params, float* m, float* v, float lr, int step,
                                      int apply, cudaStream_t stream);
NBSP_HIDDEN void nbsp_mlp_evaluate(const void* net, const float* feat, int rows, float* out,
                                   int tcgen05, int* status, cudaStream_t stream);
NBSP_HIDDEN void nbsp_mlp_set_scaling(void* net, const float* table, cudaStream_t stream);
NBSP_HIDDEN void nbsp_mlp_get_scaling(const void* net, float* table, cudaStream_t stream);

enum { IN = 10, OUT = 3, SCALING = 46 };

struct NBodySimProCudaCorrection {
    int device;
    cudaStream_t stream;
    float *params, *m, *v;  /* device FP32 master weights and Adam moments */
    void* frags;            /* training fragments */
    void* net;              /* inference network (read by the corrected walk) */
    float* partial;         /* per-CTA gradient slots */
    float* loss;            /* per-CTA loss sums */
    float* grad;            /* reduced gradient */
    int slots;
    uint32_t* x;            /* standardised BF16 features, 8 words per row */
    float* y;               /* standardised labels */
    float* feat;            /* raw features of the kept rows */
    float* lab;             /* raw labels of the kept rows */
    int* order;
    size_t rows, train_rows;
    int adam_step;
    uint64_t seed;
    float* host_loss;       /* pinned */
};

static NBodySimProStatus mfail(NBodySimProError* error, NBodySimProStatus status, int line,
                               const char* message) {
    if (error != NULL) {
        error->status = status;
        error->source_file = __FILE__;
        error->source_line = line;
        snprintf(error->message, sizeof(error->message), "%s", message);
    }
    return status;
}

static NBodySimProStatus mcuda(NBodySimProError* error, cudaError_t code, int line,
                               const char* what) {
    char text[256];
    snprintf(text, sizeof(text), "%s: %s", what, cudaGetErrorString(code));
    return mfail(error,
                 code == cudaErrorMemoryAllocation ? N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY
                                                   : N_BODY_SIM_PRO_STATUS_INVALID_STATE,
                 line, text);
}

#define MTRY(call)                                                                   \
    do {                                                                             \
        cudaError_t mtry_code = (call);                                              \
        if (mtry_code != cudaSuccess) return mcuda(error, mtry_code, __LINE__, #call); \
    } while (0)

static uint64_t splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double uniform(uint64_t* s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

static void free_data(NBodySimProCudaCorrection* c) {
    cudaFree(c->x);
    cudaFree(c->y);
    cudaFree(c->feat);
    cudaFree(c->lab);
    cudaFree(c->order);
    c->x = NULL;
    c->y = NULL;
    c->feat = c->lab = NULL;
    c->order = NULL;
    c->rows = c->train_rows = 0;
}

void n_body_sim_pro_cuda_correction_destroy(NBodySimProCudaCorrection* c) {
    if (c == NULL) return;
    cudaSetDevice(c->device);
    if (c->stream != NULL) cudaStreamSynchronize(c->stream);
    free_data(c);
    void* p[] = {c->params, c->m, c->v, c->frags, c->net, c->partial, c->loss, c->grad};
    for (size_t k = 0; k < sizeof(p) / sizeof(p[0]); ++k) cudaFree(p[k]);
    cudaFreeHost(c->host_loss);
    if (c->stream != NULL) cudaStreamDestroy(c->stream);
    free(c);
}

/* Glorot-uniform weights, zero biases, identity scaling. */
static NBodySimProStatus init_parameters(NBodySimProCudaCorrection* c, NBodySimProError* error) {
    const int np = nbsp_mlp_param_count();
    float* h = (float*)calloc((size_t)np, sizeof(float));
    if (h == NULL) return mfail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "parameters");
    uint64_t s = c->seed;
    const int layers[3][3] = {{0, 64, IN}, {64 * IN + 64, 64, 64}, {64 * IN + 64 + 64 * 64 + 64, OUT, 64}};
    for (int l = 0; l < 3; ++l) {
        const int off = layers[l][0], outs = layers[l][1], ins = layers[l][2];
        const double lim = sqrt(6.0 / (double)(ins + outs));
        for (int k = 0; k < outs * ins; ++k) h[off + k] = (float)((2.0 * uniform(&s) - 1.0) * lim);
    }
    cudaError_t code = cudaMemcpy(c->params, h, (size_t)np * sizeof(float), cudaMemcpyHostToDevice);
    free(h);
    if (code != cudaSuccess) return mcuda(error, code, __LINE__, "parameter upload");
    MTRY(cudaMemset(c->m, 0, (size_t)np * sizeof(float)));
    MTRY(cudaMemset(c->v, 0, (size_t)np * sizeof(float)));
    float table[SCALING];
    for (int i = 0; i < IN; ++i) {
        table[i] = 0.f;
        table[IN + i] = 1.f;
        table[2 * IN + i] = -INFINITY;
        table[3 * IN + i] = INFINITY;
    }
    for (int i = 0; i < OUT; ++i) {
        table[4 * IN + i] = 0.f;
        table[4 * IN + OUT + i] = 1.f;
    }
    float* d_table = NULL;
    MTRY(cudaMalloc((void**)&d_table, sizeof(table)));
    MTRY(cudaMemcpy(d_table, table, sizeof(table), cudaMemcpyHostToDevice));
    nbsp_mlp_set_scaling(c->net, d_table, c->stream);
    nbsp_mlp_build_frags(c->params, c->frags, c->net, c->stream);
    MTRY(cudaStreamSynchronize(c->stream));
    cudaFree(d_table);
    c->adam_step = 0;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProCudaCorrection* n_body_sim_pro_cuda_correction_create(uint64_t seed,
                                                                 NBodySimProError* error) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        mfail(error, N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM, __LINE__, "no CUDA device");
        return NULL;
    }
    NBodySimProCudaCorrection* c = (NBodySimProCudaCorrection*)calloc(1, sizeof(*c));
    if (c == NULL) {
        mfail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "correction allocation");
        return NULL;
    }
    c->seed = seed;
    const size_t np = (size_t)nbsp_mlp_param_count();
    cudaError_t code = cudaGetDevice(&c->device);
    if (code == cudaSuccess) code = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->params, np * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->m, np * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->v, np * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc((void**)&c->grad, np * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc(&c->frags, nbsp_mlp_frags_bytes());
    if (code == cudaSuccess) code = cudaMalloc(&c->net, nbsp_mlp_net_bytes());
    if (code == cudaSuccess) code = cudaMallocHost((void**)&c->host_loss, 1 << 20);
    if (code != cudaSuccess) {
        mcuda(error, code, __LINE__, "correction set-up");
        n_body_sim_pro_cuda_correction_destroy(c);
        return NULL;
    }
    if (init_parameters(c, error) != N_BODY_SIM_PRO_STATUS_OK) {
        n_body_sim_pro_cuda_correction_destroy(c);
        return NULL;
    }
    return c;
}

const void* nbsp_correction_net(const NBodySimProCudaCorrection* c) {
    return c != NULL ? c->net : NULL;
}

static NBodySimProStatus ensure_slots(NBodySimProCudaCorrection* c, int slots,
                                      NBodySimProError* error) {
    if (slots <= c->slots) return N_BODY_SIM_PRO_STATUS_OK;
    cudaFree(c->partial);
    cudaFree(c->loss);
    c->partial = NULL;
    c->loss = NULL;
    c->slots = 0;
    MTRY(cudaMalloc((void**)&c->partial, (size_t)slots * nbsp_mlp_param_count() * sizeof(float)));
    MTRY(cudaMalloc((void**)&c->loss, (size_t)slots * sizeof(float)));
    c->slots = slots;
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_generate(NBodySimProCudaCorrection* c,
                                                          NBodySimProCudaContext* ctx,
                                                          const NBodySimProGravity* gravity,
                                                          double theta, size_t samples,
                                                          uint64_t seed, NBodySimProError* error) {
    if (c == NULL || ctx == NULL || gravity == NULL || samples < 128 || samples > (1u << 26) ||
        !(theta > 0.0))
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "correction, context and gravity must not be null; 128 <= samples <= 2^26; "
                     "theta > 0");
    NbspTreeRef tr;
    NBodySimProStatus st = nbsp_context_tree(ctx, gravity, &tr, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    MTRY(cudaSetDevice(c->device));
    free_data(c);
    int *target = NULL, *cell = NULL, *ok = NULL;
    float *feat = NULL, *lab = NULL;
    const int ns = (int)samples;
    MTRY(cudaMalloc((void**)&target, samples * sizeof(int)));
    MTRY(cudaMalloc((void**)&cell, samples * sizeof(int)));
    MTRY(cudaMalloc((void**)&ok, samples * sizeof(int)));
    MTRY(cudaMalloc((void**)&feat, samples * IN * sizeof(float)));
    MTRY(cudaMalloc((void**)&lab, samples * OUT * sizeof(float)));
    nbsp_bh_mlp_pairs(tr.pos4, tr.n, tr.tree, (float)theta, tr.opening, seed, ns, target, cell, tr.status,
                      tr.stream);
    nbsp_bh_mlp_labels(tr.pos4, tr.n, tr.tree, target, cell, ns, (float)gravity->softening_squared,
                       feat, lab, ok, tr.stream);
    MTRY(cudaGetLastError());
    MTRY(cudaStreamSynchronize(tr.stream));
    /* keep the rows that found a cell (compaction on the host) */
    int* h_ok = (int*)malloc(samples * sizeof(int));
    float* h_feat = (float*)malloc(samples * IN * sizeof(float));
    float* h_lab = (float*)malloc(samples * OUT * sizeof(float));
    NBodySimProStatus result = N_BODY_SIM_PRO_STATUS_OK;
    if (h_ok == NULL || h_feat == NULL || h_lab == NULL) {
        result = mfail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "sample staging");
    } else if (cudaMemcpy(h_ok, ok, samples * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
               cudaMemcpy(h_feat, feat, samples * IN * sizeof(float), cudaMemcpyDeviceToHost) !=
                   cudaSuccess ||
               cudaMemcpy(h_lab, lab, samples * OUT * sizeof(float), cudaMemcpyDeviceToHost) !=
                   cudaSuccess) {
        result = mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__, "sample download");
    }
    size_t kept = 0;
    if (result == N_BODY_SIM_PRO_STATUS_OK) {
        for (size_t r = 0; r < samples; ++r) {
            if (!h_ok[r]) continue;
            int finite = 1;
            for (int q = 0; q < IN; ++q) finite &= isfinite(h_feat[r * IN + q]);
            for (int q = 0; q < OUT; ++q) finite &= isfinite(h_lab[r * OUT + q]);
            if (!finite) continue;
            memmove(h_feat + kept * IN, h_feat + r * IN, IN * sizeof(float));
            memmove(h_lab + kept * OUT, h_lab + r * OUT, OUT * sizeof(float));
            ++kept;
        }
        kept -= kept % 128; /* whole 128-row tiles */
        if (kept < 256)
            result = mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__,
                           "too few cell-target pairs (system too small?)");
    }
    cudaFree(target);
    cudaFree(cell);
    cudaFree(ok);
    cudaFree(feat);
    cudaFree(lab);
    if (result == N_BODY_SIM_PRO_STATUS_OK) {
        cudaError_t code = cudaMalloc((void**)&c->feat, kept * IN * sizeof(float));
        if (code == cudaSuccess) code = cudaMalloc((void**)&c->lab, kept * OUT * sizeof(float));
        if (code == cudaSuccess) code = cudaMalloc((void**)&c->x, kept * 8 * sizeof(uint32_t));
        if (code == cudaSuccess) code = cudaMalloc((void**)&c->y, kept * OUT * sizeof(float));
        if (code == cudaSuccess) code = cudaMalloc((void**)&c->order, kept * sizeof(int));
        if (code == cudaSuccess)
            code = cudaMemcpy(c->feat, h_feat, kept * IN * sizeof(float), cudaMemcpyHostToDevice);
        if (code == cudaSuccess)
            code = cudaMemcpy(c->lab, h_lab, kept * OUT * sizeof(float), cudaMemcpyHostToDevice);
        if (code != cudaSuccess) result = mcuda(error, code, __LINE__, "training set upload");
    }
    free(h_ok);
    free(h_feat);
    free(h_lab);
    if (result != N_BODY_SIM_PRO_STATUS_OK) {
        free_data(c);
        return result;
    }
    c->rows = kept;
    c->train_rows = kept - (kept / 16) / 128 * 128; /* last sixteenth: validation */
    nbsp_bh_mlp_stats(c->feat, c->lab, NULL, (int)kept, c->net, c->stream);
    nbsp_mlp_standardise(c->feat, c->lab, (int)kept, c->net, c->x, c->y, c->stream);
    MTRY(cudaGetLastError());
    MTRY(cudaStreamSynchronize(c->stream));
    return N_BODY_SIM_PRO_STATUS_OK;
}

/* Mean loss over rows [first, first + count) in identity order (no update). */
static NBodySimProStatus evaluate(NBodySimProCudaCorrection* c, size_t first, size_t count,
                                  double* loss, NBodySimProError* error) {
    const int per = nbsp_mlp_rows_per_cta();
    const int ctas = (int)(count / (size_t)per);
    if (ctas == 0) {
        *loss = 0.0;
        return N_BODY_SIM_PRO_STATUS_OK;
    }
    NBodySimProStatus st = ensure_slots(c, ctas, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    int* ident = (int*)malloc(count * sizeof(int));
    if (ident == NULL) return mfail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "order");
    for (size_t r = 0; r < count; ++r) ident[r] = (int)(first + r);
    cudaError_t code = cudaMemcpyAsync(c->order, ident, count * sizeof(int), cudaMemcpyHostToDevice,
                                       c->stream);
    if (code == cudaSuccess) {
        nbsp_mlp_train_step(c->x, c->y, c->order, 0, (int)count, ctas, 1.f / (3.f * (float)count),
                            c->frags, c->partial, c->loss, c->stream);
        code = cudaMemcpyAsync(c->host_loss, c->loss, (size_t)ctas * sizeof(float),
                               cudaMemcpyDeviceToHost, c->stream);
    }
    if (code == cudaSuccess) code = cudaStreamSynchronize(c->stream);
    free(ident);
    if (code != cudaSuccess) return mcuda(error, code, __LINE__, "evaluation");
    double s = 0.0;
    for (int k = 0; k < ctas; ++k) s += c->host_loss[k];
    *loss = s / (3.0 * (double)count);
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_train(NBodySimProCudaCorrection* c, int epochs,
                                                       int batch, double learning_rate,
                                                       double* train_loss, double* validation_loss,
                                                       NBodySimProError* error) {
    const int per = nbsp_mlp_rows_per_cta();
    if (c == NULL || epochs < 0 || batch < per || batch % per != 0 || !(learning_rate > 0.0))
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "epochs >= 0, batch a positive multiple of 128, learning rate > 0");
    if (c->rows == 0)
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__,
                     "no training set: call n_body_sim_pro_cuda_correction_generate first");
    MTRY(cudaSetDevice(c->device));
    const int ctas = batch / per;
    NBodySimProStatus st = ensure_slots(c, ctas, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    const size_t n = c->train_rows;
    int* order = (int*)malloc(n * sizeof(int));
    if (order == NULL) return mfail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "order");
    uint64_t s = c->seed ^ 0x5DEECE66Dull;
    for (int epoch = 0; epoch < epochs; ++epoch) {
        for (size_t r = 0; r < n; ++r) order[r] = (int)r;
        for (size_t r = n - 1; r > 0; --r) { /* Fisher-Yates */
            const size_t j = (size_t)(splitmix(&s) % (r + 1));
            const int tmp = order[r];
            order[r] = order[j];
            order[j] = tmp;
        }
        cudaError_t code = cudaMemcpyAsync(c->order, order, n * sizeof(int), cudaMemcpyHostToDevice,
                                           c->stream);
        for (size_t first = 0; code == cudaSuccess && first + (size_t)batch <= n; first += batch) {
            nbsp_mlp_train_step(c->x, c->y, c->order, (int)first, (int)n, ctas,
                                1.f / (3.f * (float)batch), c->frags, c->partial, c->loss,
                                c->stream);
            nbsp_mlp_reduce_adam(c->partial, ctas, NULL, c->params, c->m, c->v,
                                 (float)learning_rate, ++c->adam_step, 1, c->stream);
            nbsp_mlp_build_frags(c->params, c->frags, c->net, c->stream);
            code = cudaGetLastError();
        }
        if (code == cudaSuccess) code = cudaStreamSynchronize(c->stream);
        if (code != cudaSuccess) {
            free(order);
            return mcuda(error, code, __LINE__, "training step");
        }
        double tl = 0.0, vl = 0.0;
        if (train_loss != NULL && (st = evaluate(c, 0, n, &tl, error)) != N_BODY_SIM_PRO_STATUS_OK) break;
        if (validation_loss != NULL &&
            (st = evaluate(c, n, c->rows - n, &vl, error)) != N_BODY_SIM_PRO_STATUS_OK)
            break;
        if (train_loss != NULL) train_loss[epoch] = tl;
        if (validation_loss != NULL) validation_loss[epoch] = vl;
    }
    free(order);
    return st;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_get_parameters(
    NBodySimProCudaCorrection* c, float* params, float* scaling, NBodySimProError* error) {
    if (c == NULL) return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "null");
    MTRY(cudaSetDevice(c->device));
    if (params != NULL)
        MTRY(cudaMemcpy(params, c->params, (size_t)nbsp_mlp_param_count() * sizeof(float),
                        cudaMemcpyDeviceToHost));
    if (scaling != NULL) {
        float* d = NULL;
        MTRY(cudaMalloc((void**)&d, SCALING * sizeof(float)));
        nbsp_mlp_get_scaling(c->net, d, c->stream);
        cudaError_t code = cudaStreamSynchronize(c->stream);
        if (code == cudaSuccess)
            code = cudaMemcpy(scaling, d, SCALING * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(d);
        if (code != cudaSuccess) return mcuda(error, code, __LINE__, "scaling download");
    }
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_set_parameters(
    NBodySimProCudaCorrection* c, const float* params, const float* scaling,
    NBodySimProError* error) {
    if (c == NULL) return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "null");
    MTRY(cudaSetDevice(c->device));
    if (params != NULL)
        MTRY(cudaMemcpy(c->params, params, (size_t)nbsp_mlp_param_count() * sizeof(float),
                        cudaMemcpyHostToDevice));
    if (scaling != NULL) {
        float* d = NULL;
        MTRY(cudaMalloc((void**)&d, SCALING * sizeof(float)));
        cudaError_t code = cudaMemcpy(d, scaling, SCALING * sizeof(float), cudaMemcpyHostToDevice);
        if (code == cudaSuccess) {
            nbsp_mlp_set_scaling(c->net, d, c->stream);
            code = cudaStreamSynchronize(c->stream);
        }
        cudaFree(d);
        if (code != cudaSuccess) return mcuda(error, code, __LINE__, "scaling upload");
    }
    nbsp_mlp_build_frags(c->params, c->frags, c->net, c->stream);
    MTRY(cudaGetLastError());
    MTRY(cudaStreamSynchronize(c->stream));
    c->adam_step = 0;
    MTRY(cudaMemset(c->m, 0, (size_t)nbsp_mlp_param_count() * sizeof(float)));
    MTRY(cudaMemset(c->v, 0, (size_t)nbsp_mlp_param_count() * sizeof(float)));
    return N_BODY_SIM_PRO_STATUS_OK;
}

static uint32_t bf16_bits(float f) { /* round to nearest even */
    uint32_t u;
    memcpy(&u, &f, sizeof(u));
    if ((u & 0x7f800000u) == 0x7f800000u) return (u >> 16) | ((u & 0xffffu) ? 0x40u : 0u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return u >> 16;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_gradient(NBodySimProCudaCorrection* c,
                                                          const float* features,
                                                          const float* labels, size_t rows,
                                                          float* gradient, double* loss,
                                                          NBodySimProError* error) {
    const int per = nbsp_mlp_rows_per_cta();
    if (c == NULL || features == NULL || labels == NULL || gradient == NULL || rows == 0 ||
        rows % (size_t)per != 0 || rows > (1u << 20))
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "rows must be a positive multiple of 128 (<= 2^20) and buffers non-null");
    MTRY(cudaSetDevice(c->device));
    const int ctas = (int)(rows / (size_t)per);
    NBodySimProStatus st = ensure_slots(c, ctas, error);
    if (st != N_BODY_SIM_PRO_STATUS_OK) return st;
    uint32_t* hx = (uint32_t*)malloc(rows * 8 * sizeof(uint32_t));
    int* ident = (int*)malloc(rows * sizeof(int));
    uint32_t* dx = NULL;
    float* dy = NULL;
    int* dorder = NULL;
    if (hx == NULL || ident == NULL) {
        free(hx);
        free(ident);
        return mfail(error, N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY, __LINE__, "staging");
    }
    for (size_t r = 0; r < rows; ++r) {
        ident[r] = (int)r;
        for (int w = 0; w < 8; ++w) {
            const float a = 2 * w < IN ? features[r * IN + 2 * w] : 0.f;
            const float b = 2 * w + 1 < IN ? features[r * IN + 2 * w + 1] : 0.f;
            hx[r * 8 + w] = bf16_bits(a) | (bf16_bits(b) << 16);
        }
    }
    cudaError_t code = cudaMalloc((void**)&dx, rows * 8 * sizeof(uint32_t));
    if (code == cudaSuccess) code = cudaMalloc((void**)&dy, rows * OUT * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc((void**)&dorder, rows * sizeof(int));
    if (code == cudaSuccess)
        code = cudaMemcpy(dx, hx, rows * 8 * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (code == cudaSuccess)
        code = cudaMemcpy(dy, labels, rows * OUT * sizeof(float), cudaMemcpyHostToDevice);
    if (code == cudaSuccess)
        code = cudaMemcpy(dorder, ident, rows * sizeof(int), cudaMemcpyHostToDevice);
    if (code == cudaSuccess) {
        nbsp_mlp_train_step(dx, dy, dorder, 0, (int)rows, ctas, 1.f / (3.f * (float)rows),
                            c->frags, c->partial, c->loss, c->stream);
        nbsp_mlp_reduce_adam(c->partial, ctas, c->grad, c->params, c->m, c->v, 0.f, 1, 0,
                             c->stream);
        code = cudaGetLastError();
    }
    if (code == cudaSuccess)
        code = cudaMemcpyAsync(c->host_loss, c->loss, (size_t)ctas * sizeof(float),
                               cudaMemcpyDeviceToHost, c->stream);
    if (code == cudaSuccess) code = cudaStreamSynchronize(c->stream);
    if (code == cudaSuccess)
        code = cudaMemcpy(gradient, c->grad, (size_t)nbsp_mlp_param_count() * sizeof(float),
                          cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dorder);
    free(hx);
    free(ident);
    if (code != cudaSuccess) return mcuda(error, code, __LINE__, "gradient");
    if (loss != NULL) {
        double s = 0.0;
        for (int k = 0; k < ctas; ++k) s += c->host_loss[k];
        *loss = s / (3.0 * (double)rows);
    }
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_samples(NBodySimProCudaCorrection* c,
                                                         size_t* rows, float* features,
                                                         float* labels, size_t max_rows,
                                                         NBodySimProError* error) {
    if (c == NULL || rows == NULL)
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "null");
    MTRY(cudaSetDevice(c->device));
    *rows = c->rows;
    const size_t k = c->rows < max_rows ? c->rows : max_rows;
    if (features != NULL && k > 0)
        MTRY(cudaMemcpy(features, c->feat, k * IN * sizeof(float), cudaMemcpyDeviceToHost));
    if (labels != NULL && k > 0)
        MTRY(cudaMemcpy(labels, c->lab, k * OUT * sizeof(float), cudaMemcpyDeviceToHost));
    return N_BODY_SIM_PRO_STATUS_OK;
}

NBodySimProStatus n_body_sim_pro_cuda_correction_evaluate(NBodySimProCudaCorrection* c,
                                                          const float* features, size_t rows,
                                                          float* outputs, int engine,
                                                          NBodySimProError* error) {
    if (c == NULL || (rows > 0 && (features == NULL || outputs == NULL)))
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "correction, features and outputs must not be null");
    if (engine != N_BODY_SIM_PRO_CUDA_MLP_TCGEN05 && engine != N_BODY_SIM_PRO_CUDA_MLP_MMA_SYNC)
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__, "unknown engine");
    if (rows > (size_t)(1 << 30))
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                     "at most 2^30 rows per call");
    if (rows == 0) return N_BODY_SIM_PRO_STATUS_OK;
    MTRY(cudaSetDevice(c->device));
    float *d_in = NULL, *d_out = NULL;
    int* d_status = NULL;
    int host_status = 0;
    cudaError_t code = cudaMalloc((void**)&d_in, rows * IN * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc((void**)&d_out, rows * OUT * sizeof(float));
    if (code == cudaSuccess) code = cudaMalloc((void**)&d_status, sizeof(int));
    if (code == cudaSuccess) code = cudaMemsetAsync(d_status, 0, sizeof(int), c->stream);
    if (code == cudaSuccess)
        code = cudaMemcpyAsync(d_in, features, rows * IN * sizeof(float), cudaMemcpyHostToDevice,
                               c->stream);
    if (code == cudaSuccess) {
        nbsp_mlp_evaluate(c->net, d_in, (int)rows, d_out, engine == N_BODY_SIM_PRO_CUDA_MLP_TCGEN05,
                          d_status, c->stream);
        code = cudaGetLastError();
    }
    if (code == cudaSuccess)
        code = cudaMemcpyAsync(outputs, d_out, rows * OUT * sizeof(float), cudaMemcpyDeviceToHost,
                               c->stream);
    if (code == cudaSuccess)
        code = cudaMemcpyAsync(&host_status, d_status, sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream);
    if (code == cudaSuccess) code = cudaStreamSynchronize(c->stream);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_status);
    if (code != cudaSuccess) return mcuda(error, code, __LINE__, "correction evaluate");
    if (host_status != 0)
        return mfail(error, N_BODY_SIM_PRO_STATUS_INVALID_STATE, __LINE__,
                     "correction network: a tensor-core product did not complete in time");
    return N_BODY_SIM_PRO_STATUS_OK;
}
