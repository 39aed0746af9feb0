/*
 * Internal interface between the C17 host layer (api.c) and the CUDA kernel
 * launchers (*.cu).  Not installed; every symbol here has hidden visibility.
 *
 * All launchers enqueue on `stream` and never synchronise; device pointers only.
 */
#ifndef NBSP_CUDA_INTERNAL_H
#define NBSP_CUDA_INTERNAL_H

#include <cuda_runtime_api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBSP_HIDDEN __attribute__((visibility("hidden")))

/* Kernels this process has launched through the library (every <<<>>> site
 * counts itself; read by n_body_sim_pro_cuda_kernel_launches). */
NBSP_HIDDEN extern unsigned long long nbsp_kernel_launch_count;
#define NBSP_COUNT_LAUNCH(k) \
    __atomic_fetch_add(&nbsp_kernel_launch_count, (unsigned long long)(k), __ATOMIC_RELAXED)

/* Device status bits (OR-ed into one device int by kernels, read by the host). */
enum {
    NBSP_DEVICE_ERROR_NONFINITE_POSITION = 1,
    NBSP_DEVICE_ERROR_WALK_LIMIT = 2,
    NBSP_DEVICE_ERROR_TREE_INCONSISTENT = 4,
    NBSP_DEVICE_ERROR_ENSEMBLE_LIMIT = 8,
    NBSP_DEVICE_ERROR_DUPLICATE_POSITION = 16,
    /* a tensor-core product (tcgen05) did not complete within its wait limit */
    NBSP_DEVICE_ERROR_MMA_TIMEOUT = 32
};

/* ---- all-pairs / KDK / diagnostics (allpairs.cu) ------------------------- */

/* Tile shape of the all-pairs force kernel, chosen by the host autotuner. */
typedef struct NbspAllPairsShape {
    int block;        /* threads per CTA (64, 128 or 256) */
    int per_thread;   /* targets per thread (1, 2, 4 or 8) */
    int chunks;       /* source chunks S (grid.y); partials reduced in FP64 */
    int paired;       /* 1: targets processed in pairs with fma/add/mul.f32x2 */
    int min_blocks;   /* paired only: CTAs per SM the registers are capped for (0: none) */
} NbspAllPairsShape;

/* Sources of one chunk: ceil(n_padded / chunks) rounded up to a multiple of
 * NBSP_ALLPAIRS_CHUNK_ALIGN (trailing chunks may be short or empty). */
#define NBSP_ALLPAIRS_CHUNK_ALIGN 8
static inline size_t nbsp_allpairs_chunk_len(size_t n_padded, int chunks) {
    const size_t units = (n_padded + NBSP_ALLPAIRS_CHUNK_ALIGN - 1) / NBSP_ALLPAIRS_CHUNK_ALIGN;
    const size_t c = chunks < 1 ? 1 : (size_t)chunks;
    return (units + c - 1) / c * NBSP_ALLPAIRS_CHUNK_ALIGN;
}

/* Number of CTAs per SM the force kernel of this shape can keep resident. */
NBSP_HIDDEN int nbsp_allpairs_resident_ctas(NbspAllPairsShape shape);
NBSP_HIDDEN int nbsp_allpairs_shape_supported(NbspAllPairsShape shape);

/* FP64 state -> float4 (x - c, y - c, z - c, m); entries n..n_padded-1 are zero. */
NBSP_HIDDEN void nbsp_pack_relative(const double* x, const double* y, const double* z,
                                    const double* m, size_t n, size_t n_padded,
                                    const double* centre, void* packed, int* status,
                                    cudaStream_t stream);

/* Softened forces of all sources on all targets, written as S compensated
 * partials: hi[s*n + i], lo[s*n + i] (float4, w unused). */
NBSP_HIDDEN void nbsp_allpairs_force(const void* packed, size_t n, size_t n_padded,
                                     float softening_squared, NbspAllPairsShape shape,
                                     void* partial_hi, void* partial_lo, cudaStream_t stream);

/* The same for n_targets targets (float4, same frame) against the first
 * n_sources_padded packed sources (a multiple of NBSP_ALLPAIRS_CHUNK_ALIGN;
 * trailing entries massless): hi[s*n_targets + i], lo[...]. */
NBSP_HIDDEN void nbsp_allpairs_force_targets(const void* sources, size_t n_sources_padded,
                                             const void* targets, size_t n_targets,
                                             float softening_squared, NbspAllPairsShape shape,
                                             void* partial_hi, void* partial_lo,
                                             cudaStream_t stream);

/* Accelerations a = G * sum_s (hi_s + lo_s) in FP64 into ax, ay, az. */
NBSP_HIDDEN void nbsp_allpairs_finalize(const void* partial_hi, const void* partial_lo, size_t n,
                                        int chunks, double gravitational_constant, double* ax,
                                        double* ay, double* az, cudaStream_t stream);

/* Kick (v += a*h) and, when `drift` is set, drift (x += v*dt) in FP64, then
 * repack the relative float4 positions.  The leapfrog/Verlet opening half. */
NBSP_HIDDEN void nbsp_kick_drift(double* x, double* y, double* z, double* vx, double* vy,
                                 double* vz, const double* ax, const double* ay,
                                 const double* az, size_t n, double kick, double drift,
                                 cudaStream_t stream);

/* Euler: x += v*dt then v += a*dt (integrator.c:15-45 order). */
NBSP_HIDDEN void nbsp_euler_update(double* x, double* y, double* z, double* vx, double* vy,
                                   double* vz, const double* ax, const double* ay,
                                   const double* az, size_t n, double dt, cudaStream_t stream);

/* Closing half kick fused with the all-pairs reduction:
 * a = G * sum_s partials; store a; v += a*h. */
NBSP_HIDDEN void nbsp_allpairs_finalize_kick(const void* partial_hi, const void* partial_lo,
                                             size_t n, int chunks, double gravitational_constant,
                                             double* ax, double* ay, double* az, double* vx,
                                             double* vy, double* vz, double half_dt,
                                             cudaStream_t stream);

/* Closing half kick of step n fused with the opening half kick + drift of
 * step n+1 and the repack: a = G * sum partials; v += a*h; store a;
 * v += a*h; x += v*dt; packed = (x - c, m). */
NBSP_HIDDEN void nbsp_allpairs_finalize_kick_kick_drift_pack(
    const void* partial_hi, const void* partial_lo, size_t n, size_t n_padded, int chunks,
    double gravitational_constant, double* x, double* y, double* z, double* vx, double* vy,
    double* vz, double* ax, double* ay, double* az, const double* m, double half_dt, double dt,
    const double* centre, void* packed, int* status, cudaStream_t stream);

/* O(N) global quantities in FP64 (numerics.c:5-81): out[0..10] = KE, M,
 * P xyz, L xyz, sum m r xyz (the host divides by M).  Deterministic: fixed
 * block partition, fixed-order second stage. `scratch` >= 11 * 1024 doubles. */
NBSP_HIDDEN void nbsp_global_sums(const double* x, const double* y, const double* z,
                                  const double* vx, const double* vy, const double* vz,
                                  const double* m, size_t n, double* scratch, double* out,
                                  cudaStream_t stream);

/* Centre of mass into centre[0..2] (FP64; uses scratch like nbsp_global_sums). */
NBSP_HIDDEN void nbsp_centre_of_mass(const double* x, const double* y, const double* z,
                                     const double* m, size_t n, double* scratch, double* centre,
                                     cudaStream_t stream);

/* O(N^2) FP64 potential energy -G sum_{i<j} m_i m_j / sqrt(d^2 + eps^2).
 * `rows` >= n doubles; result in out[0]. */
NBSP_HIDDEN void nbsp_potential_energy(const double* x, const double* y, const double* z,
                                       const double* m, size_t n, double gravitational_constant,
                                       double softening_squared, double* rows, double* out,
                                       cudaStream_t stream);

/* FP64 direct sums on `count` target indices over all n sources
 * (gravity.c:37-67 pair arithmetic, j == i skipped), out[3*t + c].
 * `scratch` >= 2 * 3 * count * chunks doubles. */
NBSP_HIDDEN void nbsp_reference_subset(const double* x, const double* y, const double* z,
                                       const double* m, size_t n, const int64_t* targets,
                                       size_t count, double gravitational_constant,
                                       double softening_squared, double* scratch, int chunks,
                                       double* out, cudaStream_t stream);

/* Write `bytes` of junk into `buffer` (used to flush L2 between timed runs). */
NBSP_HIDDEN void nbsp_touch(void* buffer, size_t bytes, cudaStream_t stream);

/* ---- device preset generation (presets.cu) -------------------------------- */

/* FP64 scratch words nbsp_preset_generate needs for n particles. */
NBSP_HIDDEN size_t nbsp_preset_scratch_doubles(size_t n);

/* presets_parallel.c on the device into the FP64 state arrays (length n):
 * `preset` is an NBodySimProSimulationPreset value.  Returns 0, or 1 when the
 * count does not fit the preset (as the reference's INVALID_ARGUMENT). */
NBSP_HIDDEN int nbsp_preset_generate(int preset, size_t n, uint64_t seed, double* x, double* y,
                                     double* z, double* vx, double* vy, double* vz, double* m,
                                     double* scratch, cudaStream_t stream);
/* Two Plummer spheres from the parallel presets' per-particle streams
 * (presets.cu); 0 on success, 1 for n < 2. */
NBSP_HIDDEN int nbsp_plummer_collision_generate(size_t n, uint64_t seed, double a,
                                                double separation, double relative_speed,
                                                double* x, double* y, double* z, double* vx,
                                                double* vy, double* vz, double* m,
                                                double* scratch, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif
