/*
 * n_body_sim_pro_cuda.h — B200 (sm_100a) force evaluation and time step for the
 * n_body_sim_pro C engine, exposed as a C ABI.
 *
 * The library adds two algorithms behind the engine's existing force-kernel
 * plugin type
 *
 *   typedef NBodySimProStatus (*NBodySimProForceFunction)(
 *       const NBodySimProParticleSystemView*, const NBodySimProGravity*,
 *       void* context, NBodySimProError*);      (physics/integrator.h:47-49)
 *
 *   cuda             n_body_sim_pro_gravity_compute_acceleration_cuda
 *   barnes_hut_cuda  n_body_sim_pro_barnes_hut_compute_acceleration_cuda
 *
 * plus a device-resident stepping API (upload once, advance many fused
 * kick-drift-kick steps on the GPU, download) for throughput.
 *
 * Conventions (all follow the reference engine):
 *   - every function returns NBodySimProStatus and fills the optional
 *     NBodySimProError* (NULL allowed) like n_body_sim_pro_error_set
 *     (src/c/core/status.c:29);
 *   - NULL view / gravity -> N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT
 *     (src/c/physics/gravity.c:19-23);
 *   - accelerations are OVERWRITTEN, never accumulated (physics/gravity.h:43-44);
 *   - no CPU fallback: without a usable CUDA device the functions return
 *     N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM.
 *
 * Numerics: forces in FP32 on positions relative to the FP64 centre of mass,
 * with compensated (TwoSum) accumulation; positions, velocities, the drift,
 * the kick and all diagnostics in FP64.
 *
 * The reference's own types are re-declared here, layout-identical, for
 * callers that do not have the engine's headers.  When the engine's headers
 * are included BEFORE this one, their include guards suppress these copies.
 */
#ifndef N_BODY_SIM_PRO_CUDA_H
#define N_BODY_SIM_PRO_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define N_BODY_SIM_PRO_CUDA_API
#else
#define N_BODY_SIM_PRO_CUDA_API __attribute__((visibility("default")))
#endif

/* ---- reference types (layout-identical copies) ---------------------------- */

#ifndef N_BODY_SIM_PRO_CORE_STATUS_H
/* include/n_body_sim_pro/core/status.h:18-35 */
typedef enum NBodySimProStatus {
    N_BODY_SIM_PRO_STATUS_OK = 0,
    N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT,
    N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY,
    N_BODY_SIM_PRO_STATUS_INVALID_STATE,
    N_BODY_SIM_PRO_STATUS_NOT_IMPLEMENTED,
    N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM,
    N_BODY_SIM_PRO_STATUS_OVERFLOW,
    N_BODY_SIM_PRO_STATUS_IO_ERROR,
    N_BODY_SIM_PRO_STATUS_INSUFFICIENT_MEMORY
} NBodySimProStatus;

typedef struct NBodySimProError {
    NBodySimProStatus status;
    const char* source_file;
    int source_line;
    char message[256];
} NBodySimProError;
#endif

#ifndef N_BODY_SIM_PRO_CORE_PARTICLE_SYSTEM_H
/* include/n_body_sim_pro/core/particle_system.h:38-50 */
typedef struct NBodySimProParticleSystemView {
    size_t particle_count;
    double* positions_x;
    double* positions_y;
    double* positions_z;
    double* velocities_x;
    double* velocities_y;
    double* velocities_z;
    double* accelerations_x;
    double* accelerations_y;
    double* accelerations_z;
    double* masses;
} NBodySimProParticleSystemView;
#endif

#ifndef N_BODY_SIM_PRO_PHYSICS_GRAVITY_H
/* include/n_body_sim_pro/physics/gravity.h:25-29 */
typedef struct NBodySimProGravity {
    double gravitational_constant;
    double softening_length;
    double softening_squared;
} NBodySimProGravity;
#endif

#ifndef N_BODY_SIM_PRO_PHYSICS_INTEGRATOR_H
/* include/n_body_sim_pro/physics/integrator.h:31-35 */
typedef enum NBodySimProIntegratorType {
    N_BODY_SIM_PRO_INTEGRATOR_EULER,
    N_BODY_SIM_PRO_INTEGRATOR_LEAPFROG,
    N_BODY_SIM_PRO_INTEGRATOR_VELOCITY_VERLET
} NBodySimProIntegratorType;
#endif

#ifndef N_BODY_SIM_PRO_BARNES_HUT_BARNES_HUT_H
/* include/n_body_sim_pro/barnes_hut/barnes_hut.h:31-40 */
typedef struct NBodySimProBarnesHutStats {
    size_t node_count;
    size_t leaf_count;
    size_t internal_node_count;
    size_t accepted_approximations;
    size_t exact_interactions;
    size_t maximum_depth;
    double build_time_seconds;
    double evaluation_time_seconds;
} NBodySimProBarnesHutStats;
#endif

#ifndef N_BODY_SIM_PRO_DIAGNOSTICS_NUMERICS_H
/* include/n_body_sim_pro/diagnostics/numerics.h:22-34 */
typedef struct NBodySimProDiagnosticsQuantities {
    double kinetic_energy;
    double total_mass;
    double total_momentum_x;
    double total_momentum_y;
    double total_momentum_z;
    double total_angular_momentum_x;
    double total_angular_momentum_y;
    double total_angular_momentum_z;
    double center_of_mass_x;
    double center_of_mass_y;
    double center_of_mass_z;
} NBodySimProDiagnosticsQuantities;
#endif

#ifndef N_BODY_SIM_PRO_GENERATION_PRESETS_H
/* include/n_body_sim_pro/generation/presets.h:27-46 */
typedef enum NBodySimProSimulationPreset {
    N_BODY_SIM_PRO_PRESET_TWO_BODY,
    N_BODY_SIM_PRO_PRESET_RANDOM_CLOUD,
    N_BODY_SIM_PRO_PRESET_SOLAR_SYSTEM,
    N_BODY_SIM_PRO_PRESET_OPEN_CLUSTER,
    N_BODY_SIM_PRO_PRESET_GLOBULAR_CLUSTER,
    N_BODY_SIM_PRO_PRESET_SPIRAL_GALAXY,
    N_BODY_SIM_PRO_PRESET_ELLIPTICAL_GALAXY,
    N_BODY_SIM_PRO_PRESET_GALAXY_COLLISION,
    N_BODY_SIM_PRO_PRESET_TRIPLE_GALAXY,
    N_BODY_SIM_PRO_PRESET_COUNT
} NBodySimProSimulationPreset;

typedef struct NBodySimProPresetParameters {
    size_t particle_count;
    uint64_t random_seed;
} NBodySimProPresetParameters;
#endif

#ifndef N_BODY_SIM_PRO_CHECKPOINT_CHECKPOINT_H
/* include/n_body_sim_pro/checkpoint/checkpoint.h:27-41 */
enum { N_BODY_SIM_PRO_CHECKPOINT_MAGIC = 0x53504348, N_BODY_SIM_PRO_CHECKPOINT_VERSION = 1 };

typedef struct NBodySimProCheckpointHeader {
    uint32_t magic;
    uint32_t version;
    size_t particle_count;
    double simulation_time;
    double timestep;
    int32_t integrator;
    double theta;
    int32_t barnes_hut_enabled;
    uint64_t random_seed;
    int32_t preset;
} NBodySimProCheckpointHeader;
#endif

/* ---- context ----------------------------------------------------------------- */

/*
 * Algorithm state for the CUDA force functions: device buffers, the CUDA
 * stream, Barnes-Hut parameters, the all-pairs tile autotune cache and the
 * statistics of the last evaluation.  Plays the role of the reference's
 * NBodySimProBarnesHutTree context (barnes_hut/barnes_hut.h:28-43) for both
 * CUDA algorithms.  One context must not be used from two host threads at once.
 */
typedef struct NBodySimProCudaContext NBodySimProCudaContext;

typedef enum NBodySimProCudaAlgorithm {
    N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS = 0,
    N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT = 1
} NBodySimProCudaAlgorithm;

/* Per-phase device time of the most recent evaluation, milliseconds (CUDA events). */
typedef struct NBodySimProCudaTimings {
    double bounds_ms;      /* bbox + centre-of-mass reduction */
    double keys_ms;        /* Morton keys */
    double sort_ms;        /* radix sort of keys + permutation */
    double build_ms;       /* gather + octree build */
    double moments_ms;     /* monopole / quadrupole pass */
    double walk_ms;        /* tree walk (Barnes-Hut) or all-pairs tiles */
    double integrate_ms;   /* kick / drift / scatter epilogue */
    double total_ms;
} NBodySimProCudaTimings;

/* Replaces n_body_sim_pro_barnes_hut_tree_create (barnes_hut/barnes_hut.h:43).
 * Selects the current CUDA device; NULL + UNSUPPORTED_PLATFORM when none. */
N_BODY_SIM_PRO_CUDA_API NBodySimProCudaContext* n_body_sim_pro_cuda_context_create(
    NBodySimProError* error);

/* Replaces n_body_sim_pro_barnes_hut_tree_destroy (barnes_hut/barnes_hut.h:46). NULL-safe. */
N_BODY_SIM_PRO_CUDA_API void n_body_sim_pro_cuda_context_destroy(NBodySimProCudaContext* context);

/* Replace n_body_sim_pro_barnes_hut_tree_set_theta / _theta (barnes_hut/barnes_hut.h:49-50).
 * Default 0.7 (src/c/barnes_hut/barnes_hut.c:28). */
N_BODY_SIM_PRO_CUDA_API void n_body_sim_pro_cuda_context_set_theta(NBodySimProCudaContext* context,
                                                                   double theta);
N_BODY_SIM_PRO_CUDA_API double n_body_sim_pro_cuda_context_theta(
    const NBodySimProCudaContext* context);

/* Multipole order of accepted cells: 1 = monopole (the reference's
 * barnes_hut.c:600-612), 2 = monopole + trace-free quadrupole (default 1). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_multipole_order(
    NBodySimProCudaContext* context, int order, NBodySimProError* error);

/* Largest particle count of a Barnes-Hut leaf bucket, 1..64 (default 16). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_leaf_capacity(
    NBodySimProCudaContext* context, int capacity, NBodySimProError* error);

/* Barnes-Hut walk.  All accept a cell only when the reference's test
 * (2h)^2 < theta^2 d^2 holds for every one of the 32 Morton-consecutive
 * targets it is applied to (src/c/barnes_hut/barnes_hut.c:596-599), so all
 * accept the same cells; they differ in how the traversal is scheduled:
 *   STACKLESS          one node at a time per warp along depth-first skip
 *                      links;
 *   INTERACTION_LISTS  (default) 32 nodes per step tested in parallel from a
 *                      per-warp stack, accepted cells and leaves gathered and
 *                      evaluated in dense loops;
 *   SHARED_TOP         INTERACTION_LISTS with the top of the tree traversed
 *                      once per block of 4 groups: nodes every group accepts
 *                      or opens are decided once, the rest by each group
 *                      (monopole walk; the others fall back to
 *                      INTERACTION_LISTS). */
typedef enum NBodySimProCudaWalk {
    N_BODY_SIM_PRO_CUDA_WALK_STACKLESS = 0,
    N_BODY_SIM_PRO_CUDA_WALK_INTERACTION_LISTS = 1,
    N_BODY_SIM_PRO_CUDA_WALK_SHARED_TOP = 2
} NBodySimProCudaWalk;

N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_walk(
    NBodySimProCudaContext* context, int walk, NBodySimProError* error);

/* Largest particle count of one context: the radix sort's look-back counts
 * are 30-bit and the kernels index particles with 32-bit integers.  (Device
 * memory binds first: ~0.6 KB per particle for Barnes-Hut.) */
#define N_BODY_SIM_PRO_CUDA_MAX_PARTICLES ((size_t)1073676288) /* 2^30 - 2^16 */

/* Opening test of the Barnes-Hut walk (a target-cell pair at distance d from the
 * cell's centre of mass, cell side 2h):
 *   REFERENCE  accept when (2h)^2 < theta^2 d^2 (barnes_hut.c:596-599; default);
 *   OFFSET     accept when 2h / theta + shift < d, shift = the distance from the
 *              cell's geometric centre to its centre of mass (Barnes 1994), so no
 *              target inside the cell accepts it at any theta <= 1.
 * Every cell OFFSET accepts, REFERENCE accepts too. */
typedef enum NBodySimProCudaOpening {
    N_BODY_SIM_PRO_CUDA_OPENING_REFERENCE = 0,
    N_BODY_SIM_PRO_CUDA_OPENING_OFFSET = 1
} NBodySimProCudaOpening;

N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_opening(
    NBodySimProCudaContext* context, int opening, NBodySimProError* error);

/* No reference counterpart: the relative opening test (Springel 2001) on top of
 * the geometric one.  With alpha > 0 a cell of mass M and side 2h is accepted
 * for a target only when also  G M (2h)^2 / d^4 <= alpha max(|a_old|, rms),
 * a_old the target's acceleration in the state (the previous evaluation's, or
 * what was uploaded / passed in the view) and rms the root mean square of
 * |a_old| over the state.  theta becomes a geometric bound on top (the test
 * is fastest at rms force error 1e-3 with a loose one, theta 5.0, and
 * alpha 0.0045).  A state without previous accelerations (all a_old zero, or
 * not finite) is evaluated with the geometric test alone at
 * min(theta, 0.5), so its first evaluation is an ordinary Barnes-Hut one and
 * the next reads its result.  0 (default) turns it off.  A learned correction
 * still corrects the monopole of the cells the combined test accepts. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_relative_opening(
    NBodySimProCudaContext* context, double alpha, NBodySimProError* error);

/* No reference counterpart: where the plugin functions take the relative
 * test's previous accelerations.  FROM_VIEW (default): the view's acceleration
 * arrays, uploaded with every call (24 bytes per particle).  FROM_CONTEXT: the
 * accelerations this context computed in its previous plugin call, kept on the
 * device, when that call had the same particle count and the same acceleration
 * arrays and no device-resident call came between; otherwise the view's, as
 * with FROM_VIEW.  The reference's integrators pass the previous call's output
 * back unchanged (integrator.c:47-85), so both give the same forces and
 * FROM_CONTEXT saves the upload; a caller that edits the accelerations between
 * calls wants FROM_VIEW. */
typedef enum NBodySimProCudaRelativeSource {
    N_BODY_SIM_PRO_CUDA_RELATIVE_FROM_VIEW = 0,
    N_BODY_SIM_PRO_CUDA_RELATIVE_FROM_CONTEXT = 1
} NBodySimProCudaRelativeSource;

N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_relative_source(
    NBodySimProCudaContext* context, int source, NBodySimProError* error);

/* Replaces n_body_sim_pro_barnes_hut_tree_stats (barnes_hut/barnes_hut.h:116-117):
 * 0 on success, non-zero when an argument is NULL. */
N_BODY_SIM_PRO_CUDA_API int n_body_sim_pro_cuda_context_stats(
    const NBodySimProCudaContext* context, NBodySimProBarnesHutStats* stats);

/* Device-event phase timings of the last evaluation or advance. 0 on success. */
N_BODY_SIM_PRO_CUDA_API int n_body_sim_pro_cuda_context_timings(
    const NBodySimProCudaContext* context, NBodySimProCudaTimings* timings);

/* No reference counterpart: in the last Barnes-Hut evaluation, the number of
 * 32-target groups whose interaction-list stack would have overflowed and that
 * were walked again by the stackless walk (same forces, more time). 0 for NULL. */
N_BODY_SIM_PRO_CUDA_API size_t n_body_sim_pro_cuda_context_walk_restarts(
    const NBodySimProCudaContext* context);

/* No reference counterpart: in the last Barnes-Hut evaluation with a learned
 * correction set, the number of (accepted cell, 32-target group) pairs the
 * network evaluated (each one forward pass of 9,856 flop on the tensor cores).
 * 0 for NULL or without a correction. */
N_BODY_SIM_PRO_CUDA_API size_t n_body_sim_pro_cuda_context_corrected_cells(
    const NBodySimProCudaContext* context);

/* ---- force functions (NBodySimProForceFunction) -------------------------------- */

/*
 * `cuda` algorithm: exact softened all-pairs sum (j == i excluded) on the GPU,
 * semantics of n_body_sim_pro_gravity_compute_acceleration_reference
 * (physics/gravity.h:46-59, src/c/physics/gravity.c:15-70).  `context` is an
 * NBodySimProCudaContext*, or NULL for a lazily created process-wide context
 * (one host thread at a time, like the reference's integrator loop; threads
 * that compute concurrently pass contexts of their own).
 * Copies positions/masses to the device and accelerations back every call.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_gravity_compute_acceleration_cuda(
    const NBodySimProParticleSystemView* view, const NBodySimProGravity* gravity, void* context,
    NBodySimProError* error);

/*
 * `barnes_hut_cuda` algorithm: GPU Barnes-Hut with the reference's opening
 * criterion (2h)^2 < theta^2 d^2 to the cell centre of mass
 * (src/c/barnes_hut/barnes_hut.c:596-599), replacing
 * n_body_sim_pro_barnes_hut_compute_acceleration (barnes_hut/barnes_hut.h:61-63).
 * `context` must be an NBodySimProCudaContext* (NULL: the process-wide one).
 * Empty system -> INVALID_ARGUMENT (barnes_hut.c:446-451).
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_barnes_hut_compute_acceleration_cuda(
    const NBodySimProParticleSystemView* view, const NBodySimProGravity* gravity, void* context,
    NBodySimProError* error);

/* ---- device-resident stepping ---------------------------------------------------- */

/*
 * Replaces n_body_sim_pro_preset_generate_parallel (generation/presets.h:73,
 * src/c/generation/presets_parallel.c) for device-resident systems: generates
 * the preset directly into the context's device state (no host arrays, no
 * upload), one thread per particle with the reference's per-particle
 * generators (xoshiro256** seeded from mix_seed(seed, index)), then removes
 * each block's mean velocity as the reference does.  Integer random streams
 * are identical to the reference's; the FP64 transcendental functions (log,
 * cos, sin, pow, cbrt) are CUDA's, so values agree to a few ulp.  Particles
 * the reference leaves unfilled (the last n % 2 of galaxy_collision, n % 3 of
 * triple_galaxy) are zero apart from the collision's approach velocity;
 * accelerations are zero.  Same argument errors as the reference (two_body
 * needs exactly 2 particles).
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_preset_generate_parallel(
    NBodySimProCudaContext* context, NBodySimProSimulationPreset preset,
    const NBodySimProPresetParameters* parameters, NBodySimProError* error);

/*
 * Joins the parallel presets (src/c/generation/presets_parallel.c): two Plummer
 * spheres of total mass 1/2 each and scale radius `scale_radius`, built the way
 * the reference's galaxy_collision builds its two disk blocks (:392-404) but
 * with its Plummer block (fill_plummer_block, :91-155): block b in
 * [b * (count/2), ...) draws from the per-particle generators
 * mix_seed(mix_seed(seed, b), index), is centred at -/+ separation/2 on x and
 * has its mean velocity removed; then -/+ relative_speed/2 is added on y.
 * Block 1 takes count - count/2 particles.  The two-Plummer collision
 * workload (two 500k or 5M spheres 10 apart, relative speed 0.3) is this with
 * (1, 10, 0.3).  Accelerations start at zero.  count < 2, a non-positive
 * radius or non-finite arguments -> INVALID_ARGUMENT.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_plummer_collision_generate(
    NBodySimProCudaContext* context, size_t count, uint64_t seed, double scale_radius,
    double separation, double relative_speed, NBodySimProError* error);

/*
 * Replaces n_body_sim_pro_checkpoint_write (checkpoint/checkpoint.h:43-46,
 * src/c/checkpoint/checkpoint.c:9-76) for device-resident state: the file is
 * the reference's format — magic, version, the header struct as stored in
 * memory, then x, y, z, vx, vy, vz, ax, ay, az, m as FP64 arrays — written
 * straight from the device through two pinned staging buffers, so the
 * device-to-host copy of one chunk overlaps the file write of the previous
 * one.  For the same state and header the bytes equal the reference's file.
 * Errors as the reference: NULL arguments or a header count different from the
 * resident count -> INVALID_ARGUMENT, file failures -> IO_ERROR; no resident
 * state -> INVALID_STATE.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_checkpoint_write(
    NBodySimProCudaContext* context, const char* path, const NBodySimProCheckpointHeader* header,
    NBodySimProError* error);

/*
 * Replaces n_body_sim_pro_checkpoint_read (checkpoint.h:51-54, checkpoint.c:131-206):
 * the file's state becomes the context's resident state (chunks read into
 * pinned buffers and copied to the device while the next chunk is read) and
 * `header` receives the stored header.  Bad magic or version -> INVALID_STATE,
 * short or unreadable files -> IO_ERROR.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_checkpoint_read(
    NBodySimProCudaContext* context, const char* path, NBodySimProCheckpointHeader* header,
    NBodySimProError* error);

/* Copy positions, velocities, masses and accelerations of `view` to the device. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_upload(
    NBodySimProCudaContext* context, const NBodySimProParticleSystemView* view,
    NBodySimProError* error);

/* Copy the device state back into `view` (same particle count as uploaded). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_download(
    NBodySimProCudaContext* context, const NBodySimProParticleSystemView* view,
    NBodySimProError* error);

/* Recompute the accelerations of the resident state (the "initial forces"
 * step the integrators require, physics/integrator.h:26-28). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_compute_acceleration(
    NBodySimProCudaContext* context, const NBodySimProGravity* gravity,
    NBodySimProCudaAlgorithm algorithm, NBodySimProError* error);

/*
 * `steps` timesteps of n_body_sim_pro_integrator_advance semantics
 * (physics/integrator.h:58-64, src/c/physics/integrator.c:141-172) on the
 * resident state, the force pass fused with the kick/drift epilogues.
 * Leapfrog / velocity Verlet need valid accelerations first (upload them or
 * call n_body_sim_pro_cuda_compute_acceleration).  timestep <= 0 -> INVALID_ARGUMENT.
 * Returns when the work is enqueued AND finished (it synchronises once).
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_advance(
    NBodySimProCudaContext* context, const NBodySimProGravity* gravity,
    NBodySimProIntegratorType integrator, double timestep, int steps,
    NBodySimProCudaAlgorithm algorithm, NBodySimProError* error);

/*
 * All-pairs sharded by targets, one process (and context) per GPU: the
 * context's resident state is this rank's slice of the particles.  One
 * leapfrog KDK step (integrator.c:47-85) is split around the all-gather of
 * the packed sources, which the caller runs (NCCL):
 *
 *   shard_begin  opening kick + drift of the slice (skipped for timestep 0),
 *                then the slice packed as float4 (x - c, y - c, z - c, m) into
 *                `slice` (device memory, slice_capacity entries, a multiple of
 *                8 and >= the resident count; the rest written massless).
 *                `centre` c must be the same on every rank.
 *   (caller)     all-gather every rank's slice, in rank order, into `sources`.
 *   shard_end    accelerations of the slice from the source_count packed
 *                sources (this rank's own slice at entry slice_offset, so the
 *                pair of a particle with itself adds 0), then the closing kick.
 *
 * timestep 0 in both calls only sets the accelerations (the forces before the
 * first step).  Both return when their work has finished.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_shard_begin(
    NBodySimProCudaContext* context, double timestep, const double centre[3], void* slice,
    size_t slice_capacity, NBodySimProError* error);

N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_shard_end(
    NBodySimProCudaContext* context, const NBodySimProGravity* gravity, double timestep,
    const void* sources, size_t source_count, size_t slice_offset, NBodySimProError* error);

/*
 * Conservation diagnostics of the resident state in FP64 on the device:
 * n_body_sim_pro_diagnostics_compute_global (src/c/diagnostics/numerics.c:5-81)
 * and, when `potential_energy` is non-NULL, the O(N^2) softened potential
 * energy (numerics.c:83-116).
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_diagnostics(
    NBodySimProCudaContext* context, const NBodySimProGravity* gravity,
    NBodySimProDiagnosticsQuantities* quantities, double* potential_energy,
    NBodySimProError* error);

/*
 * FP64 exact accelerations of `count` resident target particles (indices in
 * `targets`) over all resident sources, with the pair arithmetic of
 * src/c/physics/gravity.c:46-61: the precision-report oracle on the device.
 * out[3*t + c]; host pointers.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_reference_acceleration(
    NBodySimProCudaContext* context, const NBodySimProGravity* gravity, const int64_t* targets,
    size_t count, double* out, NBodySimProError* error);

/*
 * Morton order of the resident positions as the Barnes-Hut build computes it:
 * keys_sorted[i] and permutation[i] (original index) for sorted position i,
 * root[4] = centre xyz and half size.  Bit-exact with the reference's
 * morton_axis_code / morton_key / radix_sort_morton_keys
 * (src/c/barnes_hut/barnes_hut.c:286-339, :453-483).  Any argument may be NULL.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_morton_order(
    NBodySimProCudaContext* context, uint64_t* keys_sorted, uint64_t* permutation, double* root,
    NBodySimProError* error);

/* Wait for all work queued on the context's stream. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_synchronize(
    NBodySimProCudaContext* context, NBodySimProError* error);

/* Name of the library's GPU architecture target ("sm_100a"). */
N_BODY_SIM_PRO_CUDA_API const char* n_body_sim_pro_cuda_architecture(void);

/* ---- learned far-field correction ------------------------------------------------ */

/*
 * A small MLP (10 -> 64 -> 64 -> 3, GELU; BF16 tensor-core products with FP32
 * accumulation) predicting, for a cell accepted by the opening test, the
 * residual between the exact cell sum and the cell's monopole term, in units
 * of G M / |d|^2.  Inputs: the target offset from the cell's centre of mass
 * over the cell side (3), the opening ratio side / |d| (1), the trace-free
 * quadrupole over M side^2 (5) and sum m |x - com|^2 over M side^2 (1).  It is
 * trained on the GPU from (cell, target) pairs of a resident system with exact
 * cell sums.  In the walk it is evaluated once per accepted cell and group of
 * 32 targets, at the group's centre; cells whose inputs fall outside the range
 * seen in training keep the plain monopole.  The reference engine has no such
 * component (its Barnes-Hut is monopole-only, barnes_hut.c:600-612).
 */
typedef struct NBodySimProCudaCorrection NBodySimProCudaCorrection;

enum {
    N_BODY_SIM_PRO_CUDA_CORRECTION_PARAMETERS = 5059, /* W1[64][10] b1 W2[64][64] b2 W3[3][64] b3 */
    N_BODY_SIM_PRO_CUDA_CORRECTION_SCALING = 46       /* x mean, 1/std, min, max [10]; y mean, std [3] */
};

N_BODY_SIM_PRO_CUDA_API NBodySimProCudaCorrection* n_body_sim_pro_cuda_correction_create(
    uint64_t seed, NBodySimProError* error);
N_BODY_SIM_PRO_CUDA_API void n_body_sim_pro_cuda_correction_destroy(
    NBodySimProCudaCorrection* correction);

/* Sample `samples` (cell, target) pairs from the resident system of `context`
 * (cells accepted at `theta` by the reference criterion), label them with exact
 * cell sums, and standardise: the training set (last sixteenth: validation). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_generate(
    NBodySimProCudaCorrection* correction, NBodySimProCudaContext* context,
    const NBodySimProGravity* gravity, double theta, size_t samples, uint64_t seed,
    NBodySimProError* error);

/* Minibatch Adam on the GPU; per-epoch mean squared errors (standardised units). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_train(
    NBodySimProCudaCorrection* correction, int epochs, int batch, double learning_rate,
    double* train_loss, double* validation_loss, NBodySimProError* error);

/* FP32 parameters (N_BODY_SIM_PRO_CUDA_CORRECTION_PARAMETERS) and scaling table. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_get_parameters(
    NBodySimProCudaCorrection* correction, float* parameters, float* scaling,
    NBodySimProError* error);
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_set_parameters(
    NBodySimProCudaCorrection* correction, const float* parameters, const float* scaling,
    NBodySimProError* error);

/* Gradient of the mean squared error over `rows` (a multiple of 128)
 * standardised rows, from the tensor-core forward/backward kernels. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_gradient(
    NBodySimProCudaCorrection* correction, const float* features, const float* labels,
    size_t rows, float* gradient, double* loss, NBodySimProError* error);

/* Copy up to max_rows raw (feature, label) training rows; *rows = rows held. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_samples(
    NBodySimProCudaCorrection* correction, size_t* rows, float* features, float* labels,
    size_t max_rows, NBodySimProError* error);

/* Engines of n_body_sim_pro_cuda_correction_evaluate. */
typedef enum NBodySimProCudaMlpEngine {
    N_BODY_SIM_PRO_CUDA_MLP_TCGEN05 = 0,  /* 5th-generation tensor cores, 128-row tiles, TMEM */
    N_BODY_SIM_PRO_CUDA_MLP_MMA_SYNC = 1  /* warp-level mma.sync, 16-row tiles */
} NBodySimProCudaMlpEngine;

/* The trained network on `rows` raw feature rows (10 floats each, the
 * features of the corrected walk: cell-to-target offset / side, side /
 * distance, trace-free quadrupole / (M side^2), spread): standardised, through
 * the BF16 layers, de-standardised into `outputs` (3 floats per row: the
 * residual (a_exact - a_monopole) |d|^2 / M in units of G).  Host arrays.  No
 * range masking: rows outside the training range are evaluated as given.
 * No reference counterpart (the reference has no learned correction). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_correction_evaluate(
    NBodySimProCudaCorrection* correction, const float* features, size_t rows, float* outputs,
    int engine, NBodySimProError* error);

/* Correct the Barnes-Hut walk of `context` with `correction` (NULL: plain). */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_context_set_correction(
    NBodySimProCudaContext* context, const NBodySimProCudaCorrection* correction,
    NBodySimProError* error);

/* ---- ensembles of many small systems ------------------------------------------- */

/*
 * Many independent systems (each 1..4096 particles, its own softened all-pairs
 * gravity, leapfrog KDK: src/c/physics/gravity.c:37-67 and
 * src/c/physics/integrator.c:47-85 per system) advanced together.  The
 * reference has no ensemble driver: a user would loop
 * n_body_sim_pro_integrator_advance over the systems.
 */
typedef struct NBodySimProCudaEnsemble NBodySimProCudaEnsemble;

typedef struct NBodySimProCudaEnsembleInfo {
    size_t systems;
    size_t particles;
    int threads_per_block;      /* autotuned tile shape */
    int targets_per_thread;
    int grid;                   /* persistent CTAs (one resident wave) */
    int work_items;             /* system bundles, longest first */
    double last_advance_ms;     /* device time of the last advance */
    double autotune_ms[3];      /* measured candidates (2 steps each) */
} NBodySimProCudaEnsembleInfo;

N_BODY_SIM_PRO_CUDA_API NBodySimProCudaEnsemble* n_body_sim_pro_cuda_ensemble_create(
    NBodySimProError* error);
N_BODY_SIM_PRO_CUDA_API void n_body_sim_pro_cuda_ensemble_destroy(NBodySimProCudaEnsemble* e);

/* `view` holds the systems back to back: system k is [offsets[k], offsets[k+1]);
 * offsets has system_count + 1 entries, offsets[0] = 0, offsets[system_count] =
 * view->particle_count. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_ensemble_upload(
    NBodySimProCudaEnsemble* e, const NBodySimProParticleSystemView* view,
    const uint64_t* offsets, size_t system_count, NBodySimProError* error);

N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_ensemble_download(
    NBodySimProCudaEnsemble* e, const NBodySimProParticleSystemView* view,
    NBodySimProError* error);

/* Measure the candidate tile shapes on the uploaded ensemble (state restored
 * afterwards) and keep the fastest; advance calls it on first use. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_ensemble_autotune(
    NBodySimProCudaEnsemble* e, const NBodySimProGravity* gravity, double timestep,
    NBodySimProError* error);

/*
 * `steps` leapfrog steps of every system.  Each call first computes the forces
 * of the current positions (the integrators' precondition), then runs the
 * steps.  one_launch_per_system = 0: one persistent kernel captured in a CUDA
 * graph for the whole ensemble and all steps; 1: the per-system path (one
 * all-pairs launch sequence per system and step), the baseline.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_ensemble_advance(
    NBodySimProCudaEnsemble* e, const NBodySimProGravity* gravity, double timestep, int steps,
    int one_launch_per_system, NBodySimProError* error);

N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_ensemble_info(
    const NBodySimProCudaEnsemble* e, NBodySimProCudaEnsembleInfo* info, NBodySimProError* error);

/* ---- all-pairs without device allocation ---------------------------------------- */

/*
 * No counterpart in the reference engine.
 *
 * All-pairs accelerations (the `cuda` algorithm's arithmetic) for callers that
 * cannot allocate device memory: code running while a CUDA graph is being
 * captured, plugins whose host framework owns every device allocation, loops
 * that must not touch the allocator after start-up.  The caller passes DEVICE
 * pointers for the inputs (positions, masses) and outputs (accelerations, FP64
 * SoA) and, optionally, a cudaStream_t (NULL: the legacy default stream); the
 * work is only enqueued, nothing synchronises and nothing is allocated or freed.
 *
 * The working memory is one static device array of about 4.3 MiB that every
 * GPU loading this library holds until the process exits, so:
 *   - particle_count must be <= 16384 (else INVALID_ARGUMENT, no GPU work);
 *   - every call shares the array: calls whose GPU work overlaps (e.g. on two
 *     unordered streams) race and give wrong results;
 *   - the first call on each device looks up the array's address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 * Host pointers are rejected with INVALID_ARGUMENT.  Non-finite positions are
 * not reported (no device status is read back): they give non-finite output.
 */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_allpairs_acceleration_noalloc(
    const double* positions_x, const double* positions_y, const double* positions_z,
    const double* masses, double* accelerations_x, double* accelerations_y,
    double* accelerations_z, size_t particle_count, double gravitational_constant,
    double softening_length, void* stream, NBodySimProError* error);

/* Measured throughput of the current GPU: scalar FFMA and paired FFMA
 * (fma.f32x2) in TFLOP/s, MUFU reciprocal square roots per second, and the
 * nominal SM clock; the denominators of the FP32 roofline.  Any pointer may be NULL. */
N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_measure_fp32_peak(
    double* ffma_tflops, double* ffma2_tflops, double* rsqrt_per_second, double* sm_clock_mhz,
    NBodySimProError* error);

/* Number of CUDA kernels this process has launched through the library. */
N_BODY_SIM_PRO_CUDA_API unsigned long long n_body_sim_pro_cuda_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* N_BODY_SIM_PRO_CUDA_H */
