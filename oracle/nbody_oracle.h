/*
 * CPU oracle for the force-evaluation / time-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker.
 * The product (n_body_sim_pro_b200/) never links or calls it.
 *
 * Every function restates one algorithm of the reference engine
 * (richie-rich90454/n_body_sim_pro, C17) in plain C, cited file:line.
 * The restatement is pinned against the reference itself: tests compile the
 * reference's own sources into oracle/_ref/libnbody_ref.so (oracle/Makefile)
 * and require bit-identical outputs on the same seeds, plus the reference's
 * analytic known answers (tests/numerical/*.c, tests/regression/*.c).
 *
 * The particle view has the exact field order of the reference's
 * NBodySimProParticleSystemView (include/n_body_sim_pro/core/particle_system.h:38-50)
 * so one ctypes structure drives both libraries.
 */
#ifndef NBODY_ORACLE_H
#define NBODY_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleView {
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
} OracleView;

typedef struct OracleRng {
    uint64_t state[4];
} OracleRng;

/* xoshiro256** seeded by splitmix64 (src/c/generation/random.c:9-58). */
void oracle_rng_init(OracleRng* rng, uint64_t seed);
uint64_t oracle_rng_next_u64(OracleRng* rng);
double oracle_rng_next_double(OracleRng* rng);
double oracle_rng_next_gaussian(OracleRng* rng);
/* per-index seed mixer (src/c/generation/presets_parallel.c:36-41) */
uint64_t oracle_mix_seed(uint64_t master_seed, uint64_t index);

/* Presets (src/c/generation/presets.c).  Return 0 on success. */
int oracle_preset_two_body(OracleView* view);
int oracle_preset_random_cloud(OracleView* view, uint64_t seed);
int oracle_preset_globular_cluster(OracleView* view, uint64_t seed);
int oracle_preset_spiral_galaxy(OracleView* view, uint64_t seed);
/* Two Plummer spheres (a, M/2 each) at x = -/+ separation/2 moving -/+ speed/2 on y. */
int oracle_preset_plummer_collision(OracleView* view, uint64_t seed, double scale_radius,
                                    double separation, double relative_speed);
/* Uniform positions in [0,1)^3, masses 10^U(-3,0) normalised to 1, zero velocity. */
int oracle_preset_uniform_log_mass(OracleView* view, uint64_t seed);
/* src/c/generation/presets_parallel.c (n_body_sim_pro_preset_generate_parallel,
 * include/n_body_sim_pro/generation/presets.h:73): preset ids as the reference's
 * NBodySimProSimulationPreset enum (presets.h:27-38). 0 on success. */
int oracle_preset_parallel(OracleView* view, int preset, uint64_t seed);
/* Two Plummer spheres (mass 1/2 each) from the parallel presets' per-particle
 * streams, block b seeded with mix_seed(seed, b); -/+ separation/2 on x,
 * -/+ relative_speed/2 on y.  0 on success. */
int oracle_preset_plummer_collision_parallel(OracleView* view, uint64_t seed,
                                             double scale_radius, double separation,
                                             double relative_speed);
/* Size of ensemble member k: round(exp(U(ln lo, ln hi))) from rng(mix_seed(master, k)). */
size_t oracle_ensemble_member_size(uint64_t master_seed, uint64_t k, size_t lo, size_t hi);
/* Plummer sphere (a = 1, M = 1) for ensemble member k, same stream as the size draw. */
int oracle_ensemble_member_generate(OracleView* view, uint64_t master_seed, uint64_t k,
                                    size_t lo, size_t hi);

/* Scalar all-pairs reference (src/c/physics/gravity.c:15-70). */
void oracle_gravity_reference(const OracleView* view, double gravitational_constant,
                              double softening_length);
/* Same loop, OpenMP over targets (src/c/physics/gravity_openmp.c:30-86). */
void oracle_gravity_openmp(const OracleView* view, double gravitational_constant,
                           double softening_length);
/* Same loop restricted to `count` target indices; writes out[3*t + c]. */
void oracle_gravity_subset(const OracleView* view, double gravitational_constant,
                           double softening_length, const int64_t* targets, size_t count,
                           double* out);

/* Integrators (src/c/physics/integrator.c:15-172) with the all-pairs oracle or
 * the Barnes-Hut oracle as force function. integrator: 0 euler, 1 leapfrog,
 * 2 velocity verlet.  force: 0 all-pairs reference, 1 all-pairs OpenMP,
 * 2 Barnes-Hut (theta). Returns 0 on success. */
int oracle_integrator_advance(OracleView* view, double gravitational_constant,
                              double softening_length, int integrator, double timestep,
                              int force, double theta);

/* Diagnostics (src/c/diagnostics/numerics.c:5-116). q[11] = KE, M, P xyz, L xyz, COM xyz. */
void oracle_diagnostics_global(const OracleView* view, double* q);
double oracle_potential_energy(const OracleView* view, double gravitational_constant,
                               double softening_length);
double oracle_potential_energy_openmp(const OracleView* view, double gravitational_constant,
                                      double softening_length);

/* Morton order (src/c/barnes_hut/barnes_hut.c:286-339, :402-483).
 * keys_sorted[i], permutation[i] in sorted order; root = cx, cy, cz, half. */
int oracle_morton_order(const OracleView* view, uint64_t* keys_sorted, uint64_t* permutation,
                        double* root);

/* Barnes-Hut force (src/c/barnes_hut/barnes_hut.c:145-253, :442-704).
 * stats[6] = node_count, leaf_count, internal_node_count, accepted_approximations,
 * exact_interactions, maximum_depth.  threads <= 0: OpenMP default. */
int oracle_barnes_hut(const OracleView* view, double gravitational_constant,
                      double softening_length, double theta, uint64_t* stats);

/* Analysis of the walk above (no reference counterpart): for each target (input
 * index), the error of every accepted cell's monopole against the exact sum
 * over the cell's particles, summed into `bins` bins of (2h / d) / theta
 * (err[target][bin][3]), and the number of accepted cells per bin
 * (count[target][bin]).  The bins of a target sum to its Barnes-Hut force minus
 * the direct sum. */
int oracle_barnes_hut_residual_bands(const OracleView* view, double gravitational_constant,
                                     double softening_length, double theta,
                                     const int64_t* targets, size_t n_targets, int bins,
                                     double* err, uint64_t* count);

#ifdef __cplusplus
}
#endif

#endif
