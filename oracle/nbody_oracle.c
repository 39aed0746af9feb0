/*
 * CPU oracle — TEST INFRASTRUCTURE ONLY (see nbody_oracle.h).
 *
 * Plain-C restatement of the reference engine's force/time-step path.  Each
 * function cites the reference file:line whose arithmetic it follows.  The
 * order of floating-point operations (and of RNG draws) is kept identical to
 * the reference so outputs are bit-identical; tests/test_oracle.py pins that
 * against the reference compiled from its own sources (oracle/_ref) and
 * against committed golden fixtures (tests/golden/).
 *
 * Built with -ffp-contract=off: the reference's scalar files are compiled
 * without -mfma, so no multiply-add is ever fused there either.
 */
#include "nbody_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------- */
/* RNG: src/c/generation/random.c:9-58                                        */
/* ------------------------------------------------------------------------- */

static uint64_t splitmix_next(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t rotl64(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

void oracle_rng_init(OracleRng* rng, uint64_t seed) {
    uint64_t s = seed;
    for (int i = 0; i < 4; ++i) rng->state[i] = splitmix_next(&s);
}

uint64_t oracle_rng_next_u64(OracleRng* rng) {
    uint64_t* s = rng->state;
    const uint64_t out = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return out;
}

double oracle_rng_next_double(OracleRng* rng) {
    return (double)(oracle_rng_next_u64(rng) >> 11) * (1.0 / 9007199254740992.0);
}

static double rng_range(OracleRng* rng, double lo, double hi) {
    return lo + (hi - lo) * oracle_rng_next_double(rng);
}

double oracle_rng_next_gaussian(OracleRng* rng) {
    double u1 = 0.0;
    while (u1 == 0.0) u1 = oracle_rng_next_double(rng);
    const double u2 = oracle_rng_next_double(rng);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

uint64_t oracle_mix_seed(uint64_t master_seed, uint64_t index) {
    uint64_t x = master_seed ^ (index + 0x9E3779B97F4A7C15ull);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* ------------------------------------------------------------------------- */
/* Presets: src/c/generation/presets.c                                        */
/* ------------------------------------------------------------------------- */

static void put(OracleView* v, size_t i, double x, double y, double z, double vx, double vy,
                double vz, double m) {
    v->positions_x[i] = x;
    v->positions_y[i] = y;
    v->positions_z[i] = z;
    v->velocities_x[i] = vx;
    v->velocities_y[i] = vy;
    v->velocities_z[i] = vz;
    v->masses[i] = m;
}

/* presets.c:80-111 — zero the block's mean velocity (two passes). */
static void zero_block_momentum(OracleView* v, size_t first, size_t count) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (size_t i = 0; i < count; ++i) {
        sx += v->velocities_x[first + i];
        sy += v->velocities_y[first + i];
        sz += v->velocities_z[first + i];
    }
    sx /= (double)count;
    sy /= (double)count;
    sz /= (double)count;
    for (size_t i = 0; i < count; ++i) {
        v->velocities_x[first + i] -= sx;
        v->velocities_y[first + i] -= sy;
        v->velocities_z[first + i] -= sz;
    }
}

/* presets.c:113-127 — unit vector from three normalised Gaussians. */
static void unit_vector(OracleRng* rng, double* x, double* y, double* z) {
    for (;;) {
        const double a = oracle_rng_next_gaussian(rng);
        const double b = oracle_rng_next_gaussian(rng);
        const double c = oracle_rng_next_gaussian(rng);
        const double n = sqrt(a * a + b * b + c * c);
        if (n > 1.0e-12) {
            *x = a / n;
            *y = b / n;
            *z = c / n;
            return;
        }
    }
}

/* presets.c:170-202 (+ :144-154): Plummer sphere into [first, first+count). */
static void plummer_block(OracleView* v, OracleRng* rng, size_t first, size_t count,
                          double scale_radius, double total_mass, const double* centre) {
    const double mass = total_mass / (double)count;
    for (size_t i = 0; i < count; ++i) {
        const double u = 1.0 - oracle_rng_next_double(rng);
        const double r = scale_radius / sqrt(pow(u, -2.0 / 3.0) - 1.0);
        double dx, dy, dz;
        unit_vector(rng, &dx, &dy, &dz);
        double px = r * dx, py = r * dy, pz = r * dz;
        if (centre != NULL) {
            px += centre[0];
            py += centre[1];
            pz += centre[2];
        }
        const double sigma =
            sqrt(1.0 * total_mass / (6.0 * sqrt(scale_radius * scale_radius + r * r)));
        const double vx = oracle_rng_next_gaussian(rng) * sigma;
        const double vy = oracle_rng_next_gaussian(rng) * sigma;
        const double vz = oracle_rng_next_gaussian(rng) * sigma;
        put(v, first + i, px, py, pz, vx, vy, vz, mass);
    }
    zero_block_momentum(v, first, count);
}

int oracle_preset_two_body(OracleView* v) {
    if (v->particle_count != 2) return 1;
    const double s = sqrt(2.0) / 2.0;
    put(v, 0, -0.5, 0.0, 0.0, 0.0, s, 0.0, 1.0);
    put(v, 1, 0.5, 0.0, 0.0, 0.0, -s, 0.0, 1.0);
    return 0;
}

/* presets.c:272-288 with random_point_in_sphere :129-141. */
int oracle_preset_random_cloud(OracleView* v, uint64_t seed) {
    const size_t n = v->particle_count;
    if (n == 0) return 1;
    OracleRng rng;
    oracle_rng_init(&rng, seed);
    const double mass = 1.0 / (double)n;
    for (size_t i = 0; i < n; ++i) {
        const double r = 1.0 * cbrt(oracle_rng_next_double(&rng));
        double dx, dy, dz;
        unit_vector(&rng, &dx, &dy, &dz);
        const double vx = rng_range(&rng, -0.05, 0.05);
        const double vy = rng_range(&rng, -0.05, 0.05);
        const double vz = rng_range(&rng, -0.05, 0.05);
        put(v, i, r * dx, r * dy, r * dz, vx, vy, vz, mass);
    }
    zero_block_momentum(v, 0, n);
    return 0;
}

/* presets.c:437-440: globular cluster = Plummer(a = 1, M = 1) about the origin. */
int oracle_preset_globular_cluster(OracleView* v, uint64_t seed) {
    if (v->particle_count == 0) return 1;
    OracleRng rng;
    oracle_rng_init(&rng, seed);
    plummer_block(v, &rng, 0, v->particle_count, 1.0, 1.0, NULL);
    return 0;
}

/* presets.c:210-258 (disk) with the spiral parameters of :446-451. */
int oracle_preset_spiral_galaxy(OracleView* v, uint64_t seed) {
    const size_t n = v->particle_count;
    if (n == 0) return 1;
    OracleRng rng;
    oracle_rng_init(&rng, seed);
    const double a = 0.7, h = 0.1, vc = 1.0, sigma = 0.12, twist = 3.5;
    const int arms = 2;
    const double mass = 1.0 / (double)n;
    for (size_t i = 0; i < n; ++i) {
        const double e1 = -log(1.0 - oracle_rng_next_double(&rng));
        const double e2 = -log(1.0 - oracle_rng_next_double(&rng));
        const double r = a * (e1 + e2);
        double phi = 2.0 * M_PI * oracle_rng_next_double(&rng);
        const double arm = oracle_rng_next_double(&rng) * (double)arms;
        const double arm_phi = 2.0 * M_PI * arm / (double)arms + twist * r / a;
        phi = arm_phi + oracle_rng_next_gaussian(&rng) * 0.15;
        const double z = oracle_rng_next_gaussian(&rng) * h;
        const double c = cos(phi), s = sin(phi);
        const double vx = vc * -s + oracle_rng_next_gaussian(&rng) * sigma;
        const double vy = vc * c + oracle_rng_next_gaussian(&rng) * sigma;
        const double vz = oracle_rng_next_gaussian(&rng) * sigma * 0.5;
        put(v, i, r * c, r * s, z, vx, vy, vz, mass);
    }
    zero_block_momentum(v, 0, n);
    return 0;
}

/* Two Plummer spheres built with presets.c:170-202 semantics, one RNG stream:
 * block 0 centred at -separation/2, block 1 at +separation/2, each with zero
 * net momentum, then -/+ relative_speed/2 added on y. */
int oracle_preset_plummer_collision(OracleView* v, uint64_t seed, double scale_radius,
                                    double separation, double relative_speed) {
    const size_t n = v->particle_count;
    if (n < 2) return 1;
    const size_t half = n / 2;
    OracleRng rng;
    oracle_rng_init(&rng, seed);
    const double left[3] = {-0.5 * separation, 0.0, 0.0};
    const double right[3] = {0.5 * separation, 0.0, 0.0};
    plummer_block(v, &rng, 0, half, scale_radius, 0.5, left);
    plummer_block(v, &rng, half, n - half, scale_radius, 0.5, right);
    for (size_t i = 0; i < n; ++i) {
        v->velocities_y[i] += i < half ? -0.5 * relative_speed : 0.5 * relative_speed;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Parallel presets: src/c/generation/presets_parallel.c.  Every particle draws */
/* from its own generator seeded with mix_seed(master, index) (:36-41), so the */
/* result does not depend on how the particles are split across threads.      */
/* ------------------------------------------------------------------------- */

/* Subtract the mean velocity of [start, start+count) given its running sums. */
static void par_subtract_mean(OracleView* v, size_t start, size_t count, double sx, double sy,
                              double sz) {
    sx /= (double)count;
    sy /= (double)count;
    sz /= (double)count;
    for (size_t k = 0; k < count; ++k) {
        v->velocities_x[start + k] -= sx;
        v->velocities_y[start + k] -= sy;
        v->velocities_z[start + k] -= sz;
    }
}

/* presets_parallel.c:91-155 (Plummer block; centre added, :428-431). */
static void par_plummer_block(OracleView* v, uint64_t master, size_t start, size_t count,
                              double a, double a2, double total_mass, double particle_mass,
                              const double* centre) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (size_t k = 0; k < count; ++k) {
        const size_t i = start + k;
        OracleRng rng;
        oracle_rng_init(&rng, oracle_mix_seed(master, i));
        const double u = 1.0 - oracle_rng_next_double(&rng);
        const double r = a / sqrt(pow(u, -2.0 / 3.0) - 1.0);
        double dx, dy, dz;
        unit_vector(&rng, &dx, &dy, &dz);
        double px = r * dx, py = r * dy, pz = r * dz;
        if (centre != NULL) {
            px = px + centre[0];
            py = py + centre[1];
            pz = pz + centre[2];
        }
        const double sigma = sqrt(1.0 * total_mass / (6.0 * sqrt(a2 + r * r)));
        const double vx = oracle_rng_next_gaussian(&rng) * sigma;
        const double vy = oracle_rng_next_gaussian(&rng) * sigma;
        const double vz = oracle_rng_next_gaussian(&rng) * sigma;
        put(v, i, px, py, pz, vx, vy, vz, particle_mass);
        sx += vx;
        sy += vy;
        sz += vz;
    }
    par_subtract_mean(v, start, count, sx, sy, sz);
}

/* Two Plummer spheres in the parallel-preset form: the reference's
 * galaxy_collision layout (presets_parallel.c:392-404: block b seeded with
 * mix_seed(seed, b), filling [b*half, ...)) with its Plummer block
 * (fill_plummer_block, :91-155, mass 1/2, centred at -/+ separation/2 on x);
 * block 1 takes n - n/2 particles; then -/+ relative_speed/2 on y. */
int oracle_preset_plummer_collision_parallel(OracleView* v, uint64_t seed, double scale_radius,
                                             double separation, double relative_speed) {
    const size_t n = v->particle_count;
    if (n < 2) return 1;
    const size_t half = n / 2;
    for (int b = 0; b < 2; ++b) {
        const size_t start = (size_t)b * half;
        const size_t count = b == 0 ? half : n - half;
        const double centre[3] = {(b == 0 ? -0.5 : 0.5) * separation, 0.0, 0.0};
        par_plummer_block(v, oracle_mix_seed(seed, (uint64_t)b), start, count, scale_radius,
                          scale_radius * scale_radius, 0.5, 0.5 / (double)count, centre);
    }
    for (size_t i = 0; i < n; ++i)
        v->velocities_y[i] += i < half ? -0.5 * relative_speed : 0.5 * relative_speed;
    return 0;
}

/* presets_parallel.c:158-217 (exponential disk block, optional arms). */
static void par_disk_block(OracleView* v, uint64_t master, size_t start, size_t count, double a,
                           double h, double vc, double sigma, double twist, int arms,
                           double particle_mass) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (size_t k = 0; k < count; ++k) {
        const size_t i = start + k;
        OracleRng rng;
        oracle_rng_init(&rng, oracle_mix_seed(master, i));
        const double e1 = -log(1.0 - oracle_rng_next_double(&rng));
        const double e2 = -log(1.0 - oracle_rng_next_double(&rng));
        const double r = a * (e1 + e2);
        double phi = 2.0 * M_PI * oracle_rng_next_double(&rng);
        if (twist > 0.0 && arms > 0) {
            const double arm = oracle_rng_next_double(&rng) * (double)arms;
            const double arm_phi = 2.0 * M_PI * arm / (double)arms + twist * r / a;
            phi = arm_phi + oracle_rng_next_gaussian(&rng) * 0.15;
        }
        const double z = oracle_rng_next_gaussian(&rng) * h;
        const double tx = -sin(phi), ty = cos(phi);
        const double px = r * cos(phi), py = r * sin(phi);
        const double vx = vc * tx + oracle_rng_next_gaussian(&rng) * sigma;
        const double vy = vc * ty + oracle_rng_next_gaussian(&rng) * sigma;
        const double vz = oracle_rng_next_gaussian(&rng) * sigma * 0.5;
        put(v, i, px, py, z, vx, vy, vz, particle_mass);
        sx += vx;
        sy += vy;
        sz += vz;
    }
    par_subtract_mean(v, start, count, sx, sy, sz);
}

int oracle_preset_parallel(OracleView* v, int preset, uint64_t seed) {
    const size_t n = v->particle_count;
    switch (preset) {
        case 0: /* two body, :43-57 */
            return oracle_preset_two_body(v);
        case 1: { /* random cloud, :219-272 */
            if (n == 0) return 1;
            const double mass = 1.0 / (double)n;
            double sx = 0.0, sy = 0.0, sz = 0.0;
            for (size_t i = 0; i < n; ++i) {
                OracleRng rng;
                oracle_rng_init(&rng, oracle_mix_seed(seed, i));
                double dx, dy, dz;
                unit_vector(&rng, &dx, &dy, &dz);
                const double r = cbrt(oracle_rng_next_double(&rng));
                const double vx = rng_range(&rng, -0.05, 0.05);
                const double vy = rng_range(&rng, -0.05, 0.05);
                const double vz = rng_range(&rng, -0.05, 0.05);
                put(v, i, r * dx, r * dy, r * dz, vx, vy, vz, mass);
                sx += vx;
                sy += vy;
                sz += vz;
            }
            par_subtract_mean(v, 0, n, sx, sy, sz);
            return 0;
        }
        case 2: { /* solar system, :59-89: one sequential stream seeded with `seed` */
            if (n == 0) return 1;
            OracleRng rng;
            oracle_rng_init(&rng, seed);
            put(v, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0);
            const size_t planets = n - 1;
            for (size_t k = 0; k < planets; ++k) {
                const double r = 1.0 + 3.0 * (double)k / (double)planets;
                const double speed = sqrt(1 / r);
                const double phi = 2.0 * M_PI * oracle_rng_next_double(&rng);
                put(v, k + 1, r * cos(phi), r * sin(phi), 0.0, -speed * sin(phi),
                    speed * cos(phi), 0.0, 0.001);
            }
            return 0;
        }
        case 3: { /* open cluster, :274-311 */
            if (n == 0) return 1;
            const double mass = 1.0 / (double)n;
            double sx = 0.0, sy = 0.0, sz = 0.0;
            for (size_t i = 0; i < n; ++i) {
                OracleRng rng;
                oracle_rng_init(&rng, oracle_mix_seed(seed, i));
                const double px = oracle_rng_next_gaussian(&rng) * 0.3;
                const double py = oracle_rng_next_gaussian(&rng) * 0.3;
                const double pz = oracle_rng_next_gaussian(&rng) * 0.3;
                const double vx = oracle_rng_next_gaussian(&rng) * 0.02;
                const double vy = oracle_rng_next_gaussian(&rng) * 0.02;
                const double vz = oracle_rng_next_gaussian(&rng) * 0.02;
                put(v, i, px, py, pz, vx, vy, vz, mass);
                sx += vx;
                sy += vy;
                sz += vz;
            }
            par_subtract_mean(v, 0, n, sx, sy, sz);
            return 0;
        }
        case 4: /* globular cluster, :372-376 */
        case 6: /* elliptical galaxy */
            if (n == 0) return 1;
            if (preset == 4) {
                par_plummer_block(v, seed, 0, n, 1.0, 1.0 * 1.0, 1.0, 1.0 / (double)n, NULL);
            } else {
                par_plummer_block(v, seed, 0, n, 2.0, 2.0 * 2.0, 1.0, 1.0 / (double)n, NULL);
            }
            return 0;
        case 5: /* spiral galaxy, :378-383 */
            if (n == 0) return 1;
            par_disk_block(v, seed, 0, n, 0.7, 0.1, 1.0, 0.12, 3.5, 2, 1.0 / (double)n);
            return 0;
        case 7: { /* galaxy collision, :384-396: particles past 2 * (n / 2) are left as they are */
            const size_t half = n / 2;
            if (half == 0) return 1;
            const double mass = 0.5 / (double)half;
            par_disk_block(v, oracle_mix_seed(seed, 0), 0, half, 0.7, 0.1, 1.0, 0.12, 0.0, 0, mass);
            par_disk_block(v, oracle_mix_seed(seed, 1), half, half, 0.7, 0.1, 1.0, 0.12, 0.0, 0,
                           mass);
            for (size_t i = 0; i < n; ++i) v->velocities_x[i] += i < half ? 0.35 : -0.35;
            return 0;
        }
        case 8: { /* triple galaxy, :397-471: particles past 3 * (n / 3) are left as they are */
            const size_t third = n / 3;
            if (third == 0) return 1;
            const double centres[3][3] = {{-1.8, 0.0, 0.0}, {1.8, 0.0, 0.0}, {0.0, 1.8, 0.0}};
            for (int g = 0; g < 3; ++g) {
                /* a = 0.7 with the literal 0.49 in the dispersion (:446), galaxy mass 1/3 */
                par_plummer_block(v, oracle_mix_seed(seed, (uint64_t)g), (size_t)g * third, third,
                                  0.7, 0.49, 1.0 / 3.0, (1.0 / 3.0) / (double)third, centres[g]);
            }
            return 0;
        }
        default:
            return 1;
    }
}

int oracle_preset_uniform_log_mass(OracleView* v, uint64_t seed) {
    const size_t n = v->particle_count;
    if (n == 0) return 1;
    OracleRng rng;
    oracle_rng_init(&rng, seed);
    double total = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double x = oracle_rng_next_double(&rng);
        const double y = oracle_rng_next_double(&rng);
        const double z = oracle_rng_next_double(&rng);
        const double m = pow(10.0, -3.0 + 3.0 * oracle_rng_next_double(&rng));
        put(v, i, x, y, z, 0.0, 0.0, 0.0, m);
        total += m;
    }
    for (size_t i = 0; i < n; ++i) v->masses[i] /= total;
    return 0;
}

size_t oracle_ensemble_member_size(uint64_t master_seed, uint64_t k, size_t lo, size_t hi) {
    OracleRng rng;
    oracle_rng_init(&rng, oracle_mix_seed(master_seed, k));
    const double u = oracle_rng_next_double(&rng);
    const double l = log((double)lo) + (log((double)hi) - log((double)lo)) * u;
    double s = floor(exp(l) + 0.5);
    if (s < (double)lo) s = (double)lo;
    if (s > (double)hi) s = (double)hi;
    return (size_t)s;
}

int oracle_ensemble_member_generate(OracleView* v, uint64_t master_seed, uint64_t k, size_t lo,
                                    size_t hi) {
    OracleRng rng;
    oracle_rng_init(&rng, oracle_mix_seed(master_seed, k));
    (void)oracle_rng_next_double(&rng); /* the size draw */
    const size_t n = oracle_ensemble_member_size(master_seed, k, lo, hi);
    if (v->particle_count != n) return 1;
    plummer_block(v, &rng, 0, n, 1.0, 1.0, NULL);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* All-pairs: src/c/physics/gravity.c:15-70, gravity_openmp.c:30-86           */
/* ------------------------------------------------------------------------- */

static void direct_sum_one(const OracleView* v, double G, double eps2, size_t i, double* out) {
    const size_t n = v->particle_count;
    const double* x = v->positions_x;
    const double* y = v->positions_y;
    const double* z = v->positions_z;
    const double* m = v->masses;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (size_t j = 0; j < n; ++j) {
        if (j == i) continue;
        const double dx = x[j] - x[i];
        const double dy = y[j] - y[i];
        const double dz = z[j] - z[i];
        const double r2 = dx * dx + dy * dy + dz * dz + eps2;
        const double inv = 1.0 / sqrt(r2);
        const double inv3 = inv * inv * inv;
        const double s = G * m[j] * inv3;
        ax += s * dx;
        ay += s * dy;
        az += s * dz;
    }
    out[0] = ax;
    out[1] = ay;
    out[2] = az;
}

void oracle_gravity_reference(const OracleView* v, double G, double eps) {
    const double eps2 = eps * eps; /* gravity.c:12 */
    for (size_t i = 0; i < v->particle_count; ++i) {
        double a[3];
        direct_sum_one(v, G, eps2, i, a);
        v->accelerations_x[i] = a[0];
        v->accelerations_y[i] = a[1];
        v->accelerations_z[i] = a[2];
    }
}

void oracle_gravity_openmp(const OracleView* v, double G, double eps) {
    const double eps2 = eps * eps;
    const long long n = (long long)v->particle_count;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
        double a[3];
        direct_sum_one(v, G, eps2, (size_t)i, a);
        v->accelerations_x[i] = a[0];
        v->accelerations_y[i] = a[1];
        v->accelerations_z[i] = a[2];
    }
}

void oracle_gravity_subset(const OracleView* v, double G, double eps, const int64_t* targets,
                           size_t count, double* out) {
    const double eps2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 16)
    for (long long t = 0; t < (long long)count; ++t) {
        direct_sum_one(v, G, eps2, (size_t)targets[t], out + 3 * t);
    }
}

/* ------------------------------------------------------------------------- */
/* Diagnostics: src/c/diagnostics/numerics.c:5-116                            */
/* ------------------------------------------------------------------------- */

void oracle_diagnostics_global(const OracleView* v, double* q) {
    double ke = 0.0, mt = 0.0, p[3] = {0, 0, 0}, l[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    for (size_t i = 0; i < v->particle_count; ++i) {
        const double m = v->masses[i];
        const double vx = v->velocities_x[i], vy = v->velocities_y[i], vz = v->velocities_z[i];
        ke += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        mt += m;
        p[0] += m * vx;
        p[1] += m * vy;
        p[2] += m * vz;
        const double x = v->positions_x[i], y = v->positions_y[i], z = v->positions_z[i];
        l[0] += m * (y * vz - z * vy);
        l[1] += m * (z * vx - x * vz);
        l[2] += m * (x * vy - y * vx);
        c[0] += m * x;
        c[1] += m * y;
        c[2] += m * z;
    }
    q[0] = ke;
    q[1] = mt;
    for (int k = 0; k < 3; ++k) {
        q[2 + k] = p[k];
        q[5 + k] = l[k];
        q[8 + k] = mt != 0.0 ? c[k] / mt : 0.0;
    }
}

double oracle_potential_energy(const OracleView* v, double G, double eps) {
    const double eps2 = eps * eps;
    const size_t n = v->particle_count;
    double sum = 0.0;
    for (size_t i = 0; i < n; ++i) {
        for (size_t j = i + 1; j < n; ++j) {
            const double dx = v->positions_x[j] - v->positions_x[i];
            const double dy = v->positions_y[j] - v->positions_y[i];
            const double dz = v->positions_z[j] - v->positions_z[i];
            const double d = sqrt(dx * dx + dy * dy + dz * dz + eps2);
            sum += v->masses[i] * v->masses[j] / d;
        }
    }
    return -G * sum;
}

/* Same pair terms; per-row partial sums added in row order (deterministic, but
 * rounded differently from the single running sum of numerics.c:101-112). */
double oracle_potential_energy_openmp(const OracleView* v, double G, double eps) {
    const double eps2 = eps * eps;
    const long long n = (long long)v->particle_count;
    double* rows = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    if (rows == NULL) return NAN;
#pragma omp parallel for schedule(dynamic, 64)
    for (long long i = 0; i < n; ++i) {
        double s = 0.0;
        for (long long j = i + 1; j < n; ++j) {
            const double dx = v->positions_x[j] - v->positions_x[i];
            const double dy = v->positions_y[j] - v->positions_y[i];
            const double dz = v->positions_z[j] - v->positions_z[i];
            const double d = sqrt(dx * dx + dy * dy + dz * dz + eps2);
            s += v->masses[i] * v->masses[j] / d;
        }
        rows[i] = s;
    }
    double sum = 0.0;
    for (long long i = 0; i < n; ++i) sum += rows[i];
    free(rows);
    return -G * sum;
}

/* ------------------------------------------------------------------------- */
/* Morton order: src/c/barnes_hut/barnes_hut.c:286-339, :402-483              */
/* ------------------------------------------------------------------------- */

static void root_cube(const OracleView* v, double* root) {
    const size_t n = v->particle_count;
    double lo[3] = {v->positions_x[0], v->positions_y[0], v->positions_z[0]};
    double hi[3] = {lo[0], lo[1], lo[2]};
    for (size_t i = 1; i < n; ++i) {
        const double p[3] = {v->positions_x[i], v->positions_y[i], v->positions_z[i]};
        for (int k = 0; k < 3; ++k) {
            if (p[k] < lo[k]) lo[k] = p[k];
            if (p[k] > hi[k]) hi[k] = p[k];
        }
    }
    double half = 0.5 * (hi[0] - lo[0]);
    for (int k = 1; k < 3; ++k) {
        const double e = 0.5 * (hi[k] - lo[k]);
        if (e > half) half = e;
    }
    if (half == 0.0) half = 0.5;
    half *= 1.0 + 1.0e-9;
    for (int k = 0; k < 3; ++k) root[k] = 0.5 * (lo[k] + hi[k]);
    root[3] = half;
}

static uint64_t axis_code(double value, double centre, double half) {
    double t = (value - centre) / (2.0 * half) + 0.5;
    if (t < 0.0) {
        t = 0.0;
    } else if (t >= 1.0) {
        t = 1.0 - 1.0e-15;
    }
    return (uint64_t)(t * 2097152.0);
}

static uint64_t interleave3(uint64_t x, uint64_t y, uint64_t z) {
    uint64_t key = 0;
    for (int b = 0; b < 21; ++b) {
        key |= ((x >> b) & 1ull) << (3 * b);
        key |= ((y >> b) & 1ull) << (3 * b + 1);
        key |= ((z >> b) & 1ull) << (3 * b + 2);
    }
    return key;
}

/* Stable LSD sort of `perm` (identity on entry) by keys[perm[i]], three
 * 21-bit digits, as barnes_hut.c:312-339. */
static int lsd_sort(const uint64_t* keys, size_t n, size_t* perm) {
    const size_t buckets = (size_t)1 << 21;
    size_t* count = (size_t*)malloc(buckets * sizeof(size_t));
    size_t* tmp = (size_t*)malloc((n ? n : 1) * sizeof(size_t));
    if (count == NULL || tmp == NULL) {
        free(count);
        free(tmp);
        return 1;
    }
    size_t* src = perm;
    size_t* dst = tmp;
    for (int pass = 0; pass < 3; ++pass) {
        const unsigned shift = 21u * (unsigned)pass;
        memset(count, 0, buckets * sizeof(size_t));
        for (size_t i = 0; i < n; ++i) ++count[(keys[src[i]] >> shift) & (buckets - 1)];
        size_t run = 0;
        for (size_t d = 0; d < buckets; ++d) {
            const size_t c = count[d];
            count[d] = run;
            run += c;
        }
        for (size_t i = 0; i < n; ++i) dst[count[(keys[src[i]] >> shift) & (buckets - 1)]++] = src[i];
        size_t* t = src;
        src = dst;
        dst = t;
    }
    /* three passes: the result sits in tmp */
    memcpy(perm, src, n * sizeof(size_t));
    free(count);
    free(tmp);
    return 0;
}

static int morton_sorted(const OracleView* v, double* root, uint64_t** keys_out,
                         size_t** perm_out) {
    const size_t n = v->particle_count;
    root_cube(v, root);
    uint64_t* keys = (uint64_t*)malloc(n * sizeof(uint64_t));
    size_t* perm = (size_t*)malloc(n * sizeof(size_t));
    if (keys == NULL || perm == NULL) {
        free(keys);
        free(perm);
        return 1;
    }
    for (size_t i = 0; i < n; ++i) {
        perm[i] = i;
        keys[i] = interleave3(axis_code(v->positions_x[i], root[0], root[3]),
                              axis_code(v->positions_y[i], root[1], root[3]),
                              axis_code(v->positions_z[i], root[2], root[3]));
    }
    if (lsd_sort(keys, n, perm)) {
        free(keys);
        free(perm);
        return 1;
    }
    *keys_out = keys;
    *perm_out = perm;
    return 0;
}

int oracle_morton_order(const OracleView* v, uint64_t* keys_sorted, uint64_t* permutation,
                        double* root) {
    if (v->particle_count == 0) return 1;
    uint64_t* keys;
    size_t* perm;
    if (morton_sorted(v, root, &keys, &perm)) return 1;
    for (size_t i = 0; i < v->particle_count; ++i) {
        permutation[i] = (uint64_t)perm[i];
        keys_sorted[i] = keys[perm[i]];
    }
    free(keys);
    free(perm);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Barnes-Hut: src/c/barnes_hut/barnes_hut.c:115-253, :442-704                 */
/* ------------------------------------------------------------------------- */

typedef struct ONode {
    int32_t child[8];
    int32_t particle; /* -1: internal or empty */
    int32_t count;
    double cx, cy, cz, mass;
} ONode;

typedef struct OTree {
    ONode* nodes;
    size_t used;
    size_t cap;
    const double *x, *y, *z, *m; /* Morton-ordered copies */
} OTree;

static size_t new_node(OTree* t) {
    ONode* n = &t->nodes[t->used];
    for (int c = 0; c < 8; ++c) n->child[c] = -1;
    n->particle = -1;
    n->count = 0;
    n->cx = n->cy = n->cz = n->mass = 0.0;
    return t->used++;
}

static void make_leaf(OTree* t, size_t node, size_t p) {
    ONode* n = &t->nodes[node];
    n->particle = (int32_t)p;
    n->count = 1;
    n->mass = t->m[p];
    n->cx = t->x[p];
    n->cy = t->y[p];
    n->cz = t->z[p];
}

static int octant(const OTree* t, size_t p, double cx, double cy, double cz) {
    return (t->x[p] > cx ? 1 : 0) | (t->y[p] > cy ? 2 : 0) | (t->z[p] > cz ? 4 : 0);
}

/* barnes_hut.c:145-212: insertion with depth bound 128 -> OVERFLOW (returns 6). */
static int insert(OTree* t, size_t node, size_t p, double cx, double cy, double cz, double h,
                  int depth) {
    for (;;) {
        if (depth > 128) return 6;
        if (t->nodes[node].particle != -1) {
            const size_t old = (size_t)t->nodes[node].particle;
            const int o = octant(t, old, cx, cy, cz);
            if (t->used + 1 > t->cap) return 2;
            t->nodes[node].particle = -1;
            const size_t c = new_node(t);
            t->nodes[node].child[o] = (int32_t)c;
            make_leaf(t, c, old);
        }
        const int o = octant(t, p, cx, cy, cz);
        const int32_t c = t->nodes[node].child[o];
        if (c == -1) {
            if (t->used + 1 > t->cap) return 2;
            const size_t fresh = new_node(t);
            t->nodes[node].child[o] = (int32_t)fresh;
            make_leaf(t, fresh, p);
            return 0;
        }
        const double q = h * 0.5;
        cx = cx + ((o & 1) ? h * 0.5 : -h * 0.5);
        cy = cy + ((o & 2) ? h * 0.5 : -h * 0.5);
        cz = cz + ((o & 4) ? h * 0.5 : -h * 0.5);
        h = q;
        node = (size_t)c;
        ++depth;
    }
}

/* barnes_hut.c:214-253 */
static void centres_of_mass(OTree* t) {
    for (size_t k = t->used; k > 0; --k) {
        ONode* n = &t->nodes[k - 1];
        if (n->particle != -1 || n->count == 0) continue;
        double m = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
        int cnt = 0;
        for (int c = 0; c < 8; ++c) {
            if (n->child[c] == -1) continue;
            const ONode* ch = &t->nodes[n->child[c]];
            if (ch->count == 0) continue;
            m += ch->mass;
            sx += ch->mass * ch->cx;
            sy += ch->mass * ch->cy;
            sz += ch->mass * ch->cz;
            cnt += ch->count;
        }
        n->mass = m;
        n->count = cnt;
        if (m != 0.0) {
            n->cx = sx / m;
            n->cy = sy / m;
            n->cz = sz / m;
        }
    }
}

static size_t depth_of(const OTree* t, size_t node) {
    size_t best = 0;
    for (int c = 0; c < 8; ++c) {
        const int32_t ch = t->nodes[node].child[c];
        if (ch == -1) continue;
        const size_t d = depth_of(t, (size_t)ch);
        if (d > best) best = d;
    }
    return best + 1;
}

typedef struct OEntry {
    int32_t node;
    double cx, cy, cz, h;
} OEntry;

/* barnes_hut.c:549-636: explicit stack of 1024 entries; children pushed 0..7. */
static void walk(const OTree* t, const double* root, double G, double eps2, double theta,
                 size_t q, double* a, uint64_t* approx, uint64_t* exact) {
    OEntry stack[1024];
    int top = 1;
    stack[0].node = 0;
    stack[0].cx = root[0];
    stack[0].cy = root[1];
    stack[0].cz = root[2];
    stack[0].h = root[3];
    const double qx = t->x[q], qy = t->y[q], qz = t->z[q];
    const double th2 = theta * theta;
    while (top > 0) {
        const OEntry e = stack[--top];
        const ONode* n = &t->nodes[e.node];
        if (n->count == 0) continue;
        if (n->particle != -1) {
            if ((size_t)n->particle != q) {
                const size_t j = (size_t)n->particle;
                const double dx = t->x[j] - qx;
                const double dy = t->y[j] - qy;
                const double dz = t->z[j] - qz;
                const double r2 = dx * dx + dy * dy + dz * dz + eps2;
                const double inv3 = 1.0 / (r2 * sqrt(r2));
                const double s = G * t->m[j] * inv3;
                a[0] += s * dx;
                a[1] += s * dy;
                a[2] += s * dz;
                ++*exact;
            }
            continue;
        }
        const double dx = n->cx - qx;
        const double dy = n->cy - qy;
        const double dz = n->cz - qz;
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double size2 = 4.0 * e.h * e.h;
        if (d2 > 0.0 && size2 < th2 * d2) {
            const double r2 = d2 + eps2;
            const double inv3 = 1.0 / (r2 * sqrt(r2));
            const double s = G * n->mass * inv3;
            a[0] += s * dx;
            a[1] += s * dy;
            a[2] += s * dz;
            ++*approx;
            continue;
        }
        const double hh = 0.5 * e.h;
        const double off = e.h * 0.5;
        for (int c = 0; c < 8; ++c) {
            const int32_t ch = n->child[c];
            if (ch == -1) continue;
            if (top >= 1024) break;
            stack[top].node = ch;
            stack[top].cx = e.cx + ((c & 1) ? off : -off);
            stack[top].cy = e.cy + ((c & 2) ? off : -off);
            stack[top].cz = e.cz + ((c & 4) ? off : -off);
            stack[top].h = hh;
            ++top;
        }
    }
}

/* The reference's tree over the Morton-ordered particles (barnes_hut.c:145-253):
 * buf holds x, y, z, m and three acceleration rows in Morton order, perm the
 * input index of each Morton slot.  0 on success; the arrays are the caller's. */
static int build_tree(const OracleView* v, OTree* t, double* root, double** buf_out,
                      size_t** perm_out) {
    const size_t n = v->particle_count;
    uint64_t* keys;
    size_t* perm;
    if (morton_sorted(v, root, &keys, &perm)) return 2;
    free(keys);
    double* buf = (double*)malloc(7 * n * sizeof(double));
    t->cap = 2 * n - 1;
    t->nodes = (ONode*)malloc(t->cap * sizeof(ONode));
    if (buf == NULL || t->nodes == NULL) {
        free(buf);
        free(t->nodes);
        free(perm);
        return 2;
    }
    double *x = buf, *y = buf + n, *z = buf + 2 * n, *m = buf + 3 * n;
    for (size_t i = 0; i < n; ++i) {
        x[i] = v->positions_x[perm[i]];
        y[i] = v->positions_y[perm[i]];
        z[i] = v->positions_z[perm[i]];
        m[i] = v->masses[perm[i]];
    }
    t->x = x;
    t->y = y;
    t->z = z;
    t->m = m;
    t->used = 0;
    new_node(t);
    int status = 0;
    for (size_t i = 0; i < n && status == 0; ++i) {
        if (t->nodes[0].count == 0) {
            make_leaf(t, 0, i);
            continue;
        }
        status = insert(t, 0, i, root[0], root[1], root[2], root[3], 0);
    }
    if (status != 0) {
        free(buf);
        free(t->nodes);
        free(perm);
        return status;
    }
    centres_of_mass(t);
    *buf_out = buf;
    *perm_out = perm;
    return 0;
}

int oracle_barnes_hut(const OracleView* v, double G, double eps, double theta, uint64_t* stats) {
    const size_t n = v->particle_count;
    if (n == 0) return 1;
    double root[4];
    double* buf;
    size_t* perm;
    OTree t;
    const int status = build_tree(v, &t, root, &buf, &perm);
    if (status != 0) return status;
    double *ax = buf + 4 * n, *ay = buf + 5 * n, *az = buf + 6 * n;
    uint64_t leaves = 0, internal = 0;
    for (size_t k = 0; k < t.used; ++k) {
        if (t.nodes[k].particle != -1) {
            ++leaves;
        } else if (t.nodes[k].count > 0) {
            ++internal;
        }
    }
    const double eps2 = eps * eps;
    uint64_t approx_total = 0, exact_total = 0;
#pragma omp parallel for schedule(static) reduction(+ : approx_total, exact_total)
    for (long long i = 0; i < (long long)n; ++i) {
        double a[3] = {0.0, 0.0, 0.0};
        uint64_t ap = 0, ex = 0;
        walk(&t, root, G, eps2, theta, (size_t)i, a, &ap, &ex);
        ax[i] = a[0];
        ay[i] = a[1];
        az[i] = a[2];
        approx_total += ap;
        exact_total += ex;
    }
    for (size_t i = 0; i < n; ++i) {
        v->accelerations_x[perm[i]] = ax[i];
        v->accelerations_y[perm[i]] = ay[i];
        v->accelerations_z[perm[i]] = az[i];
    }
    if (stats != NULL) {
        stats[0] = t.used;
        stats[1] = leaves;
        stats[2] = internal;
        stats[3] = approx_total;
        stats[4] = exact_total;
        stats[5] = depth_of(&t, 0);
    }
    free(buf);
    free(t.nodes);
    free(perm);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Analysis, no reference counterpart: the monopole error of the walk above,  */
/* split by how wide each accepted cell looks from the target                 */
/* ------------------------------------------------------------------------- */

/* The walk of barnes_hut.c:549-636 for one target; at every accepted cell (side
 * 2h, distance d to its centre of mass) the cell's error -- its monopole term
 * minus the exact softened sum over its particles (the target itself left
 * out, as in the direct sum) -- is added to the bin of (2h / d) / theta, and the
 * bin's cell count is raised.  Leaves are exact and add nothing, so the bins
 * sum to the walk's force minus the direct sum. */
static void residual_walk(const OTree* t, const int32_t* lo, const int32_t* hi, const double* root,
                          double G, double eps2, double theta, size_t q, int bins, double* err,
                          uint64_t* count) {
    OEntry stack[1024];
    int top = 1;
    stack[0].node = 0;
    stack[0].cx = root[0];
    stack[0].cy = root[1];
    stack[0].cz = root[2];
    stack[0].h = root[3];
    const double qx = t->x[q], qy = t->y[q], qz = t->z[q];
    const double th2 = theta * theta;
    while (top > 0) {
        const OEntry e = stack[--top];
        const ONode* n = &t->nodes[e.node];
        if (n->count == 0 || n->particle != -1) continue;
        const double dx = n->cx - qx;
        const double dy = n->cy - qy;
        const double dz = n->cz - qz;
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double size2 = 4.0 * e.h * e.h;
        if (d2 > 0.0 && size2 < th2 * d2) {
            const double r2 = d2 + eps2;
            const double s = G * n->mass / (r2 * sqrt(r2));
            double ex = 0.0, ey = 0.0, ez = 0.0;
            for (int32_t j = lo[e.node]; j <= hi[e.node]; ++j) {
                if ((size_t)j == q) continue;
                const double jx = t->x[j] - qx, jy = t->y[j] - qy, jz = t->z[j] - qz;
                const double rj2 = jx * jx + jy * jy + jz * jz + eps2;
                const double sj = G * t->m[j] / (rj2 * sqrt(rj2));
                ex += sj * jx;
                ey += sj * jy;
                ez += sj * jz;
            }
            int b = (int)(sqrt(size2 / d2) / theta * bins);
            b = b < 0 ? 0 : b >= bins ? bins - 1 : b;
            err[3 * b + 0] += s * dx - ex;
            err[3 * b + 1] += s * dy - ey;
            err[3 * b + 2] += s * dz - ez;
            ++count[b];
            continue;
        }
        const double hh = 0.5 * e.h;
        const double off = e.h * 0.5;
        for (int c = 0; c < 8; ++c) {
            const int32_t ch = n->child[c];
            if (ch == -1) continue;
            if (top >= 1024) break;
            stack[top].node = ch;
            stack[top].cx = e.cx + ((c & 1) ? off : -off);
            stack[top].cy = e.cy + ((c & 2) ? off : -off);
            stack[top].cz = e.cz + ((c & 4) ? off : -off);
            stack[top].h = hh;
            ++top;
        }
    }
}

int oracle_barnes_hut_residual_bands(const OracleView* v, double G, double eps, double theta,
                                     const int64_t* targets, size_t n_targets, int bins,
                                     double* err, uint64_t* count) {
    const size_t n = v->particle_count;
    if (n == 0 || bins < 1) return 1;
    double root[4];
    double* buf;
    size_t* perm;
    OTree t;
    const int status = build_tree(v, &t, root, &buf, &perm);
    if (status != 0) return status;
    /* Morton-slot range of every node: nodes are created after their parents,
     * and a cell's particles are consecutive in Morton order */
    int32_t* lo = (int32_t*)malloc(t.used * sizeof(int32_t));
    int32_t* hi = (int32_t*)malloc(t.used * sizeof(int32_t));
    size_t* slot = (size_t*)malloc(n * sizeof(size_t));
    if (lo == NULL || hi == NULL || slot == NULL) {
        free(lo);
        free(hi);
        free(slot);
        free(buf);
        free(t.nodes);
        free(perm);
        return 2;
    }
    for (size_t k = t.used; k > 0; --k) {
        const ONode* nd = &t.nodes[k - 1];
        if (nd->particle != -1) {
            lo[k - 1] = hi[k - 1] = nd->particle;
            continue;
        }
        int32_t a = INT32_MAX, b = -1;
        for (int c = 0; c < 8; ++c) {
            const int32_t ch = nd->child[c];
            if (ch == -1) continue;
            if (lo[ch] < a) a = lo[ch];
            if (hi[ch] > b) b = hi[ch];
        }
        lo[k - 1] = a;
        hi[k - 1] = b;
    }
    for (size_t i = 0; i < n; ++i) slot[perm[i]] = i;
    const double eps2 = eps * eps;
    memset(err, 0, n_targets * (size_t)bins * 3 * sizeof(double));
    memset(count, 0, n_targets * (size_t)bins * sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 4)
    for (long long k = 0; k < (long long)n_targets; ++k)
        residual_walk(&t, lo, hi, root, G, eps2, theta, slot[targets[k]], bins,
                      err + (size_t)k * bins * 3, count + (size_t)k * bins);
    free(lo);
    free(hi);
    free(slot);
    free(buf);
    free(t.nodes);
    free(perm);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Integrators: src/c/physics/integrator.c:15-172                             */
/* ------------------------------------------------------------------------- */

static int forces(OracleView* v, double G, double eps, int force, double theta) {
    switch (force) {
        case 0:
            oracle_gravity_reference(v, G, eps);
            return 0;
        case 1:
            oracle_gravity_openmp(v, G, eps);
            return 0;
        case 2:
            return oracle_barnes_hut(v, G, eps, theta, NULL);
        default:
            return 1;
    }
}

int oracle_integrator_advance(OracleView* v, double G, double eps, int integrator, double dt,
                              int force, double theta) {
    if (!(dt > 0.0)) return 1;
    const size_t n = v->particle_count;
    double *x = v->positions_x, *y = v->positions_y, *z = v->positions_z;
    double *vx = v->velocities_x, *vy = v->velocities_y, *vz = v->velocities_z;
    double *ax = v->accelerations_x, *ay = v->accelerations_y, *az = v->accelerations_z;
    if (integrator == 0) { /* integrator.c:15-45: force, drift, kick */
        const int s = forces(v, G, eps, force, theta);
        if (s) return s;
        for (size_t i = 0; i < n; ++i) {
            x[i] += vx[i] * dt;
            y[i] += vy[i] * dt;
            z[i] += vz[i] * dt;
            vx[i] += ax[i] * dt;
            vy[i] += ay[i] * dt;
            vz[i] += az[i] * dt;
        }
        return 0;
    }
    if (integrator != 1 && integrator != 2) return 1;
    /* integrator.c:47-85 and :87-139 share the kick-drift-kick arithmetic */
    const double h = 0.5 * dt;
    for (size_t i = 0; i < n; ++i) {
        vx[i] += ax[i] * h;
        vy[i] += ay[i] * h;
        vz[i] += az[i] * h;
        x[i] += vx[i] * dt;
        y[i] += vy[i] * dt;
        z[i] += vz[i] * dt;
    }
    const int s = forces(v, G, eps, force, theta);
    if (s) return s;
    for (size_t i = 0; i < n; ++i) {
        vx[i] += ax[i] * h;
        vy[i] += ay[i] * h;
        vz[i] += az[i] * h;
    }
    return 0;
}
