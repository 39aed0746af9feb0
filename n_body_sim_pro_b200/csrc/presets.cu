// Device generation of the reference's parallel presets for sm_100a.
//
// Reference: src/c/generation/presets_parallel.c (n_body_sim_pro_preset_generate_parallel,
// include/n_body_sim_pro/generation/presets.h:73) and src/c/generation/random.c.
//
// Every particle owns a xoshiro256** generator seeded through splitmix64 with
// mix_seed(master, index) (presets_parallel.c:36-41), so one CUDA thread per
// particle reproduces the reference's integer random streams exactly.  The
// FP64 formulas follow the reference operation by operation; this file is
// compiled without FMA contraction (the reference's generation code has none),
// so products and sums round as on the CPU and only CUDA's log / cos / sin /
// pow / cbrt differ from the host libm by a few ulp.  Mean velocities are
// summed per 256-particle block and then across blocks in a fixed order:
// deterministic, equal to the reference's sequential sums to ~1e-16.
#include "internal.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int kPresetThreads = 256;
constexpr double kPi = 3.14159265358979323846;
constexpr int kRetryLimit = 1000;  // rejection loops (taken with probability ~2^-53)

struct Rng {
  unsigned long long s[4];
};

// random.c:9-26
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long& state) {
  state += 0x9E3779B97F4A7C15ull;
  unsigned long long r = state;
  r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
  r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
  return r ^ (r >> 31);
}

__device__ __forceinline__ void rng_init(Rng& g, unsigned long long seed) {
  unsigned long long st = seed;
  for (int k = 0; k < 4; ++k) g.s[k] = splitmix64(st);
}

__device__ __forceinline__ unsigned long long rotl64(unsigned long long v, int k) {
  return (v << k) | (v >> (64 - k));
}

// random.c:28-40 (xoshiro256**)
__device__ __forceinline__ unsigned long long next_u64(Rng& g) {
  const unsigned long long result = rotl64(g.s[1] * 5ull, 7) * 9ull;
  const unsigned long long t = g.s[1] << 17;
  g.s[2] ^= g.s[0];
  g.s[3] ^= g.s[1];
  g.s[1] ^= g.s[2];
  g.s[0] ^= g.s[3];
  g.s[2] ^= t;
  g.s[3] = rotl64(g.s[3], 45);
  return result;
}

// random.c:42-44
__device__ __forceinline__ double next_double(Rng& g) {
  return (double)(next_u64(g) >> 11) * (1.0 / 9007199254740992.0);
}

// random.c:51-58 (Box-Muller, cosine branch)
__device__ __forceinline__ double next_gaussian(Rng& g) {
  double u1 = 0.0;
  for (int k = 0; k < kRetryLimit && u1 == 0.0; ++k) u1 = next_double(g);
  const double u2 = next_double(g);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * kPi * u2);
}

// presets_parallel.c:36-41
__host__ __device__ __forceinline__ unsigned long long mix_seed(unsigned long long master,
                                                                unsigned long long index) {
  unsigned long long x = master ^ (index + 0x9E3779B97F4A7C15ull);
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// The isotropic direction of presets_parallel.c:109-121 (normalised gaussians).
__device__ __forceinline__ void unit_vector(Rng& g, double& x, double& y, double& z) {
  x = 1.0;
  y = 0.0;
  z = 0.0;
  for (int k = 0; k < kRetryLimit; ++k) {
    const double a = next_gaussian(g);
    const double b = next_gaussian(g);
    const double c = next_gaussian(g);
    const double norm = sqrt(a * a + b * b + c * c);
    if (norm > 1.0e-12) {
      x = a / norm;
      y = b / norm;
      z = c / norm;
      return;
    }
  }
}

struct State {
  double *x, *y, *z, *vx, *vy, *vz, *m;
};

__device__ __forceinline__ void put(const State& s, size_t i, double x, double y, double z,
                                    double vx, double vy, double vz, double m) {
  s.x[i] = x;
  s.y[i] = y;
  s.z[i] = z;
  s.vx[i] = vx;
  s.vy[i] = vy;
  s.vz[i] = vz;
  s.m[i] = m;
}

// Velocity sums of one 256-particle block into partial[3 * blockIdx.x + c]
// (fixed tree order: deterministic).
__device__ __forceinline__ void block_velocity_sums(double vx, double vy, double vz,
                                                    double* __restrict__ partial) {
  __shared__ double sh[3][kPresetThreads / 32];
  for (int off = 16; off > 0; off >>= 1) {
    vx += __shfl_down_sync(0xffffffffu, vx, off);
    vy += __shfl_down_sync(0xffffffffu, vy, off);
    vz += __shfl_down_sync(0xffffffffu, vz, off);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][w] = vx;
    sh[1][w] = vy;
    sh[2][w] = vz;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int k = 0; k < kPresetThreads / 32; ++k) t += sh[threadIdx.x][k];
    partial[3 * blockIdx.x + threadIdx.x] = t;
  }
}

// presets_parallel.c:91-155 (+ the triple galaxy's centres, :428-431)
__global__ void __launch_bounds__(kPresetThreads) plummer_kernel(
    State s, unsigned long long master, size_t start, size_t count, double a, double a2,
    double total_mass, double particle_mass, int has_centre, double cx, double cy, double cz,
    double* __restrict__ partial) {
  const size_t k = blockIdx.x * (size_t)kPresetThreads + threadIdx.x;
  double vx = 0.0, vy = 0.0, vz = 0.0;
  if (k < count) {
    const size_t i = start + k;
    Rng g;
    rng_init(g, mix_seed(master, i));
    const double u = 1.0 - next_double(g);
    const double r = a / sqrt(pow(u, -2.0 / 3.0) - 1.0);
    double dx, dy, dz;
    unit_vector(g, dx, dy, dz);
    double px = r * dx, py = r * dy, pz = r * dz;
    if (has_centre) {
      px = px + cx;
      py = py + cy;
      pz = pz + cz;
    }
    const double sigma = sqrt(1.0 * total_mass / (6.0 * sqrt(a2 + r * r)));
    vx = next_gaussian(g) * sigma;
    vy = next_gaussian(g) * sigma;
    vz = next_gaussian(g) * sigma;
    put(s, i, px, py, pz, vx, vy, vz, particle_mass);
  }
  block_velocity_sums(vx, vy, vz, partial);
}

// presets_parallel.c:158-217
__global__ void __launch_bounds__(kPresetThreads) disk_kernel(
    State s, unsigned long long master, size_t start, size_t count, double a, double h, double vc,
    double sigma, double twist, int arms, double particle_mass, double* __restrict__ partial) {
  const size_t k = blockIdx.x * (size_t)kPresetThreads + threadIdx.x;
  double vx = 0.0, vy = 0.0, vz = 0.0;
  if (k < count) {
    const size_t i = start + k;
    Rng g;
    rng_init(g, mix_seed(master, i));
    const double e1 = -log(1.0 - next_double(g));
    const double e2 = -log(1.0 - next_double(g));
    const double r = a * (e1 + e2);
    double phi = 2.0 * kPi * next_double(g);
    if (twist > 0.0 && arms > 0) {
      const double arm = next_double(g) * (double)arms;
      const double arm_phi = 2.0 * kPi * arm / (double)arms + twist * r / a;
      phi = arm_phi + next_gaussian(g) * 0.15;
    }
    const double z = next_gaussian(g) * h;
    const double tx = -sin(phi), ty = cos(phi);
    const double px = r * cos(phi), py = r * sin(phi);
    vx = vc * tx + next_gaussian(g) * sigma;
    vy = vc * ty + next_gaussian(g) * sigma;
    vz = next_gaussian(g) * sigma * 0.5;
    put(s, i, px, py, z, vx, vy, vz, particle_mass);
  }
  block_velocity_sums(vx, vy, vz, partial);
}

// presets_parallel.c:219-272
__global__ void __launch_bounds__(kPresetThreads) cloud_kernel(State s, unsigned long long seed,
                                                               size_t count, double particle_mass,
                                                               double* __restrict__ partial) {
  const size_t i = blockIdx.x * (size_t)kPresetThreads + threadIdx.x;
  double vx = 0.0, vy = 0.0, vz = 0.0;
  if (i < count) {
    Rng g;
    rng_init(g, mix_seed(seed, i));
    double dx, dy, dz;
    unit_vector(g, dx, dy, dz);
    const double r = cbrt(next_double(g));
    vx = -0.05 + (0.05 - -0.05) * next_double(g);
    vy = -0.05 + (0.05 - -0.05) * next_double(g);
    vz = -0.05 + (0.05 - -0.05) * next_double(g);
    put(s, i, r * dx, r * dy, r * dz, vx, vy, vz, particle_mass);
  }
  block_velocity_sums(vx, vy, vz, partial);
}

// presets_parallel.c:274-311
__global__ void __launch_bounds__(kPresetThreads) open_cluster_kernel(
    State s, unsigned long long seed, size_t count, double particle_mass,
    double* __restrict__ partial) {
  const size_t i = blockIdx.x * (size_t)kPresetThreads + threadIdx.x;
  double vx = 0.0, vy = 0.0, vz = 0.0;
  if (i < count) {
    Rng g;
    rng_init(g, mix_seed(seed, i));
    const double px = next_gaussian(g) * 0.3;
    const double py = next_gaussian(g) * 0.3;
    const double pz = next_gaussian(g) * 0.3;
    vx = next_gaussian(g) * 0.02;
    vy = next_gaussian(g) * 0.02;
    vz = next_gaussian(g) * 0.02;
    put(s, i, px, py, pz, vx, vy, vz, particle_mass);
  }
  block_velocity_sums(vx, vy, vz, partial);
}

// presets_parallel.c:59-89: one sequential stream seeded with `seed` (one thread).
__global__ void solar_kernel(State s, unsigned long long seed, size_t count) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Rng g;
  rng_init(g, seed);
  put(s, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0);
  const size_t planets = count - 1;
  for (size_t k = 0; k < planets; ++k) {
    const double r = 1.0 + 3.0 * (double)k / (double)planets;
    const double speed = sqrt(1.0 / r);
    const double phi = 2.0 * kPi * next_double(g);
    put(s, k + 1, r * cos(phi), r * sin(phi), 0.0, -speed * sin(phi), speed * cos(phi), 0.0,
        0.001);
  }
}

// presets_parallel.c:43-57
__global__ void two_body_kernel(State s) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double speed = sqrt(2.0) / 2.0;
  put(s, 0, -0.5, 0.0, 0.0, 0.0, speed, 0.0, 1.0);
  put(s, 1, 0.5, 0.0, 0.0, 0.0, -speed, 0.0, 1.0);
}

// One block: mean = (sum of the block partials in block order) / count.
__global__ void __launch_bounds__(1024) mean_kernel(const double* __restrict__ partial,
                                                    int blocks, size_t count,
                                                    double* __restrict__ mean) {
  __shared__ double sh[3][1024];
  double t[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < blocks; b += 1024)
    for (int c = 0; c < 3; ++c) t[c] += partial[3 * b + c];
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = t[c];
  __syncthreads();
  for (int stride = 512; stride > 0; stride >>= 1) {
    if ((int)threadIdx.x < stride)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x < 3) mean[threadIdx.x] = sh[threadIdx.x][0] / (double)count;
}

__global__ void subtract_mean_kernel(State s, size_t start, size_t count,
                                     const double* __restrict__ mean) {
  const double mx = mean[0], my = mean[1], mz = mean[2];
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < count;
       k += (size_t)gridDim.x * blockDim.x) {
    s.vx[start + k] -= mx;
    s.vy[start + k] -= my;
    s.vz[start + k] -= mz;
  }
}

// Relative velocity of the two-Plummer collision: -speed/2 on y for the first
// block, +speed/2 for the second (added after each block's mean removal).
__global__ void shear_kernel(State s, size_t half, size_t count, double half_speed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x)
    s.vy[i] += i < half ? -half_speed : half_speed;
}

// presets_parallel.c:393-395: +0.35 on x for the first half, -0.35 for the rest
__global__ void approach_kernel(State s, size_t half, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x)
    s.vx[i] += i < half ? 0.35 : -0.35;
}

unsigned blocks_for(size_t count) {
  return (unsigned)((count + kPresetThreads - 1) / kPresetThreads);
}

unsigned grid_stride_blocks(size_t count) {
  size_t b = (count + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)b;
}

// Mean removal of [start, start + count) after a generation kernel filled `partial`.
void remove_mean(const State& s, size_t start, size_t count, double* partial, double* mean,
                 cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), mean_kernel<<<1, 1024, 0, stream>>>(partial, (int)blocks_for(count), count, mean);
  NBSP_COUNT_LAUNCH(1), subtract_mean_kernel<<<grid_stride_blocks(count), 256, 0, stream>>>(s, start, count, mean);
}

}  // namespace

extern "C" {

size_t nbsp_preset_scratch_doubles(size_t n) { return 3 * ((size_t)blocks_for(n) + 1) + 8; }

int nbsp_preset_generate(int preset, size_t n, uint64_t seed, double* x, double* y, double* z,
                         double* vx, double* vy, double* vz, double* m, double* scratch,
                         cudaStream_t stream) {
  const State s{x, y, z, vx, vy, vz, m};
  double* mean = scratch;         // 3 (+ padding)
  double* partial = scratch + 8;  // 3 per block
  switch (preset) {
    case 0:  // two body
      if (n != 2) return 1;
      NBSP_COUNT_LAUNCH(1), two_body_kernel<<<1, 32, 0, stream>>>(s);
      return 0;
    case 1:  // random cloud
      if (n == 0) return 1;
      NBSP_COUNT_LAUNCH(1), cloud_kernel<<<blocks_for(n), kPresetThreads, 0, stream>>>(s, seed, n, 1.0 / (double)n,
                                                                   partial);
      remove_mean(s, 0, n, partial, mean, stream);
      return 0;
    case 2:  // solar system
      if (n == 0) return 1;
      NBSP_COUNT_LAUNCH(1), solar_kernel<<<1, 32, 0, stream>>>(s, seed, n);
      return 0;
    case 3:  // open cluster
      if (n == 0) return 1;
      NBSP_COUNT_LAUNCH(1), open_cluster_kernel<<<blocks_for(n), kPresetThreads, 0, stream>>>(
          s, seed, n, 1.0 / (double)n, partial);
      remove_mean(s, 0, n, partial, mean, stream);
      return 0;
    case 4:  // globular cluster (a = 1)
    case 6: {  // elliptical galaxy (a = 2)
      if (n == 0) return 1;
      const double a = preset == 4 ? 1.0 : 2.0;
      NBSP_COUNT_LAUNCH(1), plummer_kernel<<<blocks_for(n), kPresetThreads, 0, stream>>>(
          s, seed, 0, n, a, a * a, 1.0, 1.0 / (double)n, 0, 0.0, 0.0, 0.0, partial);
      remove_mean(s, 0, n, partial, mean, stream);
      return 0;
    }
    case 5:  // spiral galaxy
      if (n == 0) return 1;
      NBSP_COUNT_LAUNCH(1), disk_kernel<<<blocks_for(n), kPresetThreads, 0, stream>>>(
          s, seed, 0, n, 0.7, 0.1, 1.0, 0.12, 3.5, 2, 1.0 / (double)n, partial);
      remove_mean(s, 0, n, partial, mean, stream);
      return 0;
    case 7: {  // galaxy collision: two arm-less disks, then the approach velocities
      const size_t half = n / 2;
      if (half == 0) return 1;
      const double pm = 0.5 / (double)half;
      for (int d = 0; d < 2; ++d) {
        NBSP_COUNT_LAUNCH(1), disk_kernel<<<blocks_for(half), kPresetThreads, 0, stream>>>(
            s, mix_seed(seed, (uint64_t)d), (size_t)d * half, half, 0.7, 0.1, 1.0, 0.12, 0.0,
            0, pm, partial);
        remove_mean(s, (size_t)d * half, half, partial, mean, stream);
      }
      NBSP_COUNT_LAUNCH(1), approach_kernel<<<grid_stride_blocks(n), 256, 0, stream>>>(s, half, n);
      return 0;
    }
    case 8: {  // triple galaxy: three Plummer spheres (a = 0.7; 0.49 as in :446)
      const size_t third = n / 3;
      if (third == 0) return 1;
      const double centres[3][3] = {{-1.8, 0.0, 0.0}, {1.8, 0.0, 0.0}, {0.0, 1.8, 0.0}};
      for (int gal = 0; gal < 3; ++gal) {
        NBSP_COUNT_LAUNCH(1), plummer_kernel<<<blocks_for(third), kPresetThreads, 0, stream>>>(
            s, mix_seed(seed, (uint64_t)gal), (size_t)gal * third, third, 0.7, 0.49,
            1.0 / 3.0, (1.0 / 3.0) / (double)third, 1, centres[gal][0], centres[gal][1],
            centres[gal][2], partial);
        remove_mean(s, (size_t)gal * third, third, partial, mean, stream);
      }
      return 0;
    }
    default:
      return 1;
  }
}

// Two Plummer spheres (scale radius a, mass 1/2 each) in the reference's
// parallel-preset form, the way its galaxy_collision (presets_parallel.c:392-404)
// builds two disk blocks: block b fills [b * half, b * half + count_b) from the
// per-particle generators mix_seed(mix_seed(seed, b), index) (fill_plummer_block,
// :91-155), centred at -/+ separation / 2 on x, its mean velocity removed;
// then -/+ relative_speed / 2 on y.  Block 1 takes n - n/2 particles.
int nbsp_plummer_collision_generate(size_t n, uint64_t seed, double a, double separation,
                                    double relative_speed, double* x, double* y, double* z,
                                    double* vx, double* vy, double* vz, double* m,
                                    double* scratch, cudaStream_t stream) {
  const State s{x, y, z, vx, vy, vz, m};
  double* mean = scratch;
  double* partial = scratch + 8;
  const size_t half = n / 2;
  if (half == 0) return 1;
  for (int b = 0; b < 2; ++b) {
    const size_t start = (size_t)b * half;
    const size_t count = b == 0 ? half : n - half;
    const double cx = (b == 0 ? -0.5 : 0.5) * separation;
    NBSP_COUNT_LAUNCH(1), plummer_kernel<<<blocks_for(count), kPresetThreads, 0, stream>>>(
        s, mix_seed(seed, (uint64_t)b), start, count, a, a * a, 0.5, 0.5 / (double)count, 1, cx,
        0.0, 0.0, partial);
    remove_mean(s, start, count, partial, mean, stream);
  }
  NBSP_COUNT_LAUNCH(1), shear_kernel<<<grid_stride_blocks(n), 256, 0, stream>>>(
      s, half, n, 0.5 * relative_speed);
  return 0;
}

}  // extern "C"
