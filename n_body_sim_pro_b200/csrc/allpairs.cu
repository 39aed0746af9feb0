// All-pairs softened gravity, fused leapfrog kick/drift, and FP64 diagnostics
// for sm_100a.
//
// Reference arithmetic (richie-rich90454/n_body_sim_pro):
//   pair force     src/c/physics/gravity.c:46-61
//   kick / drift   src/c/physics/integrator.c:47-85 (leapfrog KDK),
//                  :87-139 (velocity Verlet, same arithmetic), :15-45 (Euler)
//   diagnostics    src/c/diagnostics/numerics.c:5-116
//
// Force kernel design (FP32-pipe bound):
//   * sources are packed once per step as float4 (x - c, y - c, z - c, m) with c
//     the FP64 centre of mass, so FP32 works on small relative coordinates;
//   * each CTA owns BLOCK*K targets (K per thread, in registers) and one chunk
//     of sources (grid.y); sources stream through a BLOCK-wide shared-memory
//     tile that every lane reads with a broadcast LDS.128;
//   * per interaction: 3 FADD + 3 FFMA (r^2) + 1 MUFU.RSQ + 3 FMUL + 3 FFMA;
//   * each tile's sum is folded into a (hi, lo) pair with TwoSum, so the
//     rounding error grows with the number of tiles, not of sources;
//   * chunk partials (hi, lo) are reduced in FP64 by the epilogue kernel, which
//     also applies G and the leapfrog kick/drift in FP64.
#include "internal.h"

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

namespace {

__device__ __forceinline__ float rsqrt_mufu(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Knuth TwoSum of (hi, lo) += a; __fadd_rn/__fsub_rn are never contracted or
// reassociated.
__device__ __forceinline__ void fold(float& hi, float& lo, float a) {
  const float s = __fadd_rn(hi, a);
  const float bp = __fsub_rn(s, hi);
  const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(a, bp));
  hi = s;
  lo = __fadd_rn(lo, err);
}

// Source chunks start and end on multiples of kChunkAlign sources, so a chunk's
// last tile may be partial; the packed array is padded to a multiple of 256
// with massless sources.
constexpr int kChunkAlign = NBSP_ALLPAIRS_CHUNK_ALIGN;

template <int BLOCK, int K, bool ZERO_SOFTENING>
__global__ void __launch_bounds__(BLOCK) allpairs_force_kernel(
    const float4* __restrict__ packed, const float4* __restrict__ targets, int n, int n_padded,
    int chunk_len, float eps2, float4* __restrict__ hi_out, float4* __restrict__ lo_out) {
  __shared__ float4 tile[BLOCK];
  const int tid = threadIdx.x;
  const int first_target = blockIdx.x * (BLOCK * K) + tid;

  float xi[K], yi[K], zi[K];
  float ax[K], ay[K], az[K];
  float hx[K], hy[K], hz[K], lx[K], ly[K], lz[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i = first_target + k * BLOCK;
    const float4 q = i < n ? targets[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    xi[k] = q.x;
    yi[k] = q.y;
    zi[k] = q.z;
    hx[k] = hy[k] = hz[k] = 0.f;
    lx[k] = ly[k] = lz[k] = 0.f;
  }

  const int j0 = blockIdx.y * chunk_len;
  const int j1 = min(j0 + chunk_len, n_padded);
  float4 next = j0 + tid < j1 ? packed[j0 + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int jt = j0; jt < j1; jt += BLOCK) {
    __syncthreads();
    tile[tid] = next;
    __syncthreads();
    next = jt + BLOCK + tid < j1 ? packed[jt + BLOCK + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < K; ++k) ax[k] = ay[k] = az[k] = 0.f;
    const int count = min(BLOCK, j1 - jt);  // a multiple of kChunkAlign
    for (int j8 = 0; j8 < count; j8 += kChunkAlign)
#pragma unroll
    for (int j = j8; j < j8 + kChunkAlign; ++j) {
      const float4 s = tile[j];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const float dx = s.x - xi[k];
        const float dy = s.y - yi[k];
        const float dz = s.z - zi[k];
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        float rinv = rsqrt_mufu(r2);
        if (ZERO_SOFTENING) rinv = r2 > 0.f ? rinv : 0.f;  // self pair (gravity.c:43-45)
        const float w = s.w * (rinv * rinv * rinv);
        ax[k] = fmaf(w, dx, ax[k]);
        ay[k] = fmaf(w, dy, ay[k]);
        az[k] = fmaf(w, dz, az[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      fold(hx[k], lx[k], ax[k]);
      fold(hy[k], ly[k], ay[k]);
      fold(hz[k], lz[k], az[k]);
    }
  }

  const size_t base = (size_t)blockIdx.y * (size_t)n;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i = first_target + k * BLOCK;
    if (i < n) {
      hi_out[base + i] = make_float4(hx[k], hy[k], hz[k], 0.f);
      lo_out[base + i] = make_float4(lx[k], ly[k], lz[k], 0.f);
    }
  }
}

// Paired variant: sm_100 executes two FP32 lanes' worth of add/mul/fma per
// instruction with the .f32x2 forms, so two targets share every arithmetic
// instruction of the interaction; only the MUFU rsqrt stays scalar.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

template <int BLOCK, int K, bool ZERO_SOFTENING, int MIN_BLOCKS = 1>
__global__ void __launch_bounds__(BLOCK, MIN_BLOCKS) allpairs_force_paired_kernel(
    const float4* __restrict__ packed, const float4* __restrict__ targets, int n, int n_padded,
    int chunk_len, float eps2, float4* __restrict__ hi_out, float4* __restrict__ lo_out) {
  static_assert(K % 2 == 0, "targets are processed in pairs");
  constexpr int P = K / 2;
  __shared__ float4 tile[BLOCK];
  const int tid = threadIdx.x;
  const int first_target = blockIdx.x * (BLOCK * K) + tid;

  unsigned long long X[P], Y[P], Z[P];
  float hx[K], hy[K], hz[K], lx[K], ly[K], lz[K];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int i0 = first_target + (2 * p) * BLOCK, i1 = first_target + (2 * p + 1) * BLOCK;
    const float4 a = i0 < n ? targets[i0] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 b = i1 < n ? targets[i1] : make_float4(0.f, 0.f, 0.f, 0.f);
    X[p] = pack2(a.x, b.x);
    Y[p] = pack2(a.y, b.y);
    Z[p] = pack2(a.z, b.z);
  }
#pragma unroll
  for (int k = 0; k < K; ++k) hx[k] = hy[k] = hz[k] = lx[k] = ly[k] = lz[k] = 0.f;
  const unsigned long long E2 = pack2(eps2, eps2);

  const int j0 = blockIdx.y * chunk_len;
  const int j1 = min(j0 + chunk_len, n_padded);
  float4 next = j0 + tid < j1 ? packed[j0 + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int jt = j0; jt < j1; jt += BLOCK) {
    __syncthreads();
    tile[tid] = next;
    __syncthreads();
    next = jt + BLOCK + tid < j1 ? packed[jt + BLOCK + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned long long AX[P], AY[P], AZ[P];
#pragma unroll
    for (int p = 0; p < P; ++p) AX[p] = AY[p] = AZ[p] = 0ull;
    const int count = min(BLOCK, j1 - jt);  // a multiple of kChunkAlign
    for (int j8 = 0; j8 < count; j8 += kChunkAlign)
#pragma unroll
    for (int j = j8; j < j8 + kChunkAlign; ++j) {
      const float4 s = tile[j];
      const unsigned long long SX = pack2(s.x, s.x), SY = pack2(s.y, s.y), SZ = pack2(s.z, s.z);
      const unsigned long long SW = pack2(s.w, s.w);
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const unsigned long long dx = sub2(SX, X[p]);
        const unsigned long long dy = sub2(SY, Y[p]);
        const unsigned long long dz = sub2(SZ, Z[p]);
        const unsigned long long r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
        float r2a, r2b;
        unpack2(r2, r2a, r2b);
        float ra = rsqrt_mufu(r2a), rb = rsqrt_mufu(r2b);
        if (ZERO_SOFTENING) {
          ra = r2a > 0.f ? ra : 0.f;
          rb = r2b > 0.f ? rb : 0.f;
        }
        const unsigned long long R = pack2(ra, rb);
        const unsigned long long W = mul2(SW, mul2(mul2(R, R), R));
        AX[p] = fma2(W, dx, AX[p]);
        AY[p] = fma2(W, dy, AY[p]);
        AZ[p] = fma2(W, dz, AZ[p]);
      }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      float a, b;
      unpack2(AX[p], a, b);
      fold(hx[2 * p], lx[2 * p], a);
      fold(hx[2 * p + 1], lx[2 * p + 1], b);
      unpack2(AY[p], a, b);
      fold(hy[2 * p], ly[2 * p], a);
      fold(hy[2 * p + 1], ly[2 * p + 1], b);
      unpack2(AZ[p], a, b);
      fold(hz[2 * p], lz[2 * p], a);
      fold(hz[2 * p + 1], lz[2 * p + 1], b);
    }
  }

  const size_t base = (size_t)blockIdx.y * (size_t)n;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int i = first_target + k * BLOCK;
    if (i < n) {
      hi_out[base + i] = make_float4(hx[k], hy[k], hz[k], 0.f);
      lo_out[base + i] = make_float4(lx[k], ly[k], lz[k], 0.f);
    }
  }
}

typedef void (*ForceKernel)(const float4*, const float4*, int, int, int, float, float4*,
                            float4*);

template <int BLOCK, int K>
ForceKernel pick(bool zero_softening) {
  return zero_softening ? allpairs_force_kernel<BLOCK, K, true>
                        : allpairs_force_kernel<BLOCK, K, false>;
}

template <int BLOCK, int K, int MIN_BLOCKS = 1>
ForceKernel pick_paired(bool zero_softening) {
  return zero_softening ? allpairs_force_paired_kernel<BLOCK, K, true, MIN_BLOCKS>
                        : allpairs_force_paired_kernel<BLOCK, K, false, MIN_BLOCKS>;
}

ForceKernel select_kernel(NbspAllPairsShape s, bool zero_softening) {
  if (s.paired && s.min_blocks > 0) {  // register caps for more resident warps
    if (s.block == 256 && s.per_thread == 2 && s.min_blocks == 4)
      return pick_paired<256, 2, 4>(zero_softening);
    if (s.block == 128 && s.per_thread == 4 && s.min_blocks == 6)
      return pick_paired<128, 4, 6>(zero_softening);
    return nullptr;
  }
  if (s.paired) {
    if (s.block == 64 && s.per_thread == 4) return pick_paired<64, 4>(zero_softening);
    if (s.block == 64 && s.per_thread == 8) return pick_paired<64, 8>(zero_softening);
    if (s.block == 128 && s.per_thread == 2) return pick_paired<128, 2>(zero_softening);
    if (s.block == 256 && s.per_thread == 2) return pick_paired<256, 2>(zero_softening);
    if (s.block == 128 && s.per_thread == 4) return pick_paired<128, 4>(zero_softening);
    if (s.block == 128 && s.per_thread == 8) return pick_paired<128, 8>(zero_softening);
    if (s.block == 256 && s.per_thread == 4) return pick_paired<256, 4>(zero_softening);
    return nullptr;
  }
#define NBSP_CASE(B, K) \
  if (s.block == B && s.per_thread == K) return pick<B, K>(zero_softening);
  NBSP_CASE(64, 4)
  NBSP_CASE(64, 8)
  NBSP_CASE(128, 1)
  NBSP_CASE(128, 2)
  NBSP_CASE(128, 4)
  NBSP_CASE(128, 8)
  NBSP_CASE(256, 1)
  NBSP_CASE(256, 2)
  NBSP_CASE(256, 4)
#undef NBSP_CASE
  return nullptr;
}

// a = G * sum over chunks of (hi + lo), in FP64.
__device__ __forceinline__ void reduce_partials(const float4* __restrict__ hi,
                                                const float4* __restrict__ lo, size_t n, int chunks,
                                                size_t i, double g, double& ax, double& ay,
                                                double& az) {
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int s = 0; s < chunks; ++s) {
    const float4 h = hi[(size_t)s * n + i];
    const float4 l = lo[(size_t)s * n + i];
    sx += (double)h.x + (double)l.x;
    sy += (double)h.y + (double)l.y;
    sz += (double)h.z + (double)l.z;
  }
  ax = g * sx;
  ay = g * sy;
  az = g * sz;
}

__device__ __forceinline__ float4 relative(double x, double y, double z, double m,
                                           const double* centre) {
  return make_float4((float)__dsub_rn(x, centre[0]), (float)__dsub_rn(y, centre[1]),
                     (float)__dsub_rn(z, centre[2]), (float)m);
}

__device__ __forceinline__ bool finite3(double x, double y, double z) {
  return isfinite(x) && isfinite(y) && isfinite(z);
}

__global__ void pack_kernel(const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ m, size_t n,
                            size_t n_padded, const double* __restrict__ centre,
                            float4* __restrict__ packed, int* status) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_padded;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i < n) {
      if (!finite3(x[i], y[i], z[i])) atomicOr(status, NBSP_DEVICE_ERROR_NONFINITE_POSITION);
      packed[i] = relative(x[i], y[i], z[i], m[i], centre);
    } else {
      packed[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

__global__ void finalize_kernel(const float4* __restrict__ hi, const float4* __restrict__ lo,
                                size_t n, int chunks, double g, double* __restrict__ ax,
                                double* __restrict__ ay, double* __restrict__ az) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double a0, a1, a2;
    reduce_partials(hi, lo, n, chunks, i, g, a0, a1, a2);
    ax[i] = a0;
    ay[i] = a1;
    az[i] = a2;
  }
}

// v += a*h ; x += v*dt   (integrator.c:64-72), FP64, never contracted.
__global__ void kick_drift_kernel(double* __restrict__ x, double* __restrict__ y,
                                  double* __restrict__ z, double* __restrict__ vx,
                                  double* __restrict__ vy, double* __restrict__ vz,
                                  const double* __restrict__ ax, const double* __restrict__ ay,
                                  const double* __restrict__ az, size_t n, double h, double dt) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double u = __dadd_rn(vx[i], __dmul_rn(ax[i], h));
    const double v = __dadd_rn(vy[i], __dmul_rn(ay[i], h));
    const double w = __dadd_rn(vz[i], __dmul_rn(az[i], h));
    vx[i] = u;
    vy[i] = v;
    vz[i] = w;
    if (dt != 0.0) {
      x[i] = __dadd_rn(x[i], __dmul_rn(u, dt));
      y[i] = __dadd_rn(y[i], __dmul_rn(v, dt));
      z[i] = __dadd_rn(z[i], __dmul_rn(w, dt));
    }
  }
}

// Euler: x += v*dt ; v += a*dt   (integrator.c:35-44).
__global__ void euler_kernel(double* __restrict__ x, double* __restrict__ y,
                             double* __restrict__ z, double* __restrict__ vx,
                             double* __restrict__ vy, double* __restrict__ vz,
                             const double* __restrict__ ax, const double* __restrict__ ay,
                             const double* __restrict__ az, size_t n, double dt) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    x[i] = __dadd_rn(x[i], __dmul_rn(vx[i], dt));
    y[i] = __dadd_rn(y[i], __dmul_rn(vy[i], dt));
    z[i] = __dadd_rn(z[i], __dmul_rn(vz[i], dt));
    vx[i] = __dadd_rn(vx[i], __dmul_rn(ax[i], dt));
    vy[i] = __dadd_rn(vy[i], __dmul_rn(ay[i], dt));
    vz[i] = __dadd_rn(vz[i], __dmul_rn(az[i], dt));
  }
}

__global__ void finalize_kick_kernel(const float4* __restrict__ hi, const float4* __restrict__ lo,
                                     size_t n, int chunks, double g, double* __restrict__ ax,
                                     double* __restrict__ ay, double* __restrict__ az,
                                     double* __restrict__ vx, double* __restrict__ vy,
                                     double* __restrict__ vz, double h) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double a0, a1, a2;
    reduce_partials(hi, lo, n, chunks, i, g, a0, a1, a2);
    ax[i] = a0;
    ay[i] = a1;
    az[i] = a2;
    vx[i] = __dadd_rn(vx[i], __dmul_rn(a0, h));
    vy[i] = __dadd_rn(vy[i], __dmul_rn(a1, h));
    vz[i] = __dadd_rn(vz[i], __dmul_rn(a2, h));
  }
}

// Closing kick of step n, opening kick + drift of step n+1, repack.
__global__ void finalize_kick_kick_drift_pack_kernel(
    const float4* __restrict__ hi, const float4* __restrict__ lo, size_t n, size_t n_padded,
    int chunks, double g, double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
    double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
    double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
    const double* __restrict__ m, double h, double dt, const double* __restrict__ centre,
    float4* __restrict__ packed, int* status) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_padded;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i >= n) {
      packed[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    double a0, a1, a2;
    reduce_partials(hi, lo, n, chunks, i, g, a0, a1, a2);
    ax[i] = a0;
    ay[i] = a1;
    az[i] = a2;
    double u = __dadd_rn(vx[i], __dmul_rn(a0, h));
    double v = __dadd_rn(vy[i], __dmul_rn(a1, h));
    double w = __dadd_rn(vz[i], __dmul_rn(a2, h));
    u = __dadd_rn(u, __dmul_rn(a0, h));
    v = __dadd_rn(v, __dmul_rn(a1, h));
    w = __dadd_rn(w, __dmul_rn(a2, h));
    vx[i] = u;
    vy[i] = v;
    vz[i] = w;
    const double px = __dadd_rn(x[i], __dmul_rn(u, dt));
    const double py = __dadd_rn(y[i], __dmul_rn(v, dt));
    const double pz = __dadd_rn(z[i], __dmul_rn(w, dt));
    x[i] = px;
    y[i] = py;
    z[i] = pz;
    if (!finite3(px, py, pz)) atomicOr(status, NBSP_DEVICE_ERROR_NONFINITE_POSITION);
    packed[i] = relative(px, py, pz, m[i], centre);
  }
}

constexpr int kSumBlocks = 1024;
constexpr int kSumThreads = 256;
constexpr int kQuantities = 11;

__device__ __forceinline__ void block_sum(double* sh, double* vals, int count) {
  // sh: count * kSumThreads; fixed-order tree reduction.
  const int t = threadIdx.x;
  for (int q = 0; q < count; ++q) sh[q * kSumThreads + t] = vals[q];
  __syncthreads();
  for (int stride = kSumThreads / 2; stride > 0; stride >>= 1) {
    if (t < stride) {
      for (int q = 0; q < count; ++q)
        sh[q * kSumThreads + t] += sh[q * kSumThreads + t + stride];
    }
    __syncthreads();
  }
}

// numerics.c:35-60 per-particle terms, summed per thread in index order.
__global__ void __launch_bounds__(kSumThreads) global_sums_kernel(
    const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
    const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
    const double* __restrict__ m, size_t n, int quantities, double* __restrict__ partial) {
  __shared__ double sh[kQuantities * kSumThreads];
  double acc[kQuantities];
  for (int q = 0; q < kQuantities; ++q) acc[q] = 0.0;
  for (size_t i = blockIdx.x * (size_t)kSumThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kSumThreads) {
    const double mi = m[i];
    const double px = x[i], py = y[i], pz = z[i];
    if (quantities == kQuantities) {
      const double u = vx[i], v = vy[i], w = vz[i];
      acc[0] += 0.5 * mi * (u * u + v * v + w * w);
      acc[1] += mi;
      acc[2] += mi * u;
      acc[3] += mi * v;
      acc[4] += mi * w;
      acc[5] += mi * (py * w - pz * v);
      acc[6] += mi * (pz * u - px * w);
      acc[7] += mi * (px * v - py * u);
    } else {
      acc[1] += mi;
    }
    acc[8] += mi * px;
    acc[9] += mi * py;
    acc[10] += mi * pz;
  }
  block_sum(sh, acc, kQuantities);
  if (threadIdx.x == 0) {
    for (int q = 0; q < kQuantities; ++q) partial[blockIdx.x * kQuantities + q] = sh[q * kSumThreads];
  }
}

__global__ void __launch_bounds__(kSumThreads) global_sums_final_kernel(
    const double* __restrict__ partial, int blocks, double* __restrict__ out, int centre_only) {
  __shared__ double sh[kQuantities * kSumThreads];
  double acc[kQuantities];
  for (int q = 0; q < kQuantities; ++q) acc[q] = 0.0;
  for (int b = threadIdx.x; b < blocks; b += kSumThreads)
    for (int q = 0; q < kQuantities; ++q) acc[q] += partial[b * kQuantities + q];
  block_sum(sh, acc, kQuantities);
  if (threadIdx.x == 0) {
    if (centre_only) {
      const double mt = sh[1 * kSumThreads];
      for (int c = 0; c < 3; ++c) out[c] = mt != 0.0 ? sh[(8 + c) * kSumThreads] / mt : 0.0;
    } else {
      for (int q = 0; q < kQuantities; ++q) out[q] = sh[q * kSumThreads];
    }
  }
}

int sum_blocks(size_t n) {
  const size_t b = (n + kSumThreads - 1) / kSumThreads;
  return (int)(b < 1 ? 1 : (b > (size_t)kSumBlocks ? (size_t)kSumBlocks : b));
}

// Pair potential m_i m_j / sqrt(d^2 + eps^2) summed over j > i per row (FP64).
constexpr int kPeThreads = 128;
__global__ void __launch_bounds__(kPeThreads) potential_rows_kernel(
    const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
    const double* __restrict__ m, int n, double eps2, double* __restrict__ rows) {
  __shared__ double4 tile[kPeThreads];
  const int i = blockIdx.x * kPeThreads + threadIdx.x;
  const double xi = i < n ? x[i] : 0.0, yi = i < n ? y[i] : 0.0, zi = i < n ? z[i] : 0.0;
  double s = 0.0;
  const int first = blockIdx.x * kPeThreads;
  for (int jt = first; jt < n; jt += kPeThreads) {
    __syncthreads();
    const int j = jt + threadIdx.x;
    tile[threadIdx.x] = j < n ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int jn = min(kPeThreads, n - jt);
    for (int k = 0; k < jn; ++k) {
      if (jt + k <= i) continue;
      const double4 q = tile[k];
      const double dx = __dsub_rn(q.x, xi), dy = __dsub_rn(q.y, yi), dz = __dsub_rn(q.z, zi);
      const double r2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                            __dmul_rn(dz, dz)),
                                  eps2);
      s += q.w * rsqrt(r2);
    }
  }
  if (i < n) rows[i] = m[i] * s;
}

__global__ void __launch_bounds__(kSumThreads) rows_sum_kernel(const double* __restrict__ rows,
                                                               size_t n, double scale,
                                                               double* __restrict__ out) {
  __shared__ double sh[kSumThreads];
  double acc = 0.0;
  for (size_t i = threadIdx.x; i < n; i += kSumThreads) acc += rows[i];
  block_sum(sh, &acc, 1);
  if (threadIdx.x == 0) out[0] = scale * sh[0];
}

// FP64 exact forces on target subsets (gravity.c:46-61 pair arithmetic).
constexpr int kRefThreads = 128;
__global__ void __launch_bounds__(kRefThreads) reference_subset_kernel(
    const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
    const double* __restrict__ m, long long n, const int64_t* __restrict__ targets, int count,
    double g, double eps2, long long chunk, double* __restrict__ partial) {
  __shared__ double4 tile[kRefThreads];
  const int t = blockIdx.x * kRefThreads + threadIdx.x;
  const long long i = t < count ? targets[t] : -1;
  const double xi = i >= 0 ? x[i] : 0.0, yi = i >= 0 ? y[i] : 0.0, zi = i >= 0 ? z[i] : 0.0;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  const long long j0 = blockIdx.y * chunk;
  const long long j1 = j0 + chunk < n ? j0 + chunk : n;
  for (long long jt = j0; jt < j1; jt += kRefThreads) {
    __syncthreads();
    const long long j = jt + threadIdx.x;
    tile[threadIdx.x] = j < j1 ? make_double4(x[j], y[j], z[j], m[j]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    const int jn = (int)(j1 - jt < kRefThreads ? j1 - jt : kRefThreads);
    for (int k = 0; k < jn; ++k) {
      if (jt + k == i) continue;
      const double4 q = tile[k];
      const double dx = __dsub_rn(q.x, xi), dy = __dsub_rn(q.y, yi), dz = __dsub_rn(q.z, zi);
      const double r2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                            __dmul_rn(dz, dz)),
                                  eps2);
      const double inv = __ddiv_rn(1.0, __dsqrt_rn(r2));
      const double inv3 = __dmul_rn(__dmul_rn(inv, inv), inv);
      const double s = __dmul_rn(__dmul_rn(g, q.w), inv3);
      sx = __dadd_rn(sx, __dmul_rn(s, dx));
      sy = __dadd_rn(sy, __dmul_rn(s, dy));
      sz = __dadd_rn(sz, __dmul_rn(s, dz));
    }
  }
  if (t < count) {
    const size_t base = ((size_t)blockIdx.y * count + t) * 3;
    partial[base + 0] = sx;
    partial[base + 1] = sy;
    partial[base + 2] = sz;
  }
}

// Sum chunk partials with Neumaier compensation in chunk order.
__global__ void reference_subset_final_kernel(const double* __restrict__ partial, int count,
                                              int chunks, double* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * count) return;
  double s = 0.0, c = 0.0;
  for (int k = 0; k < chunks; ++k) {
    const double v = partial[(size_t)k * 3 * count + e];
    const double t = __dadd_rn(s, v);
    if (fabs(s) >= fabs(v)) {
      c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, t), v));
    } else {
      c = __dadd_rn(c, __dadd_rn(__dsub_rn(v, t), s));
    }
    s = t;
  }
  out[e] = __dadd_rn(s, c);
}

__global__ void touch_kernel(uint4* buf, size_t words) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words;
       i += (size_t)gridDim.x * blockDim.x)
    buf[i] = make_uint4((unsigned)i, 1u, 2u, 3u);
}

int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

}  // namespace

extern "C" {

int nbsp_allpairs_shape_supported(NbspAllPairsShape shape) {
  return select_kernel(shape, false) != nullptr && shape.chunks >= 1;
}

int nbsp_allpairs_resident_ctas(NbspAllPairsShape shape) {
  ForceKernel k = select_kernel(shape, false);
  if (k == nullptr) return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, (const void*)k, shape.block, 0) !=
      cudaSuccess)
    return 0;
  return blocks;
}

void nbsp_pack_relative(const double* x, const double* y, const double* z, const double* m,
                        size_t n, size_t n_padded, const double* centre, void* packed, int* status,
                        cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), pack_kernel<<<grid_for(n_padded, 256), 256, 0, stream>>>(x, y, z, m, n, n_padded, centre,
                                                           (float4*)packed, status);
}

void nbsp_allpairs_force_targets(const void* sources, size_t n_sources_padded, const void* targets,
                                 size_t n_targets, float softening_squared,
                                 NbspAllPairsShape shape, void* partial_hi, void* partial_lo,
                                 cudaStream_t stream) {
  ForceKernel k = select_kernel(shape, softening_squared == 0.f);
  const int targets_per_cta = shape.block * shape.per_thread;
  const int chunk_len = (int)nbsp_allpairs_chunk_len(n_sources_padded, shape.chunks);
  dim3 grid((unsigned)((n_targets + targets_per_cta - 1) / targets_per_cta), (unsigned)shape.chunks);
  NBSP_COUNT_LAUNCH(1), k<<<grid, shape.block, 0, stream>>>(
      (const float4*)sources, (const float4*)targets, (int)n_targets, (int)n_sources_padded,
      chunk_len, softening_squared, (float4*)partial_hi, (float4*)partial_lo);
}

void nbsp_allpairs_force(const void* packed, size_t n, size_t n_padded, float softening_squared,
                         NbspAllPairsShape shape, void* partial_hi, void* partial_lo,
                         cudaStream_t stream) {
  nbsp_allpairs_force_targets(packed, n_padded, packed, n, softening_squared, shape, partial_hi,
                              partial_lo, stream);
}

void nbsp_allpairs_finalize(const void* partial_hi, const void* partial_lo, size_t n, int chunks,
                            double g, double* ax, double* ay, double* az, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), finalize_kernel<<<grid_for(n, 256), 256, 0, stream>>>(
      (const float4*)partial_hi, (const float4*)partial_lo, n, chunks, g, ax, ay, az);
}

void nbsp_kick_drift(double* x, double* y, double* z, double* vx, double* vy, double* vz,
                     const double* ax, const double* ay, const double* az, size_t n, double kick,
                     double drift, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), kick_drift_kernel<<<grid_for(n, 256), 256, 0, stream>>>(x, y, z, vx, vy, vz, ax, ay, az, n,
                                                          kick, drift);
}

void nbsp_euler_update(double* x, double* y, double* z, double* vx, double* vy, double* vz,
                       const double* ax, const double* ay, const double* az, size_t n, double dt,
                       cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), euler_kernel<<<grid_for(n, 256), 256, 0, stream>>>(x, y, z, vx, vy, vz, ax, ay, az, n, dt);
}

void nbsp_allpairs_finalize_kick(const void* partial_hi, const void* partial_lo, size_t n,
                                 int chunks, double g, double* ax, double* ay, double* az,
                                 double* vx, double* vy, double* vz, double half_dt,
                                 cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), finalize_kick_kernel<<<grid_for(n, 256), 256, 0, stream>>>(
      (const float4*)partial_hi, (const float4*)partial_lo, n, chunks, g, ax, ay, az, vx, vy, vz,
      half_dt);
}

void nbsp_allpairs_finalize_kick_kick_drift_pack(const void* partial_hi, const void* partial_lo,
                                                 size_t n, size_t n_padded, int chunks, double g,
                                                 double* x, double* y, double* z, double* vx,
                                                 double* vy, double* vz, double* ax, double* ay,
                                                 double* az, const double* m, double half_dt,
                                                 double dt, const double* centre, void* packed,
                                                 int* status, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), finalize_kick_kick_drift_pack_kernel<<<grid_for(n_padded, 256), 256, 0, stream>>>(
      (const float4*)partial_hi, (const float4*)partial_lo, n, n_padded, chunks, g, x, y, z, vx,
      vy, vz, ax, ay, az, m, half_dt, dt, centre, (float4*)packed, status);
}

void nbsp_global_sums(const double* x, const double* y, const double* z, const double* vx,
                      const double* vy, const double* vz, const double* m, size_t n,
                      double* scratch, double* out, cudaStream_t stream) {
  const int blocks = sum_blocks(n);
  NBSP_COUNT_LAUNCH(1), global_sums_kernel<<<blocks, kSumThreads, 0, stream>>>(x, y, z, vx, vy, vz, m, n, kQuantities,
                                                         scratch);
  NBSP_COUNT_LAUNCH(1), global_sums_final_kernel<<<1, kSumThreads, 0, stream>>>(scratch, blocks, out, 0);
}

void nbsp_centre_of_mass(const double* x, const double* y, const double* z, const double* m,
                         size_t n, double* scratch, double* centre, cudaStream_t stream) {
  const int blocks = sum_blocks(n);
  NBSP_COUNT_LAUNCH(1), global_sums_kernel<<<blocks, kSumThreads, 0, stream>>>(x, y, z, x, y, z, m, n, 1, scratch);
  NBSP_COUNT_LAUNCH(1), global_sums_final_kernel<<<1, kSumThreads, 0, stream>>>(scratch, blocks, centre, 1);
}

void nbsp_potential_energy(const double* x, const double* y, const double* z, const double* m,
                           size_t n, double g, double eps2, double* rows, double* out,
                           cudaStream_t stream) {
  const int blocks = (int)((n + kPeThreads - 1) / kPeThreads);
  if (blocks > 0)
    NBSP_COUNT_LAUNCH(1), potential_rows_kernel<<<blocks, kPeThreads, 0, stream>>>(x, y, z, m, (int)n, eps2, rows);
  NBSP_COUNT_LAUNCH(1), rows_sum_kernel<<<1, kSumThreads, 0, stream>>>(rows, n, -g, out);
}

void nbsp_reference_subset(const double* x, const double* y, const double* z, const double* m,
                           size_t n, const int64_t* targets, size_t count, double g, double eps2,
                           double* scratch, int chunks, double* out, cudaStream_t stream) {
  if (count == 0) return;
  const long long chunk = (long long)((n + chunks - 1) / chunks);
  dim3 grid((unsigned)((count + kRefThreads - 1) / kRefThreads), (unsigned)chunks);
  NBSP_COUNT_LAUNCH(1), reference_subset_kernel<<<grid, kRefThreads, 0, stream>>>(x, y, z, m, (long long)n, targets,
                                                            (int)count, g, eps2, chunk, scratch);
  NBSP_COUNT_LAUNCH(1), reference_subset_final_kernel<<<(unsigned)((3 * count + 255) / 256), 256, 0, stream>>>(
      scratch, (int)count, chunks, out);
}

void nbsp_touch(void* buffer, size_t bytes, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), touch_kernel<<<148 * 8, 256, 0, stream>>>((uint4*)buffer, bytes / 16);
}

}  // extern "C"
