// Ensembles of many small, independent systems in one persistent launch.
//
// Each system evolves under its own softened all-pairs gravity
// (src/c/physics/gravity.c:37-67 arithmetic, FP32 with compensated sums on
// positions relative to the system's FP64 centre of mass) with leapfrog KDK
// (src/c/physics/integrator.c:47-85, FP64 state).
//
// Scheduling: the host bundles systems of the same size class into work items
// (a CTA of BLOCK threads split into subgroups of G threads — whole warps, or a
// power of two below one warp — each subgroup owning one system of at most
// G * K particles; threads past the last subgroup idle through the item) and
// orders the items by cost (sum of n^2), largest first.  The grid is one
// resident wave (SMs x CTAs-per-SM); each CTA takes the next item from an
// atomic counter and runs ALL the requested steps of its systems before it
// takes another, so no grid-wide synchronisation is ever needed: per step the
// CTA only needs __syncthreads between the force phase (all threads read the
// shared-memory positions) and the position update.
#include "internal.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace {

__device__ __forceinline__ float rsqrt_mufu(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Paired FP32 (sm_100 .f32x2): two targets share every add / mul / fma.
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

__device__ __forceinline__ void fold(float& hi, float& lo, float a) {
  const float s = __fadd_rn(hi, a);
  const float bp = __fsub_rn(s, hi);
  const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(a, bp));
  hi = s;
  lo = __fadd_rn(lo, err);
}

struct EnsembleArgs {
  double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
  const double* m;
  const long long* offset;  // [systems + 1]
  const double* centre;     // [systems * 3]
  const int* item_start;    // [items + 1] into item_systems
  const int* item_systems;
  const int* item_group;    // threads per system in the item
  int items;
  int* counter;
  int* status;
  double g, h, dt;
  float eps2;
  int steps;
};

constexpr int kTile = 64;         // sources per compensated fold
constexpr float kFarAway = 1e30f;  // padding sources: r^2 overflows to inf, rsqrt(inf) = 0

// GUARD: drop r^2 = 0 terms (eps = 0, or m / eps^3 could overflow); otherwise
// a target's own entry has d = 0 and adds W * 0 = 0.
template <int BLOCK, int K, bool GUARD>
__global__ void __launch_bounds__(BLOCK, 1) ensemble_kernel(EnsembleArgs a) {
  static_assert(K % 2 == 0, "targets are processed in pairs");
  constexpr int P = K / 2;
  // BLOCK * K particles, each as two float4 (x, x, y, y), (z, z, m, m): one
  // 16-byte load yields the broadcast operands of two paired instructions
  extern __shared__ float4 sp[];
  __shared__ int s_item;
  const int tid = threadIdx.x;
  for (int guard = 0;; ++guard) {
    if (guard > a.items) {  // each CTA takes each item at most once
      if (tid == 0) atomicOr(a.status, NBSP_DEVICE_ERROR_ENSEMBLE_LIMIT);
      break;
    }
    __syncthreads();
    if (tid == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int w = s_item;
    if (w >= a.items) break;
    const int G = a.item_group[w];
    const int first = a.item_start[w];
    const int count = a.item_start[w + 1] - first;
    const int sub = tid / G, lane = tid % G;
    const bool has = sub < count;
    const int sys = has ? a.item_systems[first + sub] : 0;
    const long long off = has ? a.offset[sys] : 0;
    int n = has ? (int)(a.offset[sys + 1] - off) : 0;
    if ((n + kTile - 1) / kTile * kTile > G * K) {  // the host sizes G so this cannot happen
      if (lane == 0) atomicOr(a.status, NBSP_DEVICE_ERROR_ENSEMBLE_LIMIT);
      n = 0;  // the padded system would not fit its shared-memory slots: skip it
    }
    float4* pos = sp + 2 * sub * (G * K);  // particle i at pos[2 i], pos[2 i + 1]
    const double cx = has ? a.centre[3 * sys] : 0.0;
    const double cy = has ? a.centre[3 * sys + 1] : 0.0;
    const double cz = has ? a.centre[3 * sys + 2] : 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int i = lane + k * G;
      if (i < n) {
        const long long p = off + i;
        const float px = (float)__dsub_rn(a.x[p], cx), py = (float)__dsub_rn(a.y[p], cy);
        const float pz = (float)__dsub_rn(a.z[p], cz), pm = (float)a.m[p];
        pos[2 * i] = make_float4(px, px, py, py);
        pos[2 * i + 1] = make_float4(pz, pz, pm, pm);
      }
    }
    // pad the system to whole tiles with massless far sources (fixed-count loops)
    const int n_pad = (n + kTile - 1) / kTile * kTile;  // <= G * K (checked above)
    for (int i = n + lane; i < n_pad; i += G) {
      pos[2 * i] = make_float4(kFarAway, kFarAway, kFarAway, kFarAway);
      pos[2 * i + 1] = make_float4(kFarAway, kFarAway, 0.f, 0.f);
    }
    __syncthreads();
    const unsigned long long E2 = pack2(a.eps2, a.eps2);
    for (int step = 0; step <= a.steps; ++step) {
      unsigned long long X[P], Y[P], Z[P];
      float hx[K], hy[K], hz[K], lx[K], ly[K], lz[K];
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const int i0 = lane + (2 * q) * G, i1 = lane + (2 * q + 1) * G;
        const float4 u0 = i0 < n ? pos[2 * i0] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 u1 = i0 < n ? pos[2 * i0 + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 v0 = i1 < n ? pos[2 * i1] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 v1 = i1 < n ? pos[2 * i1 + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
        X[q] = pack2(u0.x, v0.x);
        Y[q] = pack2(u0.z, v0.z);
        Z[q] = pack2(u1.x, v1.x);
      }
#pragma unroll
      for (int k = 0; k < K; ++k) hx[k] = hy[k] = hz[k] = lx[k] = ly[k] = lz[k] = 0.f;
      for (int j0 = 0; j0 < n_pad; j0 += kTile) {
        unsigned long long AX[P], AY[P], AZ[P];
#pragma unroll
        for (int q = 0; q < P; ++q) AX[q] = AY[q] = AZ[q] = 0ull;
#pragma unroll 8
        for (int j = 0; j < kTile; ++j) {
          const ulonglong2 s0 = reinterpret_cast<const ulonglong2*>(pos)[2 * (j0 + j)];
          const ulonglong2 s1 = reinterpret_cast<const ulonglong2*>(pos)[2 * (j0 + j) + 1];
          const unsigned long long SX = s0.x, SY = s0.y, SZ = s1.x, SW = s1.y;
#pragma unroll
          for (int q = 0; q < P; ++q) {
            const unsigned long long dx = sub2(SX, X[q]), dy = sub2(SY, Y[q]), dz = sub2(SZ, Z[q]);
            const unsigned long long r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
            float r2a, r2b;
            unpack2(r2, r2a, r2b);
            float ra = rsqrt_mufu(r2a), rb = rsqrt_mufu(r2b);
            if (GUARD) {  // the self pair (r^2 = 0 when eps = 0) contributes 0
              ra = r2a > 0.f ? ra : 0.f;
              rb = r2b > 0.f ? rb : 0.f;
            }
            const unsigned long long R = pack2(ra, rb);
            const unsigned long long W = mul2(SW, mul2(mul2(R, R), R));
            AX[q] = fma2(W, dx, AX[q]);
            AY[q] = fma2(W, dy, AY[q]);
            AZ[q] = fma2(W, dz, AZ[q]);
          }
        }
#pragma unroll
        for (int q = 0; q < P; ++q) {
          float u, v;
          unpack2(AX[q], u, v);
          fold(hx[2 * q], lx[2 * q], u);
          fold(hx[2 * q + 1], lx[2 * q + 1], v);
          unpack2(AY[q], u, v);
          fold(hy[2 * q], ly[2 * q], u);
          fold(hy[2 * q + 1], ly[2 * q + 1], v);
          unpack2(AZ[q], u, v);
          fold(hz[2 * q], lz[2 * q], u);
          fold(hz[2 * q + 1], lz[2 * q + 1], v);
        }
      }
      // the FP64 origin and offset are reloaded here (L1 hits) rather than held
      // in registers through the force loop
      const long long off_e = has ? a.offset[sys] : 0;
      const double cxe = has ? a.centre[3 * sys] : 0.0;
      const double cye = has ? a.centre[3 * sys + 1] : 0.0;
      const double cze = has ? a.centre[3 * sys + 2] : 0.0;
      float4 next[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int i = lane + k * G;
        next[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i >= n) continue;
        const long long p = off_e + i;
        const double a0 = a.g * ((double)hx[k] + (double)lx[k]);
        const double a1 = a.g * ((double)hy[k] + (double)ly[k]);
        const double a2 = a.g * ((double)hz[k] + (double)lz[k]);
        a.ax[p] = a0;
        a.ay[p] = a1;
        a.az[p] = a2;
        double u = a.vx[p], v = a.vy[p], wv = a.vz[p];
        if (step > 0) {  // closing half kick of step `step`
          u = __dadd_rn(u, __dmul_rn(a0, a.h));
          v = __dadd_rn(v, __dmul_rn(a1, a.h));
          wv = __dadd_rn(wv, __dmul_rn(a2, a.h));
        }
        if (step < a.steps) {  // opening half kick + drift of step `step + 1`
          u = __dadd_rn(u, __dmul_rn(a0, a.h));
          v = __dadd_rn(v, __dmul_rn(a1, a.h));
          wv = __dadd_rn(wv, __dmul_rn(a2, a.h));
          const double nx = __dadd_rn(a.x[p], __dmul_rn(u, a.dt));
          const double ny = __dadd_rn(a.y[p], __dmul_rn(v, a.dt));
          const double nz = __dadd_rn(a.z[p], __dmul_rn(wv, a.dt));
          a.x[p] = nx;
          a.y[p] = ny;
          a.z[p] = nz;
          next[k] = make_float4((float)__dsub_rn(nx, cxe), (float)__dsub_rn(ny, cye),
                                (float)__dsub_rn(nz, cze), (float)a.m[p]);
        }
        a.vx[p] = u;
        a.vy[p] = v;
        a.vz[p] = wv;
      }
      __syncthreads();  // every thread is done reading this step's positions
      if (step < a.steps) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int i = lane + k * G;
          if (i < n) {
            pos[2 * i] = make_float4(next[k].x, next[k].x, next[k].y, next[k].y);
            pos[2 * i + 1] = make_float4(next[k].z, next[k].z, next[k].w, next[k].w);
          }
        }
      }
      __syncthreads();
    }
  }
}

typedef void (*EnsembleKernel)(EnsembleArgs);

EnsembleKernel select(int block, int k, bool guard) {
  if (block == 512 && k == 8) return guard ? ensemble_kernel<512, 8, true> : ensemble_kernel<512, 8, false>;
  if (block == 1024 && k == 4) return guard ? ensemble_kernel<1024, 4, true> : ensemble_kernel<1024, 4, false>;
  if (block == 256 && k == 16) return guard ? ensemble_kernel<256, 16, true> : ensemble_kernel<256, 16, false>;
  return nullptr;
}

}  // namespace

extern "C" {

int nbsp_ensemble_shape_supported(int block, int per_thread) {
  return select(block, per_thread, false) != nullptr;
}

int nbsp_ensemble_resident_ctas(int block, int per_thread) {
  EnsembleKernel k = select(block, per_thread, true);
  if (k == nullptr) return 0;
  const int smem = block * per_thread * 32;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int ctas = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, k, block, smem) != cudaSuccess) return 0;
  return ctas;
}

void nbsp_ensemble_advance(int block, int per_thread, int grid, double* x, double* y, double* z,
                           double* vx, double* vy, double* vz, double* ax, double* ay, double* az,
                           const double* m, const long long* offset, const double* centre,
                           const int* item_start, const int* item_systems, const int* item_group,
                           int items, int* counter, int* status, double g, float eps2, double dt,
                           int steps, int guard, cudaStream_t stream) {
  EnsembleKernel k = select(block, per_thread, guard != 0);
  if (k == nullptr) return;
  EnsembleArgs a;
  a.x = x;
  a.y = y;
  a.z = z;
  a.vx = vx;
  a.vy = vy;
  a.vz = vz;
  a.ax = ax;
  a.ay = ay;
  a.az = az;
  a.m = m;
  a.offset = offset;
  a.centre = centre;
  a.item_start = item_start;
  a.item_systems = item_systems;
  a.item_group = item_group;
  a.items = items;
  a.counter = counter;
  a.status = status;
  a.g = g;
  a.h = 0.5 * dt;
  a.dt = dt;
  a.eps2 = eps2;
  a.steps = steps;
  const int smem = block * per_thread * 32;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  NBSP_COUNT_LAUNCH(1), k<<<grid, block, smem, stream>>>(a);
}

}  // extern "C"
