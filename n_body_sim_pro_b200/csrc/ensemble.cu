// Ensembles of many small, independent systems in one persistent launch.
//
// Each system evolves under its own softened all-pairs gravity
// (src/c/physics/gravity.c:37-67 arithmetic, FP32 with compensated sums on
// positions relative to the system's FP64 centre of mass) with leapfrog KDK
// (src/c/physics/integrator.c:47-85, FP64 state).
//
// Scheduling: the host bundles systems of the same size class into work items
// (a CTA of BLOCK threads split into subgroups of G = BLOCK / systems-per-item
// threads, each subgroup owning one system of at most G * K particles) and
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

constexpr int kTile = 32;  // sources per compensated fold

template <int BLOCK, int K>
__global__ void __launch_bounds__(BLOCK, 1) ensemble_kernel(EnsembleArgs a) {
  extern __shared__ float4 sp[];  // BLOCK * K positions
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
    if (n > G * K) {  // the host sizes G so this cannot happen
      if (lane == 0) atomicOr(a.status, NBSP_DEVICE_ERROR_ENSEMBLE_LIMIT);
      n = G * K;
    }
    float4* pos = sp + sub * (G * K);
    const double cx = has ? a.centre[3 * sys] : 0.0;
    const double cy = has ? a.centre[3 * sys + 1] : 0.0;
    const double cz = has ? a.centre[3 * sys + 2] : 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int i = lane + k * G;
      if (i < n) {
        const long long p = off + i;
        pos[i] = make_float4((float)__dsub_rn(a.x[p], cx), (float)__dsub_rn(a.y[p], cy),
                             (float)__dsub_rn(a.z[p], cz), (float)a.m[p]);
      }
    }
    __syncthreads();
    for (int step = 0; step <= a.steps; ++step) {
      float xi[K], yi[K], zi[K], hx[K], hy[K], hz[K], lx[K], ly[K], lz[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int i = lane + k * G;
        const float4 q = i < n ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        xi[k] = q.x;
        yi[k] = q.y;
        zi[k] = q.z;
        hx[k] = hy[k] = hz[k] = lx[k] = ly[k] = lz[k] = 0.f;
      }
      for (int j0 = 0; j0 < n; j0 += kTile) {
        const int j1 = min(j0 + kTile, n);
        float px[K], py[K], pz[K];
#pragma unroll
        for (int k = 0; k < K; ++k) px[k] = py[k] = pz[k] = 0.f;
        for (int j = j0; j < j1; ++j) {
          const float4 s = pos[j];
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const float dx = s.x - xi[k], dy = s.y - yi[k], dz = s.z - zi[k];
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, a.eps2)));
            const float rinv = r2 > 0.f ? rsqrt_mufu(r2) : 0.f;  // self pair contributes 0
            const float wgt = s.w * (rinv * rinv * rinv);
            px[k] = fmaf(wgt, dx, px[k]);
            py[k] = fmaf(wgt, dy, py[k]);
            pz[k] = fmaf(wgt, dz, pz[k]);
          }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
          fold(hx[k], lx[k], px[k]);
          fold(hy[k], ly[k], py[k]);
          fold(hz[k], lz[k], pz[k]);
        }
      }
      float4 next[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int i = lane + k * G;
        next[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i >= n) continue;
        const long long p = off + i;
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
          next[k] = make_float4((float)__dsub_rn(nx, cx), (float)__dsub_rn(ny, cy),
                                (float)__dsub_rn(nz, cz), (float)a.m[p]);
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
          if (i < n) pos[i] = next[k];
        }
      }
      __syncthreads();
    }
  }
}

typedef void (*EnsembleKernel)(EnsembleArgs);

EnsembleKernel select(int block, int k) {
  if (block == 512 && k == 8) return ensemble_kernel<512, 8>;
  if (block == 1024 && k == 4) return ensemble_kernel<1024, 4>;
  if (block == 256 && k == 16) return ensemble_kernel<256, 16>;
  return nullptr;
}

}  // namespace

extern "C" {

int nbsp_ensemble_shape_supported(int block, int per_thread) {
  return select(block, per_thread) != nullptr;
}

int nbsp_ensemble_resident_ctas(int block, int per_thread) {
  EnsembleKernel k = select(block, per_thread);
  if (k == nullptr) return 0;
  const int smem = block * per_thread * 16;
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
                           int steps, cudaStream_t stream) {
  EnsembleKernel k = select(block, per_thread);
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
  const int smem = block * per_thread * 16;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  NBSP_COUNT_LAUNCH(1), k<<<grid, block, smem, stream>>>(a);
}

}  // extern "C"
