// FP32 / SFU throughput probe: the measured denominators of the FP32 roofline.
//
// Three kernels of independent dependency chains, one resident wave sized from
// the occupancy API: scalar FFMA (fma.rn.f32), paired FFMA (fma.rn.f32x2,
// sm_100), and MUFU reciprocal square root (rsqrt.approx.ftz.f32).  Each is
// timed with CUDA events on the caller's stream after one warm-up launch.
#include "internal.h"
#include "n_body_sim_pro_cuda.h"

#include <cuda_runtime.h>
#include <stdio.h>

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) ffma_kernel(float* out, float a, float b, int iters) {
  float acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = (float)(threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = fmaf(acc[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  if (s == 123.456f) out[threadIdx.x] = s;  // keeps the chains alive
}

__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}

__global__ void __launch_bounds__(kThreads) ffma2_kernel(float* out, float a, float b, int iters) {
  unsigned long long acc[kChains];
  const unsigned long long aa = pack2(a, a), bb = pack2(b, b);
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = pack2((float)(threadIdx.x + c), (float)c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c)
      asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(acc[c]) : "l"(aa), "l"(bb));
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(acc[c]));
    s += lo + hi;
  }
  if (s == 123.456f) out[threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) rsqrt_kernel(float* out, int iters) {
  float acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = 1.0f + (float)(threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      float r;
      asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(acc[c]));
      acc[c] = r;
    }
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  if (s == 123.456f) out[threadIdx.x] = s;
}

}  // namespace

extern "C" N_BODY_SIM_PRO_CUDA_API NBodySimProStatus n_body_sim_pro_cuda_measure_fp32_peak(
    double* ffma_tflops, double* ffma2_tflops, double* rsqrt_per_second, double* sm_clock_mhz,
    NBodySimProError* error) {
  int device = 0, sms = 0, clock_khz = 0;
  cudaError_t code = cudaGetDevice(&device);
  if (code == cudaSuccess) code = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (code == cudaSuccess) code = cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, device);
  float* out = nullptr;
  if (code == cudaSuccess) code = cudaMalloc(&out, kThreads * sizeof(float));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (code == cudaSuccess) code = cudaEventCreate(&e0);
  if (code == cudaSuccess) code = cudaEventCreate(&e1);
  double results[3] = {0.0, 0.0, 0.0};
  const int iters = 1 << 16;
  for (int which = 0; which < 3 && code == cudaSuccess; ++which) {
    const void* fn = which == 0 ? (const void*)ffma_kernel
                     : which == 1 ? (const void*)ffma2_kernel : (const void*)rsqrt_kernel;
    int per_sm = 0;
    code = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0);
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    float ms = 0.f;
    for (int rep = 0; rep < 2 && code == cudaSuccess; ++rep) {
      cudaEventRecord(e0);
      if (which == 0) {
        NBSP_COUNT_LAUNCH(1), ffma_kernel<<<grid, kThreads>>>(out, 0.999f, 0.001f, iters);
      } else if (which == 1) {
        NBSP_COUNT_LAUNCH(1), ffma2_kernel<<<grid, kThreads>>>(out, 0.999f, 0.001f, iters);
      } else {
        NBSP_COUNT_LAUNCH(1), rsqrt_kernel<<<grid, kThreads>>>(out, iters / 16);
      }
      cudaEventRecord(e1);
      code = cudaEventSynchronize(e1);
      if (code == cudaSuccess) code = cudaGetLastError();
      cudaEventElapsedTime(&ms, e0, e1);
    }
    const double threads = (double)grid * kThreads;
    if (which == 0) results[0] = 2.0 * kChains * (double)iters * threads / (ms * 1e-3) / 1e12;
    if (which == 1) results[1] = 4.0 * kChains * (double)iters * threads / (ms * 1e-3) / 1e12;
    if (which == 2) results[2] = (double)kChains * (double)(iters / 16) * threads / (ms * 1e-3);
  }
  if (e0 != nullptr) cudaEventDestroy(e0);
  if (e1 != nullptr) cudaEventDestroy(e1);
  cudaFree(out);
  if (code != cudaSuccess) {
    if (error != nullptr) {
      error->status = N_BODY_SIM_PRO_STATUS_INVALID_STATE;
      error->source_file = __FILE__;
      error->source_line = __LINE__;
      snprintf(error->message, sizeof(error->message), "peak probe: %s", cudaGetErrorString(code));
    }
    return N_BODY_SIM_PRO_STATUS_INVALID_STATE;
  }
  if (ffma_tflops != nullptr) *ffma_tflops = results[0];
  if (ffma2_tflops != nullptr) *ffma2_tflops = results[1];
  if (rsqrt_per_second != nullptr) *rsqrt_per_second = results[2];
  if (sm_clock_mhz != nullptr) *sm_clock_mhz = clock_khz / 1000.0;
  return N_BODY_SIM_PRO_STATUS_OK;
}
