// Training of the far-field correction MLP on BF16 tensor cores.
//
// One train-step launch processes one minibatch: every CTA owns 128 rows
// (8 warps x 16 rows).  Forward and the activation gradients (dH2 = dY W3^T,
// dH1 = dZ2 W2^T) run on mma.sync m16n8k16 straight from register fragments;
// the weight gradients (dW = dZ^T H, a contraction over the 128 rows) run on
// mma.sync as well, from BF16 copies of the activations staged in shared
// memory.  Each CTA writes its gradient to its own slot; the Adam kernel sums
// the slots in a fixed order (deterministic), updates the FP32 master weights
// and a second kernel rebuilds the BF16 fragments.
//
// Loss: mean squared error over the 3 outputs of the standardised labels,
// L = 1 / (3 B) sum_r sum_c (y_rc - t_rc)^2.
#include "internal.h"
#include "mlp.cuh"
#include "mlp_umma.cuh"

#include <cuda_runtime.h>
#include <stdint.h>

using namespace nbsp_mlp;

namespace {

constexpr int kRows = 128;  // rows per CTA
constexpr int kWarps = kRows / 16;

struct TrainFrags {
  uint2 w1[kFragW1];
  uint2 w2[kFragW2];
  uint2 w3[kFragW3];
  uint2 w2t[kFragW2T];
  uint2 w3t[kFragW3T];
  float b1[kHidden], b2[kHidden], b3[kOutPad];
};

__device__ __forceinline__ unsigned short bf16_bits(float v) {
  const __nv_bfloat16 b = __float2bfloat16_rn(v);
  return *reinterpret_cast<const unsigned short*>(&b);
}

// A fragment of the transpose of a row-major [rows][cols] BF16 matrix M:
// A[i][k] = M[row0 + k][col0 + i]  (16 x 16 tile).
__device__ __forceinline__ void load_at(const unsigned short* m, int cols, int row0, int col0,
                                        int lane, uint32_t* a) {
  const int g = lane >> 2, t = lane & 3;
  auto pair = [&](int i, int k) -> uint32_t {
    const uint32_t lo = m[(row0 + k) * cols + col0 + i];
    const uint32_t hi = m[(row0 + k + 1) * cols + col0 + i];
    return lo | (hi << 16);
  };
  a[0] = pair(g, 2 * t);
  a[1] = pair(g + 8, 2 * t);
  a[2] = pair(g, 2 * t + 8);
  a[3] = pair(g + 8, 2 * t + 8);
}

// B fragment of a row-major [rows][cols] BF16 matrix N: B[k][n] = N[row0 + k][col0 + n].
__device__ __forceinline__ uint2 load_b(const unsigned short* m, int cols, int row0, int col0,
                                        int lane) {
  const int g = lane >> 2, t = lane & 3;
  const uint32_t b0 = (uint32_t)m[(row0 + 2 * t) * cols + col0 + g] |
                      ((uint32_t)m[(row0 + 2 * t + 1) * cols + col0 + g] << 16);
  const uint32_t b1 = (uint32_t)m[(row0 + 2 * t + 8) * cols + col0 + g] |
                      ((uint32_t)m[(row0 + 2 * t + 9) * cols + col0 + g] << 16);
  return make_uint2(b0, b1);
}

// Store a 16 x 8 C fragment (rows row0.., cols col0..) as BF16 into [rows][cols].
__device__ __forceinline__ void store_c(unsigned short* m, int cols, int row0, int col0, int lane,
                                        const float* c) {
  const int g = lane >> 2, t = lane & 3;
  m[(row0 + g) * cols + col0 + 2 * t] = bf16_bits(c[0]);
  m[(row0 + g) * cols + col0 + 2 * t + 1] = bf16_bits(c[1]);
  m[(row0 + g + 8) * cols + col0 + 2 * t] = bf16_bits(c[2]);
  m[(row0 + g + 8) * cols + col0 + 2 * t + 1] = bf16_bits(c[3]);
}

struct Stage {
  unsigned short x[kRows * kInPad];
  unsigned short h1[kRows * kHidden];
  unsigned short h2[kRows * kHidden];
  unsigned short dz1[kRows * kHidden];
  unsigned short dz2[kRows * kHidden];
  unsigned short dy[kRows * kOutPad];
  float db[kWarps][kHidden * 2 + kOutPad];
  float loss[kWarps];
};

// grad: [kParams] slot of this CTA.  rows_valid: rows of this CTA that exist.
__global__ void __launch_bounds__(kRows * 2) train_step_kernel(
    const uint32_t* __restrict__ x_bf16, const float* __restrict__ y, const int* __restrict__ order,
    int first_row, int rows_total, float inv_batch3, const TrainFrags* __restrict__ f,
    float* __restrict__ grad, float* __restrict__ loss_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Stage& st = *reinterpret_cast<Stage*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // rows of this warp: 16 consecutive rows of the CTA
  const int r0 = first_row + blockIdx.x * kRows + warp * 16 + g;
  const int r1 = r0 + 8;
  const bool v0 = r0 < rows_total, v1 = r1 < rows_total;
  const int s0 = v0 ? order[r0] : 0, s1 = v1 ? order[r1] : 0;

  if (warp < kWarps) {
    uint32_t xa[4];
    xa[0] = v0 ? x_bf16[s0 * 8 + t] : 0u;
    xa[1] = v1 ? x_bf16[s1 * 8 + t] : 0u;
    xa[2] = v0 ? x_bf16[s0 * 8 + t + 4] : 0u;
    xa[3] = v1 ? x_bf16[s1 * 8 + t + 4] : 0u;
    const int lr = warp * 16;  // local row base
    // stage X (BF16) for dW1
    {
      const uint32_t* xw = xa;
      unsigned int* xs = reinterpret_cast<unsigned int*>(st.x);
      xs[(lr + g) * 8 + t] = xw[0];
      xs[(lr + g + 8) * 8 + t] = xw[1];
      xs[(lr + g) * 8 + t + 4] = xw[2];
      xs[(lr + g + 8) * 8 + t + 4] = xw[3];
    }
    // forward, keeping pre-activations
    float z1[8][4], z2[8][4];
    uint32_t h1[16], h2[16];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(c, xa, f->w1[nt * 32 + lane]);
      const float bb0 = f->b1[8 * nt + 2 * t], bb1 = f->b1[8 * nt + 2 * t + 1];
      z1[nt][0] = c[0] + bb0;
      z1[nt][1] = c[1] + bb1;
      z1[nt][2] = c[2] + bb0;
      z1[nt][3] = c[3] + bb1;
      float a[4] = {gelu(z1[nt][0]), gelu(z1[nt][1]), gelu(z1[nt][2]), gelu(z1[nt][3])};
      store_c(st.h1, kHidden, lr, 8 * nt, lane, a);
      const int ks = nt >> 1, hi = (nt & 1) * 2;
      h1[4 * ks + hi] = pack_bf16(a[0], a[1]);
      h1[4 * ks + hi + 1] = pack_bf16(a[2], a[3]);
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) mma_bf16(c, &h1[4 * ks], f->w2[(ks * 8 + nt) * 32 + lane]);
      const float bb0 = f->b2[8 * nt + 2 * t], bb1 = f->b2[8 * nt + 2 * t + 1];
      z2[nt][0] = c[0] + bb0;
      z2[nt][1] = c[1] + bb1;
      z2[nt][2] = c[2] + bb0;
      z2[nt][3] = c[3] + bb1;
      float a[4] = {gelu(z2[nt][0]), gelu(z2[nt][1]), gelu(z2[nt][2]), gelu(z2[nt][3])};
      store_c(st.h2, kHidden, lr, 8 * nt, lane, a);
      const int ks = nt >> 1, hi = (nt & 1) * 2;
      h2[4 * ks + hi] = pack_bf16(a[0], a[1]);
      h2[4 * ks + hi + 1] = pack_bf16(a[2], a[3]);
    }
    float out[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) mma_bf16(out, &h2[4 * ks], f->w3[ks * 32 + lane]);
    // dY = 2 (y - t) / (3 B) on the 3 real outputs of valid rows
    float dy[4];
    float lsum = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int col = 2 * t + (q & 1);
      const bool row_ok = q < 2 ? v0 : v1;
      const int s = q < 2 ? s0 : s1;
      float d = 0.f;
      if (row_ok && col < kOut) {
        const float e = out[q] + f->b3[col] - y[s * 3 + col];
        lsum += e * e;
        d = 2.f * e * inv_batch3;
      }
      dy[q] = d;
    }
    store_c(st.dy, kOutPad, lr, 0, lane, dy);
    for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
    if (lane == 0) st.loss[warp] = lsum;
    // dH2 = dY W3^T  (K 16 with columns 8..15 zero)
    uint32_t dya[4] = {pack_bf16(dy[0], dy[1]), pack_bf16(dy[2], dy[3]), 0u, 0u};
    uint32_t dz2a[16];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(c, dya, f->w3t[nt * 32 + lane]);
      float d[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) d[q] = c[q] * gelu_grad(z2[nt][q]);
      store_c(st.dz2, kHidden, lr, 8 * nt, lane, d);
      const int ks = nt >> 1, hi = (nt & 1) * 2;
      dz2a[4 * ks + hi] = pack_bf16(d[0], d[1]);
      dz2a[4 * ks + hi + 1] = pack_bf16(d[2], d[3]);
    }
    // dH1 = dZ2 W2^T
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) mma_bf16(c, &dz2a[4 * ks], f->w2t[(ks * 8 + nt) * 32 + lane]);
      float d[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) d[q] = c[q] * gelu_grad(z1[nt][q]);
      store_c(st.dz1, kHidden, lr, 8 * nt, lane, d);
    }
  }
  __syncthreads();

  // bias gradients: column sums over the CTA's rows (threads 0..135)
  const int tid = threadIdx.x;
  if (tid < kHidden) {
    float s1 = 0.f, s2 = 0.f;
    for (int r = 0; r < kRows; ++r) {
      __nv_bfloat16 a = *reinterpret_cast<const __nv_bfloat16*>(&st.dz1[r * kHidden + tid]);
      __nv_bfloat16 b = *reinterpret_cast<const __nv_bfloat16*>(&st.dz2[r * kHidden + tid]);
      s1 += __bfloat162float(a);
      s2 += __bfloat162float(b);
    }
    grad[(size_t)blockIdx.x * kParams + kOffB1 + tid] = s1;
    grad[(size_t)blockIdx.x * kParams + kOffB2 + tid] = s2;
  } else if (tid < kHidden + kOut) {
    const int c = tid - kHidden;
    float s = 0.f;
    for (int r = 0; r < kRows; ++r)
      s += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(&st.dy[r * kOutPad + c]));
    grad[(size_t)blockIdx.x * kParams + kOffB3 + c] = s;
  } else if (tid == kHidden + kOut) {
    float s = 0.f;
    for (int w = 0; w < kWarps; ++w) s += st.loss[w];
    loss_out[blockIdx.x] = s;
  }

  // weight gradients on tensor cores: dW = dZ^T H over the 128 rows (8 k-steps)
  // output tiles: dW2 4 x 8 (32), dW1 4 x 2 (8), dW3 1 x 8 (8), shared by the CTA's warps
  const int nwarps = blockDim.x >> 5;
  for (int tile = warp; tile < 32 + 8 + 8; tile += nwarps) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    if (tile < 32) {  // dW2[out][in] = sum_r dZ2[r][out] H1[r][in]
      const int mi = tile >> 3, nj = tile & 7;
      for (int ks = 0; ks < kRows / 16; ++ks) {
        uint32_t a[4];
        load_at(st.dz2, kHidden, ks * 16, mi * 16, lane, a);
        mma_bf16(c, a, load_b(st.h1, kHidden, ks * 16, nj * 8, lane));
      }
      const int o0 = mi * 16 + g, i0 = nj * 8 + 2 * t;
      float* gw = grad + (size_t)blockIdx.x * kParams + kOffW2;
      gw[o0 * kHidden + i0] = c[0];
      gw[o0 * kHidden + i0 + 1] = c[1];
      gw[(o0 + 8) * kHidden + i0] = c[2];
      gw[(o0 + 8) * kHidden + i0 + 1] = c[3];
    } else if (tile < 40) {  // dW1[out][in] = sum_r dZ1[r][out] X[r][in], in < 10
      const int mi = (tile - 32) >> 1, nj = (tile - 32) & 1;
      for (int ks = 0; ks < kRows / 16; ++ks) {
        uint32_t a[4];
        load_at(st.dz1, kHidden, ks * 16, mi * 16, lane, a);
        mma_bf16(c, a, load_b(st.x, kInPad, ks * 16, nj * 8, lane));
      }
      const int o0 = mi * 16 + g, i0 = nj * 8 + 2 * t;
      float* gw = grad + (size_t)blockIdx.x * kParams + kOffW1;
      if (i0 < kIn) gw[o0 * kIn + i0] = c[0], gw[(o0 + 8) * kIn + i0] = c[2];
      if (i0 + 1 < kIn) gw[o0 * kIn + i0 + 1] = c[1], gw[(o0 + 8) * kIn + i0 + 1] = c[3];
    } else {  // dW3[out][in] = sum_r dY[r][out] H2[r][in], out < 3 (M 16 from 8 padded)
      const int nj = tile - 40;
      for (int ks = 0; ks < kRows / 16; ++ks) {
        uint32_t a[4];
        // A[i][k] = dY[k][i] for i < 8, zero for i >= 8
        const int gg = lane >> 2, tt = lane & 3;
        auto pair = [&](int i, int k) -> uint32_t {
          if (i >= kOutPad) return 0u;
          const uint32_t lo = st.dy[(ks * 16 + k) * kOutPad + i];
          const uint32_t hi = st.dy[(ks * 16 + k + 1) * kOutPad + i];
          return lo | (hi << 16);
        };
        a[0] = pair(gg, 2 * tt);
        a[1] = pair(gg + 8, 2 * tt);
        a[2] = pair(gg, 2 * tt + 8);
        a[3] = pair(gg + 8, 2 * tt + 8);
        mma_bf16(c, a, load_b(st.h2, kHidden, ks * 16, nj * 8, lane));
      }
      const int o0 = g, i0 = nj * 8 + 2 * t;
      float* gw = grad + (size_t)blockIdx.x * kParams + kOffW3;
      if (o0 < kOut) {
        gw[o0 * kHidden + i0] = c[0];
        gw[o0 * kHidden + i0 + 1] = c[1];
      }
    }
  }
}

// Sum the per-CTA gradient slots (fixed order) into grad_out; optional Adam.
__global__ void reduce_adam_kernel(const float* __restrict__ partial, int slots,
                                   float* __restrict__ grad_out, float* __restrict__ params,
                                   float* __restrict__ m, float* __restrict__ v, float lr,
                                   float beta1, float beta2, float eps, float bias1, float bias2,
                                   int apply) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  float gsum = 0.f;
  for (int s = 0; s < slots; ++s) gsum += partial[(size_t)s * kParams + p];
  if (grad_out != nullptr) grad_out[p] = gsum;
  if (!apply) return;
  const float mm = beta1 * m[p] + (1.f - beta1) * gsum;
  const float vv = beta2 * v[p] + (1.f - beta2) * gsum * gsum;
  m[p] = mm;
  v[p] = vv;
  params[p] -= lr * (mm / bias1) / (sqrtf(vv / bias2) + eps);
}

__device__ __forceinline__ float w_at(const float* w, int out, int in, int outs, int ins) {
  return (out < outs && in < ins) ? w[out * ins + in] : 0.f;
}

// B fragments of B[k][n] = W[n][k]  (forward: K = inputs, N = outputs)
__device__ void build_fwd(uint2* frag, const float* w, int outs, int ins, int ksteps, int ntiles) {
  for (int e = threadIdx.x; e < ksteps * ntiles * 32; e += blockDim.x) {
    const int lane = e & 31, tile = e >> 5;
    const int ks = tile / ntiles, nt = tile % ntiles;
    const int g = lane >> 2, t = lane & 3;
    const int n = nt * 8 + g, k = ks * 16 + 2 * t;
    frag[e] = make_uint2(pack_bf16(w_at(w, n, k, outs, ins), w_at(w, n, k + 1, outs, ins)),
                         pack_bf16(w_at(w, n, k + 8, outs, ins), w_at(w, n, k + 9, outs, ins)));
  }
}

// B fragments of B[k][n] = W[k][n]  (backward: K = outputs of the layer, N = inputs)
__device__ void build_bwd(uint2* frag, const float* w, int outs, int ins, int ksteps, int ntiles) {
  for (int e = threadIdx.x; e < ksteps * ntiles * 32; e += blockDim.x) {
    const int lane = e & 31, tile = e >> 5;
    const int ks = tile / ntiles, nt = tile % ntiles;
    const int g = lane >> 2, t = lane & 3;
    const int n = nt * 8 + g, k = ks * 16 + 2 * t;
    frag[e] = make_uint2(pack_bf16(w_at(w, k, n, outs, ins), w_at(w, k + 1, n, outs, ins)),
                         pack_bf16(w_at(w, k + 8, n, outs, ins), w_at(w, k + 9, n, outs, ins)));
  }
}

__global__ void build_frags_kernel(const float* __restrict__ params, TrainFrags* f, Net* net) {
  build_fwd(f->w1, params + kOffW1, kHidden, kIn, 1, 8);
  build_fwd(f->w2, params + kOffW2, kHidden, kHidden, 4, 8);
  build_fwd(f->w3, params + kOffW3, kOut, kHidden, 4, 1);
  build_bwd(f->w2t, params + kOffW2, kHidden, kHidden, 4, 8);
  build_bwd(f->w3t, params + kOffW3, kOut, kHidden, 1, 8);
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    f->b1[i] = params[kOffB1 + i];
    f->b2[i] = params[kOffB2 + i];
  }
  for (int i = threadIdx.x; i < kOutPad; i += blockDim.x) f->b3[i] = i < kOut ? params[kOffB3 + i] : 0.f;
  __syncthreads();
  if (net != nullptr) {
    for (int e = threadIdx.x; e < kFragW1; e += blockDim.x) net->w1[e] = f->w1[e];
    for (int e = threadIdx.x; e < kFragW2; e += blockDim.x) net->w2[e] = f->w2[e];
    for (int e = threadIdx.x; e < kFragW3; e += blockDim.x) net->w3[e] = f->w3[e];
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
      net->b1[i] = f->b1[i];
      net->b2[i] = f->b2[i];
    }
    for (int i = threadIdx.x; i < kOutPad; i += blockDim.x) net->b3[i] = f->b3[i];
    nbsp_umma::build_weights(params, reinterpret_cast<nbsp_umma::Weights*>(net->umma_w));
  }
}

// The network on raw feature rows (10 per row): standardised, through the
// three layers, de-standardised into out (3 per row).  tcgen05 path: one
// 128-row tile per iteration of a persistent CTA.
__global__ void __launch_bounds__(nbsp_umma::kThreads) evaluate_umma_kernel(
    const Net* __restrict__ net, const float* __restrict__ feat, int rows,
    float* __restrict__ out, int* status) {
  extern __shared__ __align__(128) unsigned char umma_smem[];
  nbsp_umma::Smem& s = *reinterpret_cast<nbsp_umma::Smem*>(umma_smem);
  nbsp_umma::setup(s, nbsp_umma::weights_of(net), net);
  const uint32_t tmem = s.tmem;
  uint32_t phase = 0;
  const int tiles = (rows + nbsp_umma::kRows - 1) / nbsp_umma::kRows;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int r = tile * nbsp_umma::kRows + threadIdx.x;
    float v[kIn];
#pragma unroll
    for (int q = 0; q < kIn; ++q)
      v[q] = r < rows ? (feat[(size_t)r * kIn + q] - net->x_mean[q]) * net->x_inv_std[q] : 0.f;
    nbsp_umma::put_inputs(s, v);
    nbsp_umma::fence_async_smem();
    __syncthreads();
    float y[3];
    if (!nbsp_umma::forward(s, tmem, phase, y)) {
      if (threadIdx.x == 0) atomicOr(status, NBSP_DEVICE_ERROR_MMA_TIMEOUT);
      break;
    }
    if (r < rows)
      for (int c = 0; c < kOut; ++c)
        out[(size_t)r * kOut + c] = fmaf(y[c], net->y_std[c], net->y_mean[c]);
  }
  nbsp_umma::teardown(s, tmem);
}

// The same with mma.sync: one warp per 16 rows (the corrected walk's former
// per-warp path, kept as the cross-check of the tcgen05 one).
__global__ void evaluate_sync_kernel(const Net* __restrict__ net, const float* __restrict__ feat,
                                     int rows, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int tile = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (tile * 16 >= rows) return;
  const int g = lane >> 2, t = lane & 3;
  auto val = [&](int row, int q) -> float {
    const int r = tile * 16 + row;
    return (r < rows && q < kIn) ? (feat[(size_t)r * kIn + q] - net->x_mean[q]) * net->x_inv_std[q]
                                 : 0.f;
  };
  const uint32_t x[4] = {pack_bf16(val(g, 2 * t), val(g, 2 * t + 1)),
                         pack_bf16(val(g + 8, 2 * t), val(g + 8, 2 * t + 1)),
                         pack_bf16(val(g, 2 * t + 8), val(g, 2 * t + 9)),
                         pack_bf16(val(g + 8, 2 * t + 8), val(g + 8, 2 * t + 9))};
  float o[4];
  forward_tile(x, net->w1, net->b1, net->w2, net->b2, net->w3, net->b3, lane, o);
  // o: C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]; outputs are columns 0..2
  for (int h = 0; h < 2; ++h) {
    const int r = tile * 16 + g + 8 * h;
    for (int k = 0; k < 2; ++k) {
      const int c = 2 * t + k;
      if (r < rows && c < kOut) out[(size_t)r * kOut + c] = fmaf(o[2 * h + k], net->y_std[c], net->y_mean[c]);
    }
  }
}

// Standardise raw features / labels into the training layout.
__global__ void standardise_kernel(const float* __restrict__ feat, const float* __restrict__ lab,
                                   int rows, const Net* __restrict__ net, uint32_t* __restrict__ x,
                                   float* __restrict__ y) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  float v[kInPad];
  for (int i = 0; i < kInPad; ++i)
    v[i] = i < kIn ? (feat[r * kIn + i] - net->x_mean[i]) * net->x_inv_std[i] : 0.f;
  for (int w = 0; w < 8; ++w) x[r * 8 + w] = pack_bf16(v[2 * w], v[2 * w + 1]);
  for (int c = 0; c < kOut; ++c) y[r * 3 + c] = (lab[r * 3 + c] - net->y_mean[c]) / net->y_std[c];
}

}  // namespace

extern "C" {

size_t nbsp_mlp_net_bytes(void) { return sizeof(Net); }

// Scaling table: x_mean[10], x_inv_std[10], x_min[10], x_max[10], y_mean[3], y_std[3],
// contiguous in Net from x_mean on.
static_assert(offsetof(Net, y_std) + sizeof(float) * kOut - offsetof(Net, x_mean) ==
                  sizeof(float) * 46, "scaling table layout");

void nbsp_mlp_set_scaling(void* net, const float* table, cudaStream_t stream) {
  cudaMemcpyAsync(static_cast<char*>(net) + offsetof(Net, x_mean), table, 46 * sizeof(float),
                  cudaMemcpyDeviceToDevice, stream);
}

void nbsp_mlp_get_scaling(const void* net, float* table, cudaStream_t stream) {
  cudaMemcpyAsync(table, static_cast<const char*>(net) + offsetof(Net, x_mean), 46 * sizeof(float),
                  cudaMemcpyDeviceToDevice, stream);
}
size_t nbsp_mlp_frags_bytes(void) { return sizeof(TrainFrags); }
int nbsp_mlp_param_count(void) { return kParams; }
int nbsp_mlp_rows_per_cta(void) { return kRows; }

void nbsp_mlp_build_frags(const float* params, void* frags, void* net, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), build_frags_kernel<<<1, 256, 0, stream>>>(params, (TrainFrags*)frags,
                                                                   (Net*)net);
}

void nbsp_mlp_standardise(const float* feat, const float* lab, int rows, const void* net,
                          uint32_t* x, float* y, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), standardise_kernel<<<(rows + 255) / 256, 256, 0, stream>>>(
      feat, lab, rows, (const Net*)net, x, y);
}

// One forward/backward over rows [first_row, first_row + ctas * 128) of `order`;
// per-CTA gradients into partial[ctas][params], per-CTA loss sums into loss.
void nbsp_mlp_train_step(const uint32_t* x, const float* y, const int* order, int first_row,
                         int rows_total, int ctas, float inv_batch3, const void* frags,
                         float* partial, float* loss, cudaStream_t stream) {
  const int smem = (int)sizeof(Stage);
  cudaFuncSetAttribute(train_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  NBSP_COUNT_LAUNCH(1), train_step_kernel<<<ctas, kRows * 2, smem, stream>>>(
      x, y, order, first_row, rows_total, inv_batch3, (const TrainFrags*)frags, partial, loss);
}

void nbsp_mlp_evaluate(const void* net, const float* feat, int rows, float* out, int tcgen05,
                       int* status, cudaStream_t stream) {
  if (rows <= 0) return;
  if (tcgen05) {
    const int smem = (int)sizeof(nbsp_umma::Smem);
    cudaFuncSetAttribute(evaluate_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int tiles = (rows + nbsp_umma::kRows - 1) / nbsp_umma::kRows;
    const int cap = 148 * nbsp_umma::kCtasPerSm;
    const int grid = tiles < cap ? tiles : cap;
    NBSP_COUNT_LAUNCH(1), evaluate_umma_kernel<<<grid, nbsp_umma::kThreads, smem, stream>>>(
        (const Net*)net, feat, rows, out, status);
  } else {
    const int warps = (rows + 15) / 16;
    NBSP_COUNT_LAUNCH(1), evaluate_sync_kernel<<<(warps + 3) / 4, 128, 0, stream>>>(
        (const Net*)net, feat, rows, out);
  }
}

void nbsp_mlp_reduce_adam(const float* partial, int slots, float* grad_out, float* params, float* m,
                          float* v, float lr, int step, int apply, cudaStream_t stream) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float bias1 = 1.f - powf(b1, (float)step), bias2 = 1.f - powf(b2, (float)step);
  NBSP_COUNT_LAUNCH(1), reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, stream>>>(
      partial, slots, grad_out, params, m, v, lr, b1, b2, 1e-8f, bias1, bias2, apply);
}

}  // extern "C"
