// Small MLP (10 -> 64 -> 64 -> 3, GELU) on BF16 tensor cores: shared device code
// of the training kernels (mlp.cu) and of the corrected Barnes-Hut walk (bh.cu).
//
// Matrix products use mma.sync.m16n8k16 (BF16 inputs, FP32 accumulate).  Fragment
// layouts (PTX ISA, "Matrix fragments for mma.m16n8k16"), with g = lane / 4 and
// t = lane % 4:
//   A 16x16 row-major : r0 = A[g][2t..2t+1]    r1 = A[g+8][2t..2t+1]
//                       r2 = A[g][2t+8..2t+9]  r3 = A[g+8][2t+8..2t+9]
//   B 16x8 col-major  : r0 = B[2t..2t+1][g]    r1 = B[2t+8..2t+9][g]
//   C 16x8 FP32       : c0,c1 = C[g][2t..2t+1] c2,c3 = C[g+8][2t..2t+1]
// so the C fragments of output n-tiles 2k and 2k+1 are exactly the A fragment
// of k-step k of the next layer (no data movement between layers).
//
// Weights are kept as ready-made B fragments: for every (k-step, n-tile) pair,
// 32 lanes x 2 registers (uint2), so a lane fetches its B fragment with one
// 64-bit load.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace nbsp_mlp {

constexpr int kIn = 10;      // features
constexpr int kInPad = 16;   // K of the first product
constexpr int kHidden = 64;
constexpr int kOut = 3;
constexpr int kOutPad = 8;   // N of the last product

// Flat FP32 parameter vector (row-major, out x in):
//   W1[64][10], b1[64], W2[64][64], b2[64], W3[3][64], b3[3]
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kIn;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kOut * kHidden;
constexpr int kParams = kOffB3 + kOut;  // 5059

// B-fragment arrays (uint2 per lane per (k-step, n-tile)).
constexpr int kFragW1 = 1 * 8 * 32;   // K 16, N 64
constexpr int kFragW2 = 4 * 8 * 32;   // K 64, N 64
constexpr int kFragW3 = 4 * 1 * 32;   // K 64, N 8
constexpr int kFragW2T = 4 * 8 * 32;  // backward: dH1 = dZ2 W2^T (K 64, N 64)
constexpr int kFragW3T = 1 * 8 * 32;  // backward: dH2 = dY W3^T  (K 8 -> 16, N 64)

// Device-resident network: fragments + biases + feature/label scaling + the
// feature range seen in training (inference outside it is skipped).
struct Net {
  uint2 w1[kFragW1];
  uint2 w2[kFragW2];
  uint2 w3[kFragW3];
  float b1[kHidden];
  float b2[kHidden];
  float b3[kOutPad];
  float x_mean[kIn], x_inv_std[kIn], x_min[kIn], x_max[kIn];
  float y_mean[kOut], y_std[kOut];
  // the same weights as BF16 operand images of the tcgen05 products
  // (nbsp_umma::Weights, mlp_umma.cuh): W1 64 x 16, W2 64 x 64, W3 16 x 64
  uint4 umma_w[(64 * 16 + 64 * 64 + 16 * 64) / 8];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

__device__ __forceinline__ float tanh_hw(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))  (Hendrycks & Gimpel).
constexpr float kGeluC = 0.7978845608028654f;
constexpr float kGeluA = 0.044715f;

__device__ __forceinline__ float gelu(float x) {
  const float u = kGeluC * fmaf(kGeluA * x * x, x, x);
  return 0.5f * x * (1.f + tanh_hw(u));
}

// Paired FP32 (sm_100 .f32x2): two activations per add / mul / fma.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// gelu() of (z0 + b0, z1 + b1) with the same roundings in the same order, two
// lanes per instruction, packed to BF16 for the next product.
__device__ __forceinline__ uint32_t gelu2_bf16(float z0, float z1, float b0, float b1) {
  const unsigned long long x = f2_add(f2_pack(z0, z1), f2_pack(b0, b1));
  const unsigned long long ka = f2_pack(kGeluA, kGeluA), kc = f2_pack(kGeluC, kGeluC);
  const unsigned long long u = f2_mul(kc, f2_fma(f2_mul(f2_mul(ka, x), x), x, x));
  float u0, u1;
  f2_unpack(u, u0, u1);
  const unsigned long long one_th = f2_add(f2_pack(1.f, 1.f), f2_pack(tanh_hw(u0), tanh_hw(u1)));
  float g0, g1;
  f2_unpack(f2_mul(f2_mul(f2_pack(0.5f, 0.5f), x), one_th), g0, g1);
  return pack_bf16(g0, g1);
}

// d gelu / dx
__device__ __forceinline__ float gelu_grad(float x) {
  const float u = kGeluC * fmaf(kGeluA * x * x, x, x);
  const float th = tanh_hw(u);
  const float du = kGeluC * fmaf(3.f * kGeluA, x * x, 1.f);
  return 0.5f * (1.f + th) + 0.5f * x * (1.f - th * th) * du;
}

// Forward pass of one 16-row tile held as an A fragment (x: 16 x 16 BF16,
// features already standardised).  Returns the 16 x 8 output C fragment (cols
// 0..2 used).  w* point to fragment arrays (shared or global memory).
__device__ __forceinline__ void forward_tile(const uint32_t* x, const uint2* w1, const float* b1,
                                             const uint2* w2, const float* b2, const uint2* w3,
                                             const float* b3, int lane, float* out) {
  const int t = lane & 3;
  uint32_t h1[16];  // A fragments of 4 k-steps of layer 2
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    mma_bf16(c, x, w1[nt * 32 + lane]);
    const float bb0 = b1[8 * nt + 2 * t], bb1 = b1[8 * nt + 2 * t + 1];
    const uint32_t top = gelu2_bf16(c[0], c[1], bb0, bb1);
    const uint32_t bot = gelu2_bf16(c[2], c[3], bb0, bb1);
    const int ks = nt >> 1;
    if ((nt & 1) == 0) {
      h1[4 * ks + 0] = top;
      h1[4 * ks + 1] = bot;
    } else {
      h1[4 * ks + 2] = top;
      h1[4 * ks + 3] = bot;
    }
  }
  // layer 2 two n-tiles at a time: their GELU outputs are exactly the A
  // fragment of one k-step of layer 3, consumed at once (4 registers live
  // instead of the 16 of the whole hidden layer)
  float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
  for (int ks3 = 0; ks3 < 4; ++ks3) {  // not unrolled: 8 weight fragments in flight, not 32
    uint32_t a3[4];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int nt = 2 * ks3 + half;
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) mma_bf16(c, &h1[4 * ks], w2[(ks * 8 + nt) * 32 + lane]);
      const float bb0 = b2[8 * nt + 2 * t], bb1 = b2[8 * nt + 2 * t + 1];
      a3[2 * half] = gelu2_bf16(c[0], c[1], bb0, bb1);
      a3[2 * half + 1] = gelu2_bf16(c[2], c[3], bb0, bb1);
    }
    mma_bf16(o, a3, w3[ks3 * 32 + lane]);
  }
  out[0] = o[0] + b3[2 * t];
  out[1] = o[1] + b3[2 * t + 1];
  out[2] = o[2] + b3[2 * t];
  out[3] = o[3] + b3[2 * t + 1];
}

}  // namespace nbsp_mlp
