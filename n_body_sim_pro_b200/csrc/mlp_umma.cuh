// The correction MLP (10 -> 64 -> 64 -> 3, GELU, BF16 weights, FP32 accumulate)
// on the 5th-generation tensor cores of sm_100a: one 128-row tile per CTA of
// 128 threads, every product a tcgen05.mma issued by one thread with both
// operands in shared memory and the FP32 accumulator in tensor memory (TMEM),
// read back with tcgen05.ld by the four warps (warp w owns TMEM lanes
// 32w..32w+31, i.e. rows 32w..32w+31 of the tile; one thread per row).
//
//   layer 1: D1[128 x 64] = X[128 x 16] . W1^T   (one K = 16 step)
//   layer 2: D2[128 x 64] = H1[128 x 64] . W2^T  (four K = 16 steps)
//   layer 3: D3[128 x 16] = H2[128 x 64] . W3^T  (four steps, N padded 3 -> 16)
//
// Between layers each thread adds the bias, applies GELU in paired FP32 and
// writes its row of the next operand as BF16.  TMEM: 64 columns per CTA, the
// three accumulators one after another (each is read out before the next
// product is issued); shared memory: one hidden-activation buffer, H2
// overwriting H1 once the product that read H1 has completed.  About 33 KB and
// 64 TMEM columns per CTA, so six CTAs share an SM and hide each other's
// latencies.
//
// Operand images are K-major without swizzle (the canonical "interleaved"
// layout of the tcgen05 shared-memory descriptor): core matrices of 8 rows x
// 16 bytes (8 BF16 along K) stored as 128 contiguous bytes; core matrix (row
// group i, K chunk j) sits at i * SBO + j * LBO with LBO = 128 bytes (the two
// K halves of one K = 16 step) and SBO = 8 chunks x 128 bytes for K = 64 (2 x
// 128 for K = 16).  Element (r, k) of a K-major operand with K = 8 * kc is the
// BF16 at byte (r / 8) * kc * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mlp.cuh"

namespace nbsp_umma {

constexpr int kRows = 128;            // M of every product; one thread per row
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 64;    // power of two >= 32
constexpr uint32_t kColD1 = 0, kColD2 = 0, kColD3 = 0;
constexpr int kCtasPerSm = 6;         // shared memory: 6 x ~33 KB; TMEM: 6 x 64 of 512 columns
constexpr uint32_t kLbo = 128;
constexpr uint32_t kSboK16 = 2 * 128;
constexpr uint32_t kSboK64 = 8 * 128;
// mbarrier polls before a wait gives up (each try_wait may itself suspend the
// thread for a while): far beyond a tile's few microseconds
constexpr int kWaitPolls = 1 << 22;

// 16-byte index of the chunk holding elements (r, 8c .. 8c+7) of a K-major
// image with `kc` chunks of 8 elements per row.
__host__ __device__ constexpr int chunk_index(int r, int c, int kc) {
  return (r >> 3) * (kc * 8) + c * 8 + (r & 7);
}

// Weight images in that layout, built once per parameter update (mlp.cu) and
// copied to shared memory by each CTA: W1 as N 64 x K 16 (inputs 10..15 zero),
// W2 as N 64 x K 64, W3 as N 16 x K 64 (outputs 3..15 zero).
struct Weights {
  uint4 w1[64 * 16 / 8];
  uint4 w2[64 * 64 / 8];
  uint4 w3[16 * 64 / 8];
};

static_assert(sizeof(Weights) == sizeof(nbsp_mlp::Net::umma_w), "weight image size");

__device__ __forceinline__ const Weights* weights_of(const nbsp_mlp::Net* net) {
  return reinterpret_cast<const Weights*>(net->umma_w);
}

struct __align__(128) Smem {
  uint4 x[kRows * 16 / 8];
  uint4 h[kRows * 64 / 8];  // H1, then H2
  Weights w;
  float b1[64], b2[64], b3[16];
  unsigned long long bar;
  uint32_t tmem;
  int failed;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, LBO, SBO (all >> 4), the
// Blackwell descriptor version (bit 46), no swizzle, base offset 0.
__device__ __forceinline__ uint64_t sdesc(const void* p, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((smem_u32(p) >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on `bar` when every tcgen05.mma this thread issued so far is done.
__device__ __forceinline__ void commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes made visible to the tensor core's reads
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for phase `parity` of `bar`; false when it did not complete.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < kWaitPolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Allocation by warp 0 (the whole warp), address published through shared memory.
__device__ __forceinline__ void tmem_alloc(Smem& s) {
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(&s.tmem)), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
}
__device__ __forceinline__ void tmem_free(uint32_t tmem) {
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(kTmemCols)
                 : "memory");
}

// CTA set-up: weights and biases into shared memory, the barrier, TMEM.
__device__ __forceinline__ void setup(Smem& s, const Weights* w, const nbsp_mlp::Net* net) {
  const uint4* src = reinterpret_cast<const uint4*>(w);
  uint4* dst = reinterpret_cast<uint4*>(&s.w);
  for (int k = threadIdx.x; k < (int)(sizeof(Weights) / 16); k += kThreads) dst[k] = src[k];
  for (int k = threadIdx.x; k < 64; k += kThreads) {
    s.b1[k] = net->b1[k];
    s.b2[k] = net->b2[k];
  }
  if (threadIdx.x < 16) s.b3[threadIdx.x] = threadIdx.x < nbsp_mlp::kOutPad ? net->b3[threadIdx.x] : 0.f;
  if (threadIdx.x == 0) {
    bar_init(&s.bar);
    s.failed = 0;
  }
  fence_async_smem();
  tmem_alloc(s);
  fence_before();
  __syncthreads();
  fence_after();
}

// Release TMEM (all threads call; every tcgen05.ld has completed).
__device__ __forceinline__ void teardown(Smem& s, uint32_t tmem) {
  fence_before();
  __syncthreads();
  fence_after();
  tmem_free(tmem);
}

// Writes this thread's row of the standardised input tile (10 features, the
// rest zero) into s.x.
__device__ __forceinline__ void put_inputs(Smem& s, const float* v) {
  const int r = threadIdx.x;
  s.x[chunk_index(r, 0, 2)] = make_uint4(nbsp_mlp::pack_bf16(v[0], v[1]), nbsp_mlp::pack_bf16(v[2], v[3]),
                                         nbsp_mlp::pack_bf16(v[4], v[5]), nbsp_mlp::pack_bf16(v[6], v[7]));
  s.x[chunk_index(r, 1, 2)] = make_uint4(nbsp_mlp::pack_bf16(v[8], v[9]), 0u, 0u, 0u);
}

// One hidden layer's epilogue: 64 accumulator columns of this thread's row,
// plus the bias, through GELU, as BF16 into the row of the next operand.
__device__ __forceinline__ void hidden_epilogue(uint32_t taddr, const float* bias, uint4* dst) {
  const int r = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float v[16];
    tmem_ld16(taddr + 16 * q, v);
    tmem_wait_ld();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = 16 * q + 8 * h;
      dst[chunk_index(r, k >> 3, 8)] = make_uint4(
          nbsp_mlp::gelu2_bf16(v[8 * h + 0], v[8 * h + 1], bias[k + 0], bias[k + 1]),
          nbsp_mlp::gelu2_bf16(v[8 * h + 2], v[8 * h + 3], bias[k + 2], bias[k + 3]),
          nbsp_mlp::gelu2_bf16(v[8 * h + 4], v[8 * h + 5], bias[k + 4], bias[k + 5]),
          nbsp_mlp::gelu2_bf16(v[8 * h + 6], v[8 * h + 7], bias[k + 6], bias[k + 7]));
    }
  }
}

// Forward pass of the tile in s.x (written by every thread, then a
// __syncthreads by the caller after fence_async_smem).  On return out[0..2]
// holds this thread's row of the network output (standardised units).  Returns
// false on every thread when a product did not complete in time (the caller
// stops; s.failed is set).
__device__ __forceinline__ bool forward(Smem& s, uint32_t tmem, uint32_t& phase, float* out) {
  const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31) << 16;  // TMEM lane of the warp
  const bool issuer = threadIdx.x == 0;
  // layer 1
  if (issuer) {
    fence_after();
    mma(tmem + kColD1, sdesc(s.x, kLbo, kSboK16), sdesc(s.w.w1, kLbo, kSboK16),
        idesc_bf16(kRows, 64), 0u);
    commit(&s.bar);
  }
  bool ok = bar_wait(&s.bar, phase);
  phase ^= 1u;
  if (__syncthreads_or(!ok)) return false;
  fence_after();
  hidden_epilogue(tmem + lane_base + kColD1, s.b1, s.h);
  fence_async_smem();
  fence_before();
  __syncthreads();
  // layer 2
  if (issuer) {
    fence_after();
#pragma unroll
    for (int k = 0; k < 4; ++k)
      mma(tmem + kColD2, sdesc(reinterpret_cast<const char*>(s.h) + 2 * kLbo * k, kLbo, kSboK64),
          sdesc(reinterpret_cast<const char*>(s.w.w2) + 2 * kLbo * k, kLbo, kSboK64),
          idesc_bf16(kRows, 64), k > 0 ? 1u : 0u);
    commit(&s.bar);
  }
  ok = bar_wait(&s.bar, phase);
  phase ^= 1u;
  if (__syncthreads_or(!ok)) return false;
  fence_after();
  // H2 overwrites H1: the product that read H1 has completed (its commit)
  hidden_epilogue(tmem + lane_base + kColD2, s.b2, s.h);
  fence_async_smem();
  fence_before();
  __syncthreads();
  // layer 3 (its accumulator reuses the columns read above)
  if (issuer) {
    fence_after();
#pragma unroll
    for (int k = 0; k < 4; ++k)
      mma(tmem + kColD3, sdesc(reinterpret_cast<const char*>(s.h) + 2 * kLbo * k, kLbo, kSboK64),
          sdesc(reinterpret_cast<const char*>(s.w.w3) + 2 * kLbo * k, kLbo, kSboK64),
          idesc_bf16(kRows, 16), k > 0 ? 1u : 0u);
    commit(&s.bar);
  }
  ok = bar_wait(&s.bar, phase);
  phase ^= 1u;
  if (__syncthreads_or(!ok)) return false;
  fence_after();
  float v[16];
  tmem_ld16(tmem + lane_base + kColD3, v);
  tmem_wait_ld();
  out[0] = v[0] + s.b3[0];
  out[1] = v[1] + s.b3[1];
  out[2] = v[2] + s.b3[2];
  // the next tile's products overwrite these columns after its __syncthreads
  fence_before();
  return true;
}

// Builds the three weight images from the FP32 parameter vector (row-major
// W[out][in], as nbsp_mlp's offsets); called by one CTA.
__device__ __forceinline__ void build_weights(const float* params, Weights* w) {
  using namespace nbsp_mlp;
  auto put = [](uint4* img, int kc, int n, int c, const float* row, int valid_k) {
    float e[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) e[q] = (8 * c + q < valid_k) ? row[8 * c + q] : 0.f;
    img[chunk_index(n, c, kc)] = make_uint4(pack_bf16(e[0], e[1]), pack_bf16(e[2], e[3]),
                                            pack_bf16(e[4], e[5]), pack_bf16(e[6], e[7]));
  };
  for (int i = threadIdx.x; i < 64 * 2; i += blockDim.x) {  // W1: n 64, 2 chunks
    const int n = i >> 1, c = i & 1;
    put(w->w1, 2, n, c, params + kOffW1 + n * kIn, kIn);
  }
  for (int i = threadIdx.x; i < 64 * 8; i += blockDim.x) {  // W2: n 64, 8 chunks
    const int n = i >> 3, c = i & 7;
    put(w->w2, 8, n, c, params + kOffW2 + n * kHidden, kHidden);
  }
  for (int i = threadIdx.x; i < 16 * 8; i += blockDim.x) {  // W3: n 16 (3 real), 8 chunks
    const int n = i >> 3, c = i & 7;
    if (n < kOut) {
      put(w->w3, 8, n, c, params + kOffW3 + n * kHidden, kHidden);
    } else {
      w->w3[chunk_index(n, c, 8)] = make_uint4(0u, 0u, 0u, 0u);
    }
  }
}

}  // namespace nbsp_umma
