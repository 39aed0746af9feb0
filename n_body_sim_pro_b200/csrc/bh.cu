// GPU Barnes-Hut kernels for sm_100a.
//
// Reference (richie-rich90454/n_body_sim_pro, src/c/barnes_hut/barnes_hut.c):
//   root cube      :453-483   keys  :286-305   sort  :312-339
//   reorder        :402-440   COM   :214-253   walk  :549-636   scatter :692-704
//
// The Morton keys and the sort permutation are bit-exact with the reference:
// all FP64 arithmetic of the root cube and of morton_axis_code is done with
// explicitly rounded __d*_rn intrinsics (no contraction), and the 8 x 8-bit
// stable LSD sort yields the same permutation as the reference's stable
// 3 x 21-bit LSD sort (a stable sort by the full key, ties by original index).
//
// The tree differs from the reference's pointer octree by design: it is built
// in parallel from the sorted keys (a Karras binary radix tree, one thread per
// internal node), collapsed to a path-compressed octree whose leaves hold up to
// `leaf_capacity` Morton-contiguous particles, and stored in depth-first order
// with skip links so the walk needs no stack.  Parity is judged on forces
// against the FP64 all-pairs oracle, and the opening test is the reference's:
// accept a cell when (2h)^2 < theta^2 d^2, d to the cell centre of mass.  A
// bucket of >= 2 particles is the reference's cell of the same side and
// particles, so it takes the same test; where the reference would open it, its
// particles are summed exactly (a single particle is always exact).
#include "bh.h"
#include "mlp.cuh"
#include "mlp_umma.cuh"

#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>

namespace {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// bounds
// ---------------------------------------------------------------------------

constexpr int kBoundsThreads = 256;
constexpr int kBoundsBlocks = 4 * 148;  // one wave at 4 blocks of 256 per SM (58 registers)
constexpr int kBoundsVals = 11;  // min xyz, max xyz, m, mx, my, mz, |a|^2

// The block's combined values in thread 0: each warp by shuffles, then the
// warps' results by the first warp.
__device__ __forceinline__ void bounds_block_reduce(double (&v)[kBoundsVals],
                                                    double (*sh)[kBoundsThreads / 32]) {
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int q = 0; q < kBoundsVals; ++q) {
      const double o = __shfl_xor_sync(0xffffffffu, v[q], off);
      v[q] = q < 3 ? fmin(v[q], o) : q < 6 ? fmax(v[q], o) : v[q] + o;
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < kBoundsVals; ++q) sh[q][w] = v[q];
  __syncthreads();
  if (w != 0) return;
#pragma unroll
  for (int q = 0; q < kBoundsVals; ++q)
    v[q] = lane < kBoundsThreads / 32 ? sh[q][lane]
           : q < 3                    ? INFINITY
           : q < 6                    ? -INFINITY
                                      : 0.0;
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int q = 0; q < kBoundsVals; ++q) {
      const double o = __shfl_xor_sync(0xffffffffu, v[q], off);
      v[q] = q < 3 ? fmin(v[q], o) : q < 6 ? fmax(v[q], o) : v[q] + o;
    }
  }
}

// KICK: the opening kick and drift of a device-resident leapfrog step first
// (kick_drift_kernel's arithmetic), the reductions then of the drifted state.
template <bool KICK>
__global__ void __launch_bounds__(kBoundsThreads) bounds_kernel(
    double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
    const double* __restrict__ m, size_t n, double* __restrict__ partial, int* status,
    const double* __restrict__ ax, const double* __restrict__ ay,
    const double* __restrict__ az, bool rms_of_a, double* __restrict__ vx,
    double* __restrict__ vy, double* __restrict__ vz, double h, double dt) {
  __shared__ double sh[kBoundsVals][kBoundsThreads / 32];
  double v[kBoundsVals] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY,
                           0.0,      0.0,      0.0,      0.0,       0.0};
  bool bad = false;
#pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)kBoundsThreads + threadIdx.x; i < n;
       i += (size_t)gridDim.x * kBoundsThreads) {
    double px = x[i], py = y[i], pz = z[i];
    const double pm = m[i];
    if (KICK) {
      const double u = __dadd_rn(vx[i], __dmul_rn(ax[i], h));
      const double w = __dadd_rn(vy[i], __dmul_rn(ay[i], h));
      const double q = __dadd_rn(vz[i], __dmul_rn(az[i], h));
      vx[i] = u;
      vy[i] = w;
      vz[i] = q;
      px = __dadd_rn(px, __dmul_rn(u, dt));
      py = __dadd_rn(py, __dmul_rn(w, dt));
      pz = __dadd_rn(pz, __dmul_rn(q, dt));
      x[i] = px;
      y[i] = py;
      z[i] = pz;
    }
    bad |= !(isfinite(px) && isfinite(py) && isfinite(pz));
    v[0] = fmin(v[0], px);
    v[1] = fmin(v[1], py);
    v[2] = fmin(v[2], pz);
    v[3] = fmax(v[3], px);
    v[4] = fmax(v[4], py);
    v[5] = fmax(v[5], pz);
    v[6] += pm;
    v[7] += pm * px;
    v[8] += pm * py;
    v[9] += pm * pz;
    if (rms_of_a) v[10] += ax[i] * ax[i] + ay[i] * ay[i] + az[i] * az[i];
  }
  if (bad) atomicOr(status, NBSP_DEVICE_ERROR_NONFINITE_POSITION);
  bounds_block_reduce(v, sh);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kBoundsVals; ++q) partial[blockIdx.x * kBoundsVals + q] = v[q];
}

// Root cube with the exact FP64 operation sequence of barnes_hut.c:471-483.
__global__ void __launch_bounds__(kBoundsThreads) bounds_final_kernel(
    const double* __restrict__ partial, int blocks, size_t n, double* __restrict__ geometry) {
  __shared__ double sh[kBoundsVals][kBoundsThreads / 32];
  double v[kBoundsVals] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY,
                           0.0,      0.0,      0.0,      0.0,       0.0};
  for (int b = threadIdx.x; b < blocks; b += kBoundsThreads) {
    for (int q = 0; q < 3; ++q) v[q] = fmin(v[q], partial[b * kBoundsVals + q]);
    for (int q = 3; q < 6; ++q) v[q] = fmax(v[q], partial[b * kBoundsVals + q]);
    for (int q = 6; q < kBoundsVals; ++q) v[q] += partial[b * kBoundsVals + q];
  }
  bounds_block_reduce(v, sh);
  if (threadIdx.x == 0) {
    const double lo[3] = {v[0], v[1], v[2]};
    const double hi[3] = {v[3], v[4], v[5]};
    double half = __dmul_rn(0.5, __dsub_rn(hi[0], lo[0]));
    for (int k = 1; k < 3; ++k) {
      const double e = __dmul_rn(0.5, __dsub_rn(hi[k], lo[k]));
      if (e > half) half = e;
    }
    if (half == 0.0) half = 0.5;
    half = __dmul_rn(half, 1.0 + 1.0e-9);
    for (int k = 0; k < 3; ++k) geometry[k] = __dmul_rn(0.5, __dadd_rn(lo[k], hi[k]));
    geometry[3] = half;
    const double mt = v[6];
    for (int k = 0; k < 3; ++k) geometry[4 + k] = mt != 0.0 ? v[7 + k] / mt : 0.0;
    geometry[7] = n > 0 ? sqrt(v[10] / (double)n) : 0.0;  // rms |a| (when given)
  }
}

// ---------------------------------------------------------------------------
// Morton keys
// ---------------------------------------------------------------------------

// barnes_hut.c:286-294 with every FP64 operation explicitly rounded.
__device__ __forceinline__ uint64_t axis_code(double value, double centre, double half) {
  double t = __dadd_rn(__ddiv_rn(__dsub_rn(value, centre), __dmul_rn(2.0, half)), 0.5);
  if (t < 0.0) {
    t = 0.0;
  } else if (t >= 1.0) {
    t = 1.0 - 1.0e-15;
  }
  return (uint64_t)__double2ull_rz(__dmul_rn(t, 2097152.0));
}

// Spread the low 21 bits of v to every third bit (bit b -> bit 3b).
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x001f00000000ffffull;
  v = (v | (v << 16)) & 0x001f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

// ---------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits, one kernel per pass
//
// The keys kernel also counts the 8 digit histograms (one read of the keys);
// one block turns them into each pass's digit bases.  Every pass is then a
// single kernel: tiles take tickets in launch order, rank their keys in shared
// memory, and find their global offsets with a decoupled look-back over the
// preceding tiles' published digit counts (flag A: this tile's count, flag P:
// inclusive prefix).  A tile only waits on tiles with earlier tickets, which
// are already resident; every wait is bounded and flags an error when it
// runs out.
// ---------------------------------------------------------------------------

// 512 threads of 8 keys: twice the warps of 256 x 16 at the same tile (the
// ranking chain per warp is half as long); at 10M keys 0.92 ms for the 8
// passes against 1.10 with 256 x 16 (and 1.17 with 1024 x 4, one block per SM)
constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kRadix = 256;
constexpr int kLookback = 8;  // predecessors' flags read at once in the look-back
static_assert(kSortThreads >= kRadix, "one thread per digit");
constexpr int kSortPasses = 8;
constexpr uint32_t kFlagA = 1u << 30, kFlagP = 2u << 30, kCountMask = (1u << 30) - 1u;
constexpr int kLookbackSpins = 1 << 22;  // ~ms per predecessor before the error flag
constexpr int kKeysBlocks = 5 * 148;  // 40 warps per SM (48 registers): enough loads in flight

// Sort scratch (32-bit words): hist[8][256] | base[8][256] | ticket[8] | status[8][tiles][256]
struct SortScratch {
  uint32_t* hist;
  uint32_t* base;
  uint32_t* ticket;
  uint32_t* status;
};
__host__ __device__ inline size_t sort_tiles(size_t n) { return (n + kSortTile - 1) / kSortTile; }
inline SortScratch sort_scratch(uint32_t* w, size_t n) {
  SortScratch s;
  s.hist = w;
  s.base = w + kSortPasses * kRadix;
  s.ticket = s.base + kSortPasses * kRadix;
  s.status = s.ticket + kSortPasses;
  (void)n;
  return s;
}
inline size_t sort_scratch_words(size_t n) {
  return 2 * kSortPasses * kRadix + kSortPasses + kSortPasses * sort_tiles(n) * kRadix;
}

__global__ void __launch_bounds__(256) keys_kernel(
    const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
    const double* __restrict__ m, size_t n, const double* __restrict__ geometry,
    uint64_t* __restrict__ keys, uint32_t* __restrict__ index, float4* __restrict__ unsorted,
    uint32_t* __restrict__ hist, const double* __restrict__ ax, const double* __restrict__ ay,
    const double* __restrict__ az, double tol_scale, float* __restrict__ unsorted_tol) {
  __shared__ uint32_t h[kSortPasses][kRadix];
  for (int k = threadIdx.x; k < kSortPasses * kRadix; k += blockDim.x) (&h[0][0])[k] = 0;
  __syncthreads();
  const double cx = geometry[0], cy = geometry[1], cz = geometry[2], hs = geometry[3];
  const double mx = geometry[4], my = geometry[5], mz = geometry[6];  // centre of mass
  const double a_floor = geometry[7];  // rms |a_old|: the relative test's floor
  const unsigned lane = threadIdx.x & 31;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t first = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  // every lane runs the same number of iterations (match_any needs the whole warp)
  const size_t rounds = (n + stride - 1) / stride;
  for (size_t r = 0; r < rounds; ++r) {
    const size_t i = first + r * stride;
    const bool valid = i < n;
    uint64_t key = 0;
    if (valid) {
      const double xi = x[i], yi = y[i], zi = z[i];
      key = spread3(axis_code(xi, cx, hs)) | (spread3(axis_code(yi, cy, hs)) << 1) |
            (spread3(axis_code(zi, cz, hs)) << 2);
      keys[i] = key;
      index[i] = (uint32_t)i;
      // the walk's float4 (relative to the centre of mass), still in input
      // order: the gather then moves one 16-byte record per particle
      unsorted[i] = make_float4((float)__dsub_rn(xi, mx), (float)__dsub_rn(yi, my),
                                (float)__dsub_rn(zi, mz), (float)m[i]);
      if (unsorted_tol != nullptr) {  // relative opening test: alpha max(|a_old|, rms) / G
        const double a = fmax(sqrt(ax[i] * ax[i] + ay[i] * ay[i] + az[i] * az[i]), a_floor);
        unsorted_tol[i] = a > 0.0 && isfinite(a) ? (float)(tol_scale * a) : INFINITY;
      }
    }
#pragma unroll
    // digit counts: the low six bytes of the keys of one warp are spread over
    // many values (plain shared atomics); the top two bytes (the first octree
    // levels) repeat, so they are aggregated per warp first
    for (int p = 0; p < kSortPasses; ++p) {
      if (p < 6) {
        if (valid) atomicAdd(&h[p][(unsigned)(key >> (8 * p)) & 0xffu], 1u);
      } else {
        const unsigned d = valid ? (unsigned)(key >> (8 * p)) & 0xffu : 0x100u;
        const unsigned peers = __match_any_sync(kFull, d);
        if (valid && lane == (unsigned)(__ffs(peers) - 1)) atomicAdd(&h[p][d], (uint32_t)__popc(peers));
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kSortPasses * kRadix; k += blockDim.x) {
    const uint32_t v = (&h[0][0])[k];
    if (v != 0) atomicAdd(&hist[k], v);
  }
}

// One block of 256 threads: base[p][d] = number of keys whose digit p is < d.
__global__ void __launch_bounds__(kRadix) sort_bases_kernel(const uint32_t* __restrict__ hist,
                                                            uint32_t* __restrict__ base) {
  __shared__ uint32_t sh[kRadix];
  const int d = threadIdx.x;
  for (int p = 0; p < kSortPasses; ++p) {
    const uint32_t own = hist[p * kRadix + d];
    uint32_t v = own;
    sh[d] = v;
    for (int off = 1; off < kRadix; off <<= 1) {
      __syncthreads();
      const uint32_t add = d >= off ? sh[d - off] : 0u;
      __syncthreads();
      v += add;
      sh[d] = v;
    }
    base[p * kRadix + d] = v - own;
    __syncthreads();
  }
}

__device__ __forceinline__ uint32_t load_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

__global__ void __launch_bounds__(kSortThreads, 2) sort_pass_kernel(
    const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, size_t n, int shift,
    const uint32_t* __restrict__ base, uint32_t* ticket, uint32_t* status, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* sk = reinterpret_cast<uint64_t*>(smem);                     // kSortTile
  uint32_t* sv = reinterpret_cast<uint32_t*>(sk + kSortTile);           // kSortTile
  uint32_t* wc = sv + kSortTile;                                        // kSortWarps * 256
  uint32_t* start = wc + kSortWarps * kRadix;                           // 256
  uint32_t* gofs = start + kRadix;                                      // 256
  __shared__ int s_tile;

  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  if (t == 0) s_tile = (int)atomicAdd(ticket, 1u);
  for (int k = t; k < kSortWarps * kRadix; k += kSortThreads) wc[k] = 0;
  __syncthreads();
  const int tile = s_tile;

  const size_t base_i = (size_t)tile * kSortTile + (size_t)w * (kSortItems * 32);
  const unsigned lt = (1u << lane) - 1u;
  uint64_t key[kSortItems];
  uint32_t val[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {  // every load of the tile in flight at once
    const size_t i = base_i + (size_t)it * 32 + lane;
    const bool valid = i < n;
    key[it] = valid ? keys_in[i] : 0ull;
    val[it] = valid ? vals_in[i] : 0u;
  }
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const bool valid = base_i + (size_t)it * 32 + lane < n;
    const unsigned digit = valid ? ((unsigned)(key[it] >> shift) & 0xffu) : 0x100u;
    const unsigned peers = __match_any_sync(kFull, digit);
    uint32_t before = 0;
    if (valid) before = wc[w * kRadix + digit];
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) wc[w * kRadix + digit] = before + __popc(peers);
    __syncwarp();
    rank[it] = before + __popc(peers & lt);
  }
  __syncthreads();
  // threads t < 256: digit t — this tile's count, publish, look back, and the
  // exclusive scan of the tile's digit totals (warp shuffles, then warp sums)
  __shared__ uint32_t s_wsum[kRadix / 32];
  if (t < kRadix) {
    uint32_t run = 0;
    for (int ww = 0; ww < kSortWarps; ++ww) {
      const uint32_t c = wc[ww * kRadix + t];
      wc[ww * kRadix + t] = run;
      run += c;
    }
    const uint32_t count = run;  // this tile's keys with digit t
    uint32_t* st = status + (size_t)tile * kRadix + t;
    atomicExch(st, (tile == 0 ? kFlagP : kFlagA) | count);
    uint32_t prefix = 0;
    if (tile > 0) {
      // kLookback predecessors at a time, nearest first: counts are added up
      // to the first unpublished flag (read again) or the first inclusive one
      int j = tile - 1, spins = 0;
      for (;;) {
        uint32_t v[kLookback];
#pragma unroll
        for (int k = 0; k < kLookback; ++k)
          v[k] = j - k >= 0 ? load_volatile(status + (size_t)(j - k) * kRadix + t) : kFlagP;
        int used = 0;
        bool done = false;
#pragma unroll
        for (int k = 0; k < kLookback; ++k) {
          if (done || used < k) continue;
          const uint32_t flag = v[k] & ~kCountMask;
          if (flag == 0u) continue;
          prefix += v[k] & kCountMask;
          used = k + 1;
          if (flag == kFlagP) done = true;
        }
        if (done) break;
        if (used == 0 && ++spins > kLookbackSpins) {
          atomicOr(err, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
          break;
        }
        j -= used;
      }
      atomicExch(st, kFlagP | ((prefix + count) & kCountMask));
    }
    gofs[t] = base[t] + prefix;
    uint32_t x = count;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t u = __shfl_up_sync(kFull, x, off);
      if (lane >= off) x += u;
    }
    if (lane == 31) s_wsum[w] = x;
    start[t] = x - count;
  }
  __syncthreads();
  if (t < kRadix) {
    uint32_t before = 0;
    for (int k = 0; k < w; ++k) before += s_wsum[k];
    start[t] += before;
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const size_t i = base_i + (size_t)it * 32 + lane;
    if (i < n) {
      const unsigned digit = (unsigned)(key[it] >> shift) & 0xffu;
      const uint32_t pos = start[digit] + wc[w * kRadix + digit] + rank[it];
      if (pos < (uint32_t)kSortTile) {
        sk[pos] = key[it];
        sv[pos] = val[it];
      } else {
        atomicOr(err, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      }
    }
  }
  __syncthreads();
  const size_t tile_base = (size_t)tile * kSortTile;
  const int count_all = (int)(n - tile_base < (size_t)kSortTile ? n - tile_base : (size_t)kSortTile);
  for (int q = t; q < count_all; q += kSortThreads) {
    const uint64_t k = sk[q];
    const unsigned digit = (unsigned)(k >> shift) & 0xffu;
    const size_t dst = (size_t)gofs[digit] + (size_t)(q - (int)start[digit]);
    if (dst < n) {
      keys_out[dst] = k;
      vals_out[dst] = sv[q];
    } else {
      atomicOr(err, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
    }
  }
}

constexpr size_t kDownsweepSmem =
    (size_t)kSortTile * (sizeof(uint64_t) + sizeof(uint32_t)) +
    (size_t)(kSortWarps * kRadix + 2 * kRadix) * sizeof(uint32_t);

// The reference's insertion build fails with OVERFLOW when two particles share
// a position (barnes_hut.c:149-153: more than 128 subdivisions).  Equal
// positions have equal keys, so after the sort they sit in one run of equal
// keys; each particle is compared with the next kDupWindow particles of its run
// (runs of equal 63-bit keys are otherwise rare: cells of 2^-21 of the root).
constexpr int kDupWindow = 32;
__global__ void duplicates_kernel(const uint64_t* __restrict__ keys,
                                  const uint32_t* __restrict__ perm, const double* __restrict__ x,
                                  const double* __restrict__ y, const double* __restrict__ z,
                                  size_t n, int* status) {
  for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s + 1 < n;
       s += (size_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[s];
    if (keys[s + 1] != k) continue;
    const uint32_t i = perm[s];
    if (i >= n) continue;
    const double px = x[i], py = y[i], pz = z[i];
    for (size_t t = s + 1; t < n && t <= s + kDupWindow && keys[t] == k; ++t) {
      const uint32_t j = perm[t];
      if (j < n && x[j] == px && y[j] == py && z[j] == pz) {
        atomicOr(status, NBSP_DEVICE_ERROR_DUPLICATE_POSITION);
        return;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// gather / scatter
// ---------------------------------------------------------------------------

// pos[s] = unsorted[perm[s]]; the relative opening test's tolerances the same
// way when present.
__global__ void gather_kernel(const float4* __restrict__ unsorted,
                              const uint32_t* __restrict__ perm, size_t n,
                              float4* __restrict__ pos, const float* __restrict__ unsorted_tol,
                              float* __restrict__ tol, int* status) {
  for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < n;
       s += (size_t)gridDim.x * blockDim.x) {
    const uint32_t i = perm[s];
    if (i >= n) {
      atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      pos[s] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    pos[s] = unsorted[i];
    if (tol != nullptr) tol[s] = unsorted_tol[i];
  }
}

// a[i] = G * acc[i]: the walk wrote each target's sum at its input index
// (one aligned 32-byte record), so this pass is coalesced both ways.  KICK:
// the closing kick of a device-resident leapfrog step, v += h a, with
// kick_drift_kernel's arithmetic on the accelerations just written.
template <bool KICK>
__global__ void unsort_kernel(const double4* __restrict__ acc, size_t n, double g,
                              double* __restrict__ ax, double* __restrict__ ay,
                              double* __restrict__ az, double* __restrict__ vx,
                              double* __restrict__ vy, double* __restrict__ vz, double h) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double4 a = acc[i];
    const double gx = g * a.x, gy = g * a.y, gz = g * a.z;
    ax[i] = gx;
    ay[i] = gy;
    az[i] = gz;
    if (KICK) {
      vx[i] = __dadd_rn(vx[i], __dmul_rn(gx, h));
      vy[i] = __dadd_rn(vy[i], __dmul_rn(gy, h));
      vz[i] = __dadd_rn(vz[i], __dmul_rn(gz, h));
    }
  }
}

// ---------------------------------------------------------------------------
// tree
// ---------------------------------------------------------------------------

// Scratch layout of one tree; binary ids: internal node i -> i (0..n-2),
// particle leaf k -> (n-1) + k.
struct Tree {
  int n;
  int2* range;        // [n-1] first, last of internal nodes
  int2* child;        // [n-1] binary ids of the two children
  int* cell;          // [2n-1] octree level of a cell node, -1 otherwise
  int* oparent;       // [2n-1] octree parent (binary id) of a cell node, from keep_kernel
  uint32_t* mask;     // [n]   levels of kept nodes starting at particle k
  uint32_t* offset;   // [n+1] exclusive scan of popcounts; offset[n] = node count
  uint32_t* block_sums;  // scan scratch
  // octree nodes, depth-first order, capacity 2n-1
  int4* info;         // next, begin, leaf count (0: internal), parent
  int* level;
  int* nchild;
  int* arrive;
  int* height;
  double4* mom;       // mass, com xyz (relative to the centre of mass)
  double* quad64;     // 6 per node: xx xy xz yy yz zz (trace-free)
  float4* com;        // walk format: com xyz, mass
  float* ropen2;      // (2h / theta)^2
  float4* quad;       // 2 per node: (xx, xy, xz, yy), (yz, 0, 0, 0)
  int* children;      // 8 per internal node, depth-first order (interaction-list walk)
  double* trace64;    // sum m |x - com|^2 per node (FP64)
  float* side;        // cell side 2h = root side / 2^level
  float* spread;      // sum m |x - com|^2 / (M side^2): the correction MLP's 10th feature
  float* shift;       // distance from the cell's geometric centre to its centre of mass
  float* kmass;       // M side^2: the relative opening test's cell term
  // what the interaction-list walk reads of a node, in one 32-byte record:
  // (com xyz, mass), (ropen2, kmass, first particle, count as int bits: the
  // particle count of a bucket, minus the number of children of an internal node)
  float4* wnode;      // 2 per node
  unsigned long long* leaves;  // [1]
};

constexpr int kScanItems = 2048;

// Sub-buffers of the tree scratch, each 256-byte aligned, carved from an
// integer base address (tree_bytes() carves from 0 to measure the layout).
template <typename T>
__host__ __device__ inline T* carve(uintptr_t& p, size_t count) {
  T* out = reinterpret_cast<T*>(p);
  p += (count * sizeof(T) + 255) & ~(size_t)255;
  return out;
}

__host__ __device__ inline Tree tree_layout(uintptr_t p, size_t n_, uintptr_t* end) {
  Tree t;
  const size_t n = n_ < 2 ? 2 : n_;
  const size_t ni = n - 1, nb = 2 * n - 1;
  t.n = (int)n_;
  t.range = carve<int2>(p, ni);
  t.child = carve<int2>(p, ni);
  t.cell = carve<int>(p, nb);
  t.oparent = carve<int>(p, nb);
  t.mask = carve<uint32_t>(p, n);
  t.offset = carve<uint32_t>(p, n + 1);
  t.block_sums = carve<uint32_t>(p, (n + kScanItems - 1) / kScanItems + 1);
  t.info = carve<int4>(p, nb);
  t.level = carve<int>(p, nb);
  t.nchild = carve<int>(p, nb);
  t.arrive = carve<int>(p, nb);
  t.height = carve<int>(p, nb);
  t.mom = carve<double4>(p, nb);
  t.quad64 = carve<double>(p, 6 * nb);
  t.com = carve<float4>(p, nb);
  t.ropen2 = carve<float>(p, nb);
  t.quad = carve<float4>(p, 2 * nb);
  t.children = carve<int>(p, 8 * nb);
  t.trace64 = carve<double>(p, nb);
  t.side = carve<float>(p, nb);
  t.spread = carve<float>(p, nb);
  t.shift = carve<float>(p, nb);
  t.kmass = carve<float>(p, nb);
  t.wnode = carve<float4>(p, 2 * nb);
  t.leaves = carve<unsigned long long>(p, 1);
  if (end != nullptr) *end = p;
  return t;
}

inline Tree tree_view(void* base, size_t n) {
  return tree_layout(reinterpret_cast<uintptr_t>(base), n, nullptr);
}

size_t tree_bytes(size_t n) {
  uintptr_t end = 0;
  tree_layout(0, n, &end);
  return (size_t)end;
}

// Common prefix length of sorted keys i and j in bits (Karras 2012, with the
// index as tie breaker); -1 outside [0, n).
__device__ __forceinline__ int prefix(const uint64_t* __restrict__ keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint64_t a = keys[i], b = keys[j];
  if (a != b) return __clzll(a ^ b) - 1;  // keys use the low 63 bits
  return 63 + __clz((unsigned)(i ^ j));
}

__device__ __forceinline__ int level_of_delta(int delta) { return min(delta / 3, 21); }

// Karras's radix tree over the sorted keys, and which of its nodes are octree
// cells: an internal node whose octree level (prefix length / 3) is deeper
// than its parent's, the root, and a particle below a node above level 21.
// The parent's prefix length is that of the node's range extended by one key
// on the side with the longer common prefix, max(delta(first - 1, first),
// delta(last, last + 1)), so each thread decides its own node and its leaf
// children without reading another thread's results.
__global__ void radix_tree_kernel(const uint64_t* __restrict__ keys, Tree t, int* status) {
  const int n = t.n;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = prefix(keys, n, i, i + 1) - prefix(keys, n, i, i - 1) >= 0 ? 1 : -1;
  const int dmin = prefix(keys, n, i, i - d);
  int lmax = 2;
  while (prefix(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int step = lmax >> 1; step >= 1; step >>= 1)
    if (prefix(keys, n, i, i + (l + step) * d) > dmin) l += step;
  const int j = i + l * d;
  const int dnode = prefix(keys, n, i, j);
  int s = 0;
  int div = 2;
  for (;;) {
    const int step = (l + div - 1) / div;
    if (prefix(keys, n, i, i + (s + step) * d) > dnode) s += step;
    if (step <= 1) break;
    div <<= 1;
  }
  const int gamma = i + s * d + (d < 0 ? -1 : 0);
  const int first = min(i, j), last = max(i, j);
  if (first < 0 || last >= n || gamma < first || gamma >= last) {
    atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
    return;
  }
  const int left = first == gamma ? (n - 1) + gamma : gamma;
  const int right = last == gamma + 1 ? (n - 1) + gamma + 1 : gamma + 1;
  t.range[i] = make_int2(first, last);
  t.child[i] = make_int2(left, right);
  const int lvl = level_of_delta(dnode);
  const int pdelta = max(prefix(keys, n, first, first - 1), prefix(keys, n, last, last + 1));
  t.cell[i] = (i == 0 || level_of_delta(pdelta) < lvl) ? lvl : -1;
  if (left >= n - 1) t.cell[left] = lvl <= 20 ? 22 : -1;
  if (right >= n - 1) t.cell[right] = lvl <= 20 ? 22 : -1;
}


__device__ __forceinline__ int first_of(const Tree& t, int b) {
  return b < t.n - 1 ? t.range[b].x : b - (t.n - 1);
}
__device__ __forceinline__ int last_of(const Tree& t, int b) {
  return b < t.n - 1 ? t.range[b].y : b - (t.n - 1);
}

// A splitting cell: an octree cell (binary node b with cell level >= 0) of
// more than leaf_capacity particles above level 21 — an internal node of the
// bucketed octree, whose octree children are all kept.  (A cell is kept when
// its octree parent splits; the root always is.)
__device__ __forceinline__ bool splits(const Tree& t, int b, int leaf_capacity) {
  if (b >= t.n - 1) return false;  // a particle
  const int lvl = t.cell[b];
  if (lvl < 0 || lvl >= 21) return false;
  const int2 r = t.range[b];
  return r.y - r.x + 1 > leaf_capacity;
}

// The octree children of splitting cell b, in Morton order: the cells met
// first below b in the binary tree.  The binary nodes passed on the way have
// b's own level (they are not cells), at most 7 of them, so the descent is a
// stack of at most 8 entries; visit(c) is called for each child cell c.
template <typename Visit>
__device__ __forceinline__ int octree_children(const Tree& t, int b, int* status, Visit visit) {
  int stack[8];
  int top = 0, kids = 0;
  const int2 c0 = t.child[b];
  stack[top++] = c0.y;  // right pushed first: the left subtree is visited first
  stack[top++] = c0.x;
  for (int guard = 0; top > 0; ++guard) {
    const int c = stack[--top];
    if (guard > 16 || c < 0 || c >= 2 * t.n - 1) {
      atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      return kids;
    }
    if (t.cell[c] >= 0) {
      if (kids == 8) {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        return kids;
      }
      visit(c, kids++);
    } else if (c < t.n - 1 && top <= 6) {  // a binary node at b's level: its children
      const int2 cc = t.child[c];
      stack[top++] = cc.y;
      stack[top++] = cc.x;
    } else {  // a particle that is no cell, or a descent deeper than one octree level
      atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      return kids;
    }
  }
  return kids;
}

// The kept cells, marked in mask[first particle] at their level (the depth-
// first numbering counts them): the root, and the octree children of every
// splitting cell, found by the splitting cell's own thread, which also records
// itself as their octree parent.  One thread per internal binary node; only
// the splitting cells (~N / leaf capacity of them) do work.
__global__ void keep_kernel(Tree t, int leaf_capacity, int* status) {
  const int n = t.n;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n - 1) return;
  if (b == 0) {
    t.oparent[0] = -1;
    if (t.cell[0] < 0) {
      atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      return;
    }
    atomicOr(&t.mask[0], 1u << t.cell[0]);
  }
  if (!splits(t, b, leaf_capacity)) return;
  octree_children(t, b, status, [&](int c, int) {
    t.oparent[c] = b;
    const int f = first_of(t, c);
    if (f >= 0 && f < n) {
      atomicOr(&t.mask[f], 1u << t.cell[c]);
    } else {
      atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
    }
  });
}
// Exclusive scan of popc(mask[k]) into offset[0..n].
__global__ void scan_reduce_kernel(Tree t) {
  __shared__ uint32_t sh[256];
  const int n = t.n;
  const size_t base = (size_t)blockIdx.x * kScanItems;
  uint32_t s = 0;
  for (int k = threadIdx.x; k < kScanItems; k += 256) {
    const size_t i = base + k;
    if (i < (size_t)n) s += __popc(t.mask[i]);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int stride = 128; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) sh[threadIdx.x] += sh[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0) t.block_sums[blockIdx.x] = sh[0];
}

// Exclusive scan of the block sums in place (one block of 1024 threads, in
// chunks of 1024), total into offset[n].
__global__ void __launch_bounds__(1024) scan_blocks_kernel(Tree t, int blocks) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < blocks; base += 1024) {
    const int b = base + threadIdx.x;
    const uint32_t v = b < blocks ? t.block_sums[b] : 0u;
    uint32_t x = v;
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t u = __shfl_up_sync(kFull, x, off);
      if (lane >= off) x += u;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t w = warp_sums[lane];
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, w, off);
        if (lane >= off) w += u;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const uint32_t incl = x + (wid > 0 ? warp_sums[wid - 1] : 0u);
    const uint32_t c = carry;
    if (b < blocks) t.block_sums[b] = c + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = c + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) t.offset[t.n] = carry;
}

__global__ void scan_apply_kernel(Tree t) {
  __shared__ uint32_t sh[256];
  const int n = t.n;
  const size_t base = (size_t)blockIdx.x * kScanItems;
  constexpr int per = kScanItems / 256;  // 8 contiguous items per thread
  uint32_t v[per];
  uint32_t s = 0;
  for (int k = 0; k < per; ++k) {
    const size_t i = base + (size_t)threadIdx.x * per + k;
    v[k] = i < (size_t)n ? __popc(t.mask[i]) : 0u;
    s += v[k];
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  uint32_t incl = s;
  for (int off = 1; off < 256; off <<= 1) {
    const uint32_t add = threadIdx.x >= off ? sh[threadIdx.x - off] : 0u;
    __syncthreads();
    incl += add;
    sh[threadIdx.x] = incl;
    __syncthreads();
  }
  uint32_t run = t.block_sums[blockIdx.x] + incl - s;
  for (int k = 0; k < per; ++k) {
    const size_t i = base + (size_t)threadIdx.x * per + k;
    if (i < (size_t)n) t.offset[i] = run;
    run += v[k];
  }
}

__device__ __forceinline__ int dfs_index(const Tree& t, int begin, int lvl) {
  return (int)(t.offset[begin] + __popc(t.mask[begin] & ((1u << lvl) - 1u)));
}

// The record of kept cell b at depth-first index `node`: next (the first node
// after its subtree), first particle, particle count (0: internal) and octree
// parent (-1: the root).
__device__ __forceinline__ void write_node(const Tree& t, int b, int node, int parent_node,
                                           bool leaf, int total) {
  const int begin = first_of(t, b), end = last_of(t, b) + 1;
  const int next = end >= t.n ? total : (int)t.offset[end];
  t.info[node] = make_int4(next, begin, leaf ? end - begin : 0, parent_node);
  t.level[node] = t.cell[b];
  t.arrive[node] = 0;
  t.height[node] = 1;
}

// Octree records in depth-first order.  Every splitting cell writes its own
// record, its children list (in Morton order, which is depth-first order) and
// the records of its children that are buckets; a splitting child writes its
// own.  One thread per internal binary node, like keep_kernel.
__global__ void place_kernel(Tree t, int leaf_capacity, int* status) {
  const int n = t.n;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = (int)t.offset[n];
  int leaves = 0;
  if (b < n - 1 && (total < 1 || total > 2 * n - 1)) {
    if (b == 0) atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
  } else if (b < n - 1) {
    const bool split = splits(t, b, leaf_capacity);
    if (b == 0 && !split) {  // the root is the only node: one bucket
      if (total == 1) {
        write_node(t, 0, 0, -1, true, total);
        t.nchild[0] = 0;
        leaves = 1;
      } else {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      }
    } else if (split) {
      const int node = dfs_index(t, first_of(t, b), t.cell[b]);
      int parent_node = -1;
      bool ok = node >= 0 && node < total;
      if (b != 0) {
        const int p = t.oparent[b];  // keep_kernel: the splitting cell that found b
        ok = ok && p >= 0 && p < n - 1;
        if (ok) parent_node = dfs_index(t, first_of(t, p), t.cell[p]);
        ok = ok && parent_node >= 0 && parent_node < node;  // parents precede children
      }
      if (!ok) {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      } else {
        write_node(t, b, node, parent_node, false, total);
        const int kids = octree_children(t, b, status, [&](int c, int k) {
          const int cn = dfs_index(t, first_of(t, c), t.cell[c]);
          if (cn <= node || cn >= total) {
            atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
            t.children[8 * node + k] = -1;
            return;
          }
          t.children[8 * node + k] = cn;
          if (!splits(t, c, leaf_capacity)) {  // a bucket
            write_node(t, c, cn, node, true, total);
            t.nchild[cn] = 0;
            ++leaves;
          }
        });
        for (int k = kids; k < 8; ++k) t.children[8 * node + k] = -1;
        t.nchild[node] = kids;
      }
    }
  }
  leaves = (int)__reduce_add_sync(kFull, (unsigned)leaves);
  if ((threadIdx.x & 31) == 0 && leaves > 0) atomicAdd(t.leaves, (unsigned long long)leaves);
}

// Trace-free quadrupole accumulation helpers (FP64).
struct Moments {
  double m, cx, cy, cz;
  double q[6];  // xx xy xz yy yz zz
  double t2;    // sum m |x - com|^2
};

// Inverse of spread3: bits 0, 3, 6, ... of v gathered into the low 21 bits.
__device__ __forceinline__ uint32_t compact3(uint64_t v) {
  v &= 0x1249249249249249ull;
  v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
  v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
  v = (v ^ (v >> 8)) & 0x001f0000ff0000ffull;
  v = (v ^ (v >> 16)) & 0x001f00000000ffffull;
  v = (v ^ (v >> 32)) & 0x1fffffull;
  return (uint32_t)v;
}

// What the opening test of every node is built from.
struct Opening {
  const uint64_t* keys;  // sorted Morton keys (a node's first key names its cell)
  const double* geometry;
  double inv_theta, inv_theta2;
  // relative opening test on: a state without previous accelerations (rms
  // |a_old| in geometry[7] zero or not finite) is opened at the start angle
  double start_inv_theta, start_inv_theta2;
  int relative;
  int criterion;         // NBSP_BH_OPENING_*
};

template <bool QUAD>
__device__ void finish_node(const Tree& t, int node, const Moments& mo, int first, int lvl,
                            const Opening& o, int count) {
  t.mom[node] = make_double4(mo.m, mo.cx, mo.cy, mo.cz);
  if (QUAD) {
    for (int k = 0; k < 6; ++k) t.quad64[6 * node + k] = mo.q[k];
    t.trace64[node] = mo.t2;
  }
  t.com[node] = make_float4((float)mo.cx, (float)mo.cy, (float)mo.cz, (float)mo.m);
  // cell side 2h = root side / 2^lvl; the cell's centre from the first key's
  // top 3 lvl bits, in the particles' frame (relative to the centre of mass)
  const int l = min(lvl, 21);
  const double half = o.geometry[3];
  const double side = ldexp(2.0 * half, -l);
  const uint64_t key = o.keys[first];
  double shift2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double lo = o.geometry[a] - half - o.geometry[4 + a];
    const double centre = lo + ((double)(compact3(key >> a) >> (21 - l)) + 0.5) * side;
    const double d = (a == 0 ? mo.cx : a == 1 ? mo.cy : mo.cz) - centre;
    shift2 += d * d;
  }
  const double shift = sqrt(shift2);
  // Without previous accelerations every target's relative test passes (its
  // tolerance is +inf), so the geometric test alone decides: at the start
  // angle, not at the loose bound the relative test runs under.
  const double a_rms = o.geometry[7];
  const bool start = o.relative && !(a_rms > 0.0 && a_rms < INFINITY);
  const double it = start ? o.start_inv_theta : o.inv_theta;
  const double it2 = start ? o.start_inv_theta2 : o.inv_theta2;
  // reference: accept when (2h)^2 < theta^2 d^2; offset: when 2h / theta + shift < d
  const double r2 = o.criterion == NBSP_BH_OPENING_OFFSET
                        ? (side * it + shift) * (side * it + shift)
                        : side * side * it2;
  t.ropen2[node] = (float)r2;
  t.side[node] = (float)side;
  t.shift[node] = (float)shift;
  t.kmass[node] = (float)(mo.m * side * side);
  t.wnode[2 * node] = make_float4((float)mo.cx, (float)mo.cy, (float)mo.cz, (float)mo.m);
  t.wnode[2 * node + 1] = make_float4((float)r2, (float)(mo.m * side * side), __int_as_float(first),
                                      __int_as_float(count));
  if (QUAD) {
    t.spread[node] = mo.m > 0.0 ? (float)(mo.t2 / (mo.m * side * side)) : 0.f;
    t.quad[2 * node] = make_float4((float)mo.q[0], (float)mo.q[1], (float)mo.q[2], (float)mo.q[3]);
    t.quad[2 * node + 1] = make_float4((float)mo.q[4], 0.f, 0.f, 0.f);
  }
}

// L2-coherent load of a double4 written by another thread of this grid.
__device__ __forceinline__ double4 ldcg_d4(const double4* p) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Arrival at a parent: a release (this thread's node records are visible
// before the increment) and an acquire (the last child to arrive sees every
// sibling's records) in one atomic, instead of two full fences around it.
__device__ __forceinline__ int arrive_acq_rel(int* p) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

// Bottom-up moments: leaves sum their particles, the last child to finish
// combines its parent.  place_kernel wrote each children list in depth-first
// (= octant) order, so the combine's sums run in a fixed order and the result
// is deterministic; it loads all the children at once.
// QUAD: also the trace-free quadrupoles and the spread (the quadrupole walk,
// the correction's features); the monopole walk reads neither.
// Monopole pass at 6 blocks per SM (40 registers, a few spilled to L1): it is
// bound by the latency of its loads and of the climb, and the extra warps hide
// more of it (0.246 -> 0.228 ms at 10M); the quadrupole pass is left to the
// compiler (its moments would spill hundreds of bytes per thread at 40 or 64)
template <bool QUAD>
__global__ void __launch_bounds__(256, QUAD ? 1 : 6) moments_kernel(const float4* __restrict__ pos, Tree t,
                                                      Opening open, int* status) {
  const int total = (int)t.offset[t.n];
  for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < total;
       node += gridDim.x * blockDim.x) {
    const int4 info = t.info[node];
    if (info.z == 0) continue;  // internal nodes are finished by their last child
    if (info.z < 0 || info.y < 0 || info.y + info.z > t.n) {
      atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      continue;
    }
    Moments mo;
    {
      double m = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
      // eight particles' loads in flight at once (padding adds exact zeros, so
      // the sums are those of the plain sequential loop)
      const int end = info.y + info.z;
      for (int j0 = info.y; j0 < end; j0 += 8) {
        float4 q[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
          q[k] = j0 + k < end ? pos[j0 + k] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          m += (double)q[k].w;
          sx += (double)q[k].w * (double)q[k].x;
          sy += (double)q[k].w * (double)q[k].y;
          sz += (double)q[k].w * (double)q[k].z;
        }
      }
      mo.m = m;
      mo.cx = m != 0.0 ? sx / m : (double)pos[info.y].x;
      mo.cy = m != 0.0 ? sy / m : (double)pos[info.y].y;
      mo.cz = m != 0.0 ? sz / m : (double)pos[info.y].z;
      for (int k = 0; k < 6; ++k) mo.q[k] = 0.0;
      mo.t2 = 0.0;
#pragma unroll 4
      for (int j = info.y; QUAD && j < info.y + info.z; ++j) {
        const float4 p = pos[j];
        const double dx = (double)p.x - mo.cx, dy = (double)p.y - mo.cy, dz = (double)p.z - mo.cz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double w = (double)p.w;
        mo.t2 += w * r2;
        mo.q[0] += w * (3.0 * dx * dx - r2);
        mo.q[1] += w * (3.0 * dx * dy);
        mo.q[2] += w * (3.0 * dx * dz);
        mo.q[3] += w * (3.0 * dy * dy - r2);
        mo.q[4] += w * (3.0 * dy * dz);
        mo.q[5] += w * (3.0 * dz * dz - r2);
      }
    }
    finish_node<QUAD>(t, node, mo, info.y, t.level[node], open, info.z);
    int parent = info.w;
    for (int climb = 0; parent >= 0; ++climb) {
      if (climb > 64 || parent >= total) {  // octree depth <= 23 levels
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        break;
      }
      const int nc = __ldcg(&t.nchild[parent]);
      const int arrived = arrive_acq_rel(&t.arrive[parent]);
      if (arrived != nc - 1) break;
      if (nc < 1 || nc > 8) {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        break;
      }
      const int4 pinfo = __ldcg(&t.info[parent]);
      const int4 ca = __ldcg(reinterpret_cast<const int4*>(t.children) + 2 * parent);
      const int4 cb = __ldcg(reinterpret_cast<const int4*>(t.children) + 2 * parent + 1);
      const int ch[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
      bool bad = false;
#pragma unroll
      for (int k = 0; k < 8; ++k) bad |= k < nc && (ch[k] <= parent || ch[k] >= total);
      if (bad) {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        break;
      }
      double4 cm[8];
      int hmax = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        cm[k] = make_double4(0.0, 0.0, 0.0, 0.0);
        if (k < nc) {
          cm[k] = ldcg_d4(&t.mom[ch[k]]);
          hmax = max(hmax, __ldcg(&t.height[ch[k]]));
        }
      }
      double m = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k < nc) {
          m += cm[k].x;
          sx += cm[k].x * cm[k].y;
          sy += cm[k].x * cm[k].z;
          sz += cm[k].x * cm[k].w;
        }
      }
      Moments pm;
      pm.m = m;
      pm.cx = m != 0.0 ? sx / m : 0.0;
      pm.cy = m != 0.0 ? sy / m : 0.0;
      pm.cz = m != 0.0 ? sz / m : 0.0;
      for (int k = 0; k < 6; ++k) pm.q[k] = 0.0;
      pm.t2 = 0.0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (QUAD && k < nc) {
          const int c = ch[k];
          const double dx = cm[k].y - pm.cx, dy = cm[k].z - pm.cy, dz = cm[k].w - pm.cz;
          const double r2 = dx * dx + dy * dy + dz * dz;
          const double w = cm[k].x;
          pm.t2 += __ldcg(&t.trace64[c]) + w * r2;
          pm.q[0] += __ldcg(&t.quad64[6 * c + 0]) + w * (3.0 * dx * dx - r2);
          pm.q[1] += __ldcg(&t.quad64[6 * c + 1]) + w * (3.0 * dx * dy);
          pm.q[2] += __ldcg(&t.quad64[6 * c + 2]) + w * (3.0 * dx * dz);
          pm.q[3] += __ldcg(&t.quad64[6 * c + 3]) + w * (3.0 * dy * dy - r2);
          pm.q[4] += __ldcg(&t.quad64[6 * c + 4]) + w * (3.0 * dy * dz);
          pm.q[5] += __ldcg(&t.quad64[6 * c + 5]) + w * (3.0 * dz * dz - r2);
        }
      }
      t.height[parent] = hmax + 1;
      finish_node<QUAD>(t, parent, pm, pinfo.y, __ldcg(&t.level[parent]), open, -nc);
      parent = pinfo.w;
    }
  }
}

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

constexpr int kWalkThreads = 256;

// Warp-cooperative stackless walk: the 32 lanes own 32 Morton-consecutive
// targets and visit the same node sequence; a cell is opened when any lane's
// opening test fails (so every lane's own test holds for every cell it
// accepts), otherwise all lanes apply its multipole and skip its subtree.
// Buckets (leaves of up to leaf_capacity particles) take the same test and are
// summed particle by particle when it fails; single particles are always exact.
// Opening test of a (node, target) pair at squared distance d2 from the node's
// centre of mass: the geometric test (d2 > ro, ro = the node's opening radius
// squared) and, with REL, the relative test G M side^2 / d^4 <= alpha |a_old|,
// i.e. M side^2 <= tol d^4 with tol = alpha |a_old| / G per target (Springel
// 2001); tol = +inf (no previous acceleration) leaves the geometric test.
template <bool REL>
__device__ __forceinline__ bool opening_passes(float d2, float ro, float km, float tol) {
  return d2 > ro && (!REL || d2 * d2 * tol >= km);
}

struct WalkAcc {
  float hx, hy, hz, lx, ly, lz;  // compensated acceleration / G
  unsigned approx, exact;        // accepted cells, particle-particle terms
};

template <int ORDER, bool REL>
__device__ __forceinline__ void stackless_walk(const float4* __restrict__ pos, int n,
                                               const Tree& t, float eps2, int s, bool active,
                                               float4 p, float tol, int lane, int* status,
                                               WalkAcc& out) {
  const int total = (int)t.offset[n];
  const int limit = 2 * total + 64;

  float hx = 0.f, hy = 0.f, hz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
  float px = 0.f, py = 0.f, pz = 0.f;
  int pending = 0;
  unsigned approx = 0, exact = 0;
  int node = 0, steps = 0;
  while ((unsigned)node < (unsigned)total) {
    if (++steps > limit) {
      if (lane == 0) atomicOr(status, NBSP_DEVICE_ERROR_WALK_LIMIT);
      break;
    }
    const int4 info = t.info[node];
    if (info.z < 0 || info.y < 0 || info.y + info.z > n || info.x <= node) {
      if (lane == 0) atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      break;
    }
    // A bucket of >= 2 particles is a cell like any other: its multipole is
    // used when every lane's opening test passes (barnes_hut.c:596-599).
    bool direct = info.z == 1;
    if (info.z >= 2) {
      const float4 c = t.com[node];
      const float dx = c.x - p.x, dy = c.y - p.y, dz = c.z - p.z;
      const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      direct = __any_sync(kFull, active && !opening_passes<REL>(d2, t.ropen2[node],
                                                               REL ? t.kmass[node] : 0.f, tol));
    }
    if (direct) {
      const int j1 = info.y + info.z;
      for (int j = info.y; j < j1; ++j) {
        const float4 q = pos[j];
        const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
        const float rinv = j == s ? 0.f : rsqrt_mufu(r2);  // barnes_hut.c:572
        const float w = q.w * (rinv * rinv * rinv);
        px = fmaf(w, dx, px);
        py = fmaf(w, dy, py);
        pz = fmaf(w, dz, pz);
      }
      exact += active ? (unsigned)(info.z - ((s >= info.y && s < j1) ? 1 : 0)) : 0u;
      pending += info.z;
      node = info.x;
    } else {
      const float4 c = t.com[node];
      const float dx = c.x - p.x, dy = c.y - p.y, dz = c.z - p.z;
      const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const bool open =
          active && !opening_passes<REL>(d2, t.ropen2[node], REL ? t.kmass[node] : 0.f, tol);
      if (__any_sync(kFull, open)) {
        node = node + 1;
        continue;
      }
      const float r2 = d2 + eps2;
      const float rinv = rsqrt_mufu(r2);
      const float rinv2 = rinv * rinv;
      const float rinv3 = rinv * rinv2;
      float w = c.w * rinv3;
      if (ORDER == 2) {
        const float4 qa = t.quad[2 * node];
        const float qyz = t.quad[2 * node + 1].x;
        const float qzz = -qa.x - qa.w;
        // Q d and d.Q.d, d = com - target
        const float qdx = fmaf(qa.x, dx, fmaf(qa.y, dy, qa.z * dz));
        const float qdy = fmaf(qa.y, dx, fmaf(qa.w, dy, qyz * dz));
        const float qdz = fmaf(qa.z, dx, fmaf(qyz, dy, qzz * dz));
        const float dqd = fmaf(dx, qdx, fmaf(dy, qdy, dz * qdz));
        const float rinv5 = rinv3 * rinv2;
        const float rinv7 = rinv5 * rinv2;
        // a = G [ M d / r^3 - Q d / r^5 + 5/2 (d.Q.d) d / r^7 ]
        w = fmaf(2.5f * dqd, rinv7, w);
        px = fmaf(-qdx, rinv5, px);
        py = fmaf(-qdy, rinv5, py);
        pz = fmaf(-qdz, rinv5, pz);
      }
      px = fmaf(w, dx, px);
      py = fmaf(w, dy, py);
      pz = fmaf(w, dz, pz);
      approx += active ? 1u : 0u;
      pending += 1;
      node = info.x;
    }
    if (pending >= 32) {
      fold(hx, lx, px);
      fold(hy, ly, py);
      fold(hz, lz, pz);
      px = py = pz = 0.f;
      pending = 0;
    }
  }
  fold(hx, lx, px);
  fold(hy, ly, py);
  fold(hz, lz, pz);
  out.hx = hx;
  out.hy = hy;
  out.hz = hz;
  out.lx = lx;
  out.ly = ly;
  out.lz = lz;
  out.approx = approx;
  out.exact = exact;
}

// The compensated (hi, lo) sums combined in FP64, stored at the target's input
// index perm[s]: one aligned 32-byte record per target, so the scattered store
// writes whole sectors and the pass that scales them into the state's arrays is
// coalesced.
__device__ __forceinline__ void store_walk(const WalkAcc& a, int s, bool active, int lane,
                                           const uint32_t* __restrict__ perm, int n,
                                           double4* __restrict__ acc,
                                           unsigned long long* __restrict__ counters) {
  if (active) {
    const uint32_t i = perm[s];
    if (i < (uint32_t)n)  // (a bad permutation is flagged by the gather)
      acc[i] = make_double4((double)a.hx + (double)a.lx, (double)a.hy + (double)a.ly,
                            (double)a.hz + (double)a.lz, 0.0);
  }
  unsigned long long ap = a.approx, ex = a.exact;
  for (int off = 16; off > 0; off >>= 1) {
    ap += __shfl_down_sync(kFull, ap, off);
    ex += __shfl_down_sync(kFull, ex, off);
  }
  if (lane == 0) {
    atomicAdd(&counters[0], ap);
    atomicAdd(&counters[1], ex);
  }
}

template <int ORDER, bool REL>
__global__ void __launch_bounds__(kWalkThreads) walk_kernel(
    const float4* __restrict__ pos, const float* __restrict__ tol, int n, Tree t, float eps2,
    const uint32_t* __restrict__ perm, double4* __restrict__ acc,
    unsigned long long* __restrict__ counters, int* status) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kWalkThreads + threadIdx.x) >> 5;
  if (warp * 32 >= n) return;
  const int s = warp * 32 + lane;
  const bool active = s < n;
  const float4 p = pos[active ? s : n - 1];
  const float tl = REL ? tol[active ? s : n - 1] : 0.f;
  WalkAcc a;
  stackless_walk<ORDER, REL>(pos, n, t, eps2, s, active, p, tl, lane, status, a);
  store_walk(a, s, active, lane, perm, n, acc, counters);
}

// Point sources (bucket particles and monopole cells) gathered per warp in
// shared memory, interleaved by pairs so that one 16-byte load yields the
// 64-bit operands {x_2i, x_2i+1} and {y_2i, y_2i+1} (resp. z and m) of the
// paired .f32x2 instructions.
constexpr int kStage = 64;              // sources per tile
constexpr float kFarAway = 1e30f;       // padding: r^2 overflows to inf, rsqrt(inf) = 0
struct SourceTile {
  ulonglong2 xy[kStage / 2];  // {x_2i, x_2i+1}, {y_2i, y_2i+1}
  ulonglong2 zm[kStage / 2];  // {z_2i, z_2i+1}, {m_2i, m_2i+1}
};

__device__ __forceinline__ void stage_source(SourceTile& s, int k, float4 q) {
  float* a = reinterpret_cast<float*>(&s.xy[k >> 1]) + (k & 1);
  float* b = reinterpret_cast<float*>(&s.zm[k >> 1]) + (k & 1);
  a[0] = q.x;
  a[2] = q.y;
  b[0] = q.z;
  b[2] = q.w;
}

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

// The kStage terms of a full tile on this lane's target, two sources per
// instruction (every lane reads the same words: shared-memory broadcasts),
// summed in FP32 and folded once.  The target's own entry, when staged, has
// d = 0 and r^2 = eps^2 exactly: it adds W * 0 = 0 while its weight W = m /
// eps^3 is finite (checked once per warp by self_term_is_finite); otherwise
// GUARD drops every term with r^2 <= eps^2 (barnes_hut.c:572 skips it).
template <bool GUARD>
__device__ __forceinline__ void source_terms(const SourceTile& s, float4 p, float eps2,
                                             unsigned long long& ax, unsigned long long& ay,
                                             unsigned long long& az) {
  const unsigned long long PX = pack2(p.x, p.x), PY = pack2(p.y, p.y), PZ = pack2(p.z, p.z);
  const unsigned long long E2 = pack2(eps2, eps2);
#pragma unroll
  for (int j = 0; j < kStage / 2; ++j) {
    const ulonglong2 a = s.xy[j], b = s.zm[j];
    const unsigned long long dx = sub2(a.x, PX), dy = sub2(a.y, PY), dz = sub2(b.x, PZ);
    const unsigned long long r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
    float r2a, r2b;
    unpack2(r2, r2a, r2b);
    float ra = rsqrt_mufu(r2a), rb = rsqrt_mufu(r2b);
    if (GUARD) {
      ra = r2a > eps2 ? ra : 0.f;
      rb = r2b > eps2 ? rb : 0.f;
    }
    const unsigned long long R = pack2(ra, rb);
    const unsigned long long W = mul2(b.y, mul2(mul2(R, R), R));
    ax = fma2(W, dx, ax);
    ay = fma2(W, dy, ay);
    az = fma2(W, dz, az);
  }
}

__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// Accepted cells of the quadrupole walk, pair-interleaved like SourceTile:
// centre of mass, mass and the five independent trace-free components.
struct QuadTile {
  ulonglong2 xy[kStage / 2];         // {x}, {y}
  ulonglong2 zm[kStage / 2];         // {z}, {m}
  ulonglong2 qa[kStage / 2];         // {Qxx}, {Qxy}
  ulonglong2 qb[kStage / 2];         // {Qxz}, {Qyy}
  unsigned long long qc[kStage / 2];  // {Qyz}
};

// c = (com, mass); qa = (Qxx, Qxy, Qxz, Qyy); qyz = Qyz.
__device__ __forceinline__ void stage_cell(QuadTile& s, int k, float4 c, float4 qa, float qyz) {
  const int i = k >> 1, o = k & 1;
  float* a = reinterpret_cast<float*>(&s.xy[i]) + o;
  float* b = reinterpret_cast<float*>(&s.zm[i]) + o;
  float* e = reinterpret_cast<float*>(&s.qa[i]) + o;
  float* f = reinterpret_cast<float*>(&s.qb[i]) + o;
  a[0] = c.x;
  a[2] = c.y;
  b[0] = c.z;
  b[2] = c.w;
  e[0] = qa.x;
  e[2] = qa.y;
  f[0] = qa.z;
  f[2] = qa.w;
  reinterpret_cast<float*>(&s.qc[i])[o] = qyz;
}

// The kStage cell terms of a full QuadTile on this lane's target, two cells per
// instruction: a = G [ M d / r^3 - Q d / r^5 + 5/2 (d.Q.d) d / r^7 ],
// d = com - target, r^2 = d^2 + eps^2, Qzz = -Qxx - Qyy.  Padding cells
// (far away, massless, Q = 0) add exactly 0.
__device__ __forceinline__ void quad_tile(const QuadTile& s, float4 p, float eps2, float& hx,
                                          float& hy, float& hz, float& lx, float& ly, float& lz) {
  const unsigned long long PX = pack2(p.x, p.x), PY = pack2(p.y, p.y), PZ = pack2(p.z, p.z);
  const unsigned long long E2 = pack2(eps2, eps2), H = pack2(2.5f, 2.5f);
  const unsigned long long ZERO = 0ull;
  unsigned long long ax = 0ull, ay = 0ull, az = 0ull;
#pragma unroll 8
  for (int j = 0; j < kStage / 2; ++j) {
    const ulonglong2 a = s.xy[j], b = s.zm[j], qa = s.qa[j], qb = s.qb[j];
    const unsigned long long qyz = s.qc[j];
    const unsigned long long dx = sub2(a.x, PX), dy = sub2(a.y, PY), dz = sub2(b.x, PZ);
    const unsigned long long r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, E2)));
    float r2a, r2b;
    unpack2(r2, r2a, r2b);
    const unsigned long long R = pack2(rsqrt_mufu(r2a), rsqrt_mufu(r2b));
    const unsigned long long R2 = mul2(R, R);
    const unsigned long long R3 = mul2(R2, R);
    const unsigned long long R5 = mul2(R3, R2);
    const unsigned long long R7 = mul2(R5, R2);
    const unsigned long long qdx = fma2(qa.x, dx, fma2(qa.y, dy, mul2(qb.x, dz)));
    const unsigned long long qdy = fma2(qa.y, dx, fma2(qb.y, dy, mul2(qyz, dz)));
    const unsigned long long qdz =
        sub2(fma2(qb.x, dx, mul2(qyz, dy)), mul2(add2(qa.x, qb.y), dz));
    const unsigned long long dqd = fma2(dx, qdx, fma2(dy, qdy, mul2(dz, qdz)));
    const unsigned long long w = fma2(mul2(H, dqd), R7, mul2(b.y, R3));
    const unsigned long long nr5 = sub2(ZERO, R5);
    ax = fma2(qdx, nr5, fma2(w, dx, ax));
    ay = fma2(qdy, nr5, fma2(w, dy, ay));
    az = fma2(qdz, nr5, fma2(w, dz, az));
  }
  float u, v;
  unpack2(ax, u, v);
  fold(hx, lx, u);
  fold(hx, lx, v);
  unpack2(ay, u, v);
  fold(hy, ly, u);
  fold(hy, ly, v);
  unpack2(az, u, v);
  fold(hz, lz, u);
  fold(hz, lz, v);
}

// True when the target's own term in source_terms is W * 0 with W finite:
// eps^2 a normal number and m * rsqrt(eps^2)^3, in the same operation order,
// below overflow.
__device__ __forceinline__ bool self_term_is_finite(float m, float eps2) {
  if (!(eps2 >= 1.17549435e-38f)) return false;
  const float r = rsqrt_mufu(eps2);
  return isfinite(m * ((r * r) * r));
}

__device__ __forceinline__ void source_tile(const SourceTile& s, float4 p, float eps2, bool guard,
                                            float& hx, float& hy, float& hz, float& lx,
                                            float& ly, float& lz) {
  unsigned long long ax = 0ull, ay = 0ull, az = 0ull;  // {0.f, 0.f}
  if (guard) {
    source_terms<true>(s, p, eps2, ax, ay, az);
  } else {
    source_terms<false>(s, p, eps2, ax, ay, az);
  }
  float a, b;
  unpack2(ax, a, b);
  fold(hx, lx, a);
  fold(hx, lx, b);
  unpack2(ay, a, b);
  fold(hy, ly, a);
  fold(hy, ly, b);
  unpack2(az, a, b);
  fold(hz, lz, a);
  fold(hz, lz, b);
}

// ---------------------------------------------------------------------------
// learned far-field correction: features, training pairs, labels
// ---------------------------------------------------------------------------

// The 10 MLP inputs of cell `node` seen from point (tx, ty, tz) (coordinates
// relative to the system's centre of mass, like the node data):
//   f0..2 = (t - com) / side          f3 = side / |t - com|   (opening ratio)
//   f4..8 = trace-free Q / (M side^2): xx, xy, xz, yy, yz
//   f9    = sum m |x - com|^2 / (M side^2)
// false for a massless cell.
__device__ __forceinline__ bool features_of(float4 c, float s, float4 qa, float qyz,
                                            float spread, float tx, float ty, float tz,
                                            float* f) {
  if (!(c.w > 0.f) || !(s > 0.f)) return false;
  const float rx = tx - c.x, ry = ty - c.y, rz = tz - c.z;
  const float inv_s = 1.f / s;
  const float d = sqrtf(fmaf(rx, rx, fmaf(ry, ry, rz * rz)));
  if (!(d > 0.f)) return false;
  f[0] = rx * inv_s;
  f[1] = ry * inv_s;
  f[2] = rz * inv_s;
  f[3] = s / d;
  const float qs = 1.f / (c.w * s * s);
  f[4] = qa.x * qs;
  f[5] = qa.y * qs;
  f[6] = qa.z * qs;
  f[7] = qa.w * qs;
  f[8] = qyz * qs;
  f[9] = spread;
  return true;
}

__device__ __forceinline__ bool cell_features(const Tree& t, int node, float4 c, float tx,
                                              float ty, float tz, float* f) {
  return features_of(c, t.side[node], t.quad[2 * node], t.quad[2 * node + 1].x, t.spread[node],
                     tx, ty, tz, f);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// The corrected walk evaluates the network once per (cell, 32-target group) at
// the group centre, for cells whose distance from that centre exceeds the
// group radius / kCorrGroup.
constexpr float kCorrGroup = 0.3f;
// Training pairs are the accepted cells with side / distance >= kCorrNear x
// theta: the near cells, where the monopole's residual is largest.  The
// trained feature range then excludes the far cells, so the walk leaves them
// to the plain monopole (the fallback outside the training range); measured on
// the 1M collision at theta 1.0 this both cuts the network evaluations and
// lowers the rms error (7.7e-3 -> 5.6e-3 against 8.6e-3 uncorrected).
constexpr float kCorrNear = 0.7f;

// Training pairs: sample k picks a random target and, walking the tree with the
// opening criterion at theta_train, one of the cells that target accepts and
// its group would correct, uniformly (reservoir sampling).  Up to 8 targets
// are tried per sample.
__global__ void mlp_pairs_kernel(const float4* __restrict__ pos, int n, Tree t, float theta,
                                 int opening, unsigned long long seed, int samples, int* __restrict__ target,
                                 int* __restrict__ cell, int* status) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= samples) return;
  const int total = (int)t.offset[n];
  const float th2 = theta * theta;
  unsigned long long state = mix64(seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(k + 1)));
  int chosen = -1, tgt = 0;
  for (int attempt = 0; attempt < 8 && chosen < 0; ++attempt) {
    state = mix64(state + 0x9E3779B97F4A7C15ull);
    tgt = (int)(state % (unsigned long long)n);
    const float4 p = pos[tgt];
    // the target's walk group (32 Morton-consecutive particles): only cells
    // the corrected walk would correct for this group are sampled
    const int g0 = tgt & ~31, g1 = min(g0 + 32, n);
    float bx0 = p.x, bx1 = p.x, by0 = p.y, by1 = p.y, bz0 = p.z, bz1 = p.z;
    for (int j = g0; j < g1; ++j) {
      const float4 q = pos[j];
      bx0 = fminf(bx0, q.x);
      bx1 = fmaxf(bx1, q.x);
      by0 = fminf(by0, q.y);
      by1 = fmaxf(by1, q.y);
      bz0 = fminf(bz0, q.z);
      bz1 = fmaxf(bz1, q.z);
    }
    const float gx = 0.5f * (bx0 + bx1), gy = 0.5f * (by0 + by1), gz = 0.5f * (bz0 + bz1);
    const float ex = 0.5f * (bx1 - bx0), ey = 0.5f * (by1 - by0), ez = 0.5f * (bz1 - bz0);
    const float rg2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
    unsigned count = 0;
    int node = 0, steps = 0;
    while ((unsigned)node < (unsigned)total) {
      if (++steps > total + 64) {
        atomicOr(status, NBSP_DEVICE_ERROR_WALK_LIMIT);
        break;
      }
      const int4 info = t.info[node];
      if (info.x <= node || info.z == 1) {  // single particles are always exact
        node = info.x > node ? info.x : total;
        continue;
      }
      const float4 c = t.com[node];
      const float dx = c.x - p.x, dy = c.y - p.y, dz = c.z - p.z;
      const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const float s = t.side[node];
      const float ro = s / theta + t.shift[node];
      const bool pass = opening == NBSP_BH_OPENING_OFFSET ? d2 > ro * ro : s * s < th2 * d2;
      if (d2 > 0.f && pass && c.w > 0.f) {
        const float gdx = c.x - gx, gdy = c.y - gy, gdz = c.z - gz;
        const float near = kCorrNear * theta;
        if (kCorrGroup * kCorrGroup * fmaf(gdx, gdx, fmaf(gdy, gdy, gdz * gdz)) > rg2 &&
            s * s >= near * near * d2) {
          ++count;
          state = mix64(state + 0x9E3779B97F4A7C15ull);
          if (state % count == 0) chosen = node;
        }
        node = info.x;
      } else {
        node = info.z > 0 ? info.x : node + 1;  // a failing bucket is summed exactly
      }
    }
  }
  target[k] = tgt;
  cell[k] = chosen;
}

// Labels from exact cell sums (all-pairs arithmetic, gravity.c:46-61, FP32
// with compensated per-lane sums; target excluded): one warp per pair.
//   label = (a_exact - a_monopole) |d|^2 / M   (units of G; d = com - target)
__global__ void mlp_labels_kernel(const float4* __restrict__ pos, int n, Tree t,
                                  const int* __restrict__ target, const int* __restrict__ cell,
                                  int samples, float eps2, float* __restrict__ feat,
                                  float* __restrict__ lab, int* __restrict__ ok) {
  const int lane = threadIdx.x & 31;
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= samples) return;
  const int node = cell[k], i = target[k];
  const int total = (int)t.offset[n];
  if (node < 0 || node >= total || i < 0 || i >= n) {
    if (lane == 0) ok[k] = 0;
    return;
  }
  const int4 info = t.info[node];
  const float4 p = pos[i];
  float hx = 0.f, hy = 0.f, hz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
  // A node's particles: [its first particle, the first particle of the node
  // that follows its subtree) — or its own count for a leaf.
  const int first = info.y;
  const int end = info.z > 0 ? first + info.z : (info.x < total ? t.info[info.x].y : n);
  float px = 0.f, py = 0.f, pz = 0.f;
  int pending = 0;
  for (int j = first + lane; j < end; j += 32) {
    if (j == i) continue;
    const float4 q = pos[j];
    const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    const float rinv = rsqrt_mufu(r2);
    const float w = q.w * (rinv * rinv * rinv);
    px = fmaf(w, dx, px);
    py = fmaf(w, dy, py);
    pz = fmaf(w, dz, pz);
    if (++pending == 32) {
      fold(hx, lx, px);
      fold(hy, ly, py);
      fold(hz, lz, pz);
      px = py = pz = 0.f;
      pending = 0;
    }
  }
  fold(hx, lx, px);
  fold(hy, ly, py);
  fold(hz, lz, pz);
  double ax = (double)hx + (double)lx, ay = (double)hy + (double)ly, az = (double)hz + (double)lz;
  for (int off = 16; off > 0; off >>= 1) {
    ax += __shfl_xor_sync(kFull, ax, off);
    ay += __shfl_xor_sync(kFull, ay, off);
    az += __shfl_xor_sync(kFull, az, off);
  }
  if (lane != 0) return;
  const float4 c = t.com[node];
  float f[nbsp_mlp::kIn];
  if (!cell_features(t, node, c, p.x, p.y, p.z, f)) {
    ok[k] = 0;
    return;
  }
  const double dx = (double)c.x - p.x, dy = (double)c.y - p.y, dz = (double)c.z - p.z;
  const double d2 = dx * dx + dy * dy + dz * dz;
  const double r2 = d2 + (double)eps2;
  const double mono = (double)c.w / (r2 * sqrt(r2));
  const double scale = d2 / (double)c.w;
  for (int q = 0; q < nbsp_mlp::kIn; ++q) feat[(size_t)k * nbsp_mlp::kIn + q] = f[q];
  lab[(size_t)k * 3 + 0] = (float)((ax - mono * dx) * scale);
  lab[(size_t)k * 3 + 1] = (float)((ay - mono * dy) * scale);
  lab[(size_t)k * 3 + 2] = (float)((az - mono * dz) * scale);
  ok[k] = 1;
}

// Column statistics of the kept rows: mean, 1/std, min, max of the 10 features
// and mean, std of the 3 labels, into the network's scaling tables.
__global__ void mlp_stats_kernel(const float* __restrict__ feat, const float* __restrict__ lab,
                                 const int* __restrict__ ok, int rows, nbsp_mlp::Net* net) {
  __shared__ double sh[4][256];
  const int col = blockIdx.x;  // 0..9 features, 10..12 labels
  const float* src = col < nbsp_mlp::kIn ? feat : lab;
  const int stride = col < nbsp_mlp::kIn ? nbsp_mlp::kIn : 3;
  const int c = col < nbsp_mlp::kIn ? col : col - nbsp_mlp::kIn;
  double s = 0.0, s2 = 0.0, mn = 1e300, mx = -1e300, cnt = 0.0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    if (ok != nullptr && !ok[r]) continue;
    const double v = src[(size_t)r * stride + c];
    s += v;
    s2 += v * v;
    mn = fmin(mn, v);
    mx = fmax(mx, v);
    cnt += 1.0;
  }
  sh[0][threadIdx.x] = s;
  sh[1][threadIdx.x] = s2;
  sh[2][threadIdx.x] = cnt;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + st];
    __syncthreads();
  }
  const double tot = sh[0][0], tot2 = sh[1][0], n = sh[2][0];
  __syncthreads();
  sh[0][threadIdx.x] = mn;
  sh[1][threadIdx.x] = mx;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      sh[0][threadIdx.x] = fmin(sh[0][threadIdx.x], sh[0][threadIdx.x + st]);
      sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + st]);
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double mean = n > 0 ? tot / n : 0.0;
  const double var = n > 1 ? fmax(tot2 / n - mean * mean, 0.0) : 1.0;
  const double sd = var > 1e-30 ? sqrt(var) : 1.0;
  if (col < nbsp_mlp::kIn) {
    net->x_mean[c] = (float)mean;
    net->x_inv_std[c] = (float)(1.0 / sd);
    net->x_min[c] = (float)sh[0][0];
    net->x_max[c] = (float)sh[1][0];
  } else {
    net->y_mean[c] = (float)mean;
    net->y_std[c] = (float)sd;
  }
}

// Particle index of slot f of the concatenated buckets: the last bucket e
// with pref[e] <= f (pref: exclusive prefix of the counts, all counts >= 1).
__device__ __forceinline__ int bucket_source(const int* pref, const int2* leaves, int nleaf,
                                             int f) {
  int lo = 0, hi = nleaf - 1;
#pragma unroll
  for (int it = 0; it < 6; ++it) {  // nleaf <= 64
    const int mid = (lo + hi + 1) >> 1;
    if (lo < hi) {
      if (pref[mid] <= f) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
  }
  return leaves[lo].x + (f - pref[lo]);
}

constexpr int kListThreads = 128;  // 4 warps, one traversal group each
constexpr int kListCap = 64;       // cells / leaves gathered before a flush (>= 32 + 32)
constexpr int kListStack = 1024;   // node ids per warp (4 KiB); overflow -> stackless walk
// the relative-test walk's stack: 960 ids per warp, so that its block (with
// the tolerances' words, 24,064 B of shared memory) fits 9 times in an SM
constexpr int kListStackRel = 960;
// blocks per SM of the monopole list walks (at most 56 registers at 9): 9
// where shared memory allows (the plain and the corrected walk's block at
// 1024 ids is 24,576 B)
template <int ORDER, int STACK, bool CORR, bool REL, bool SHARED>
constexpr int list_walk_blocks() {
  return ORDER != 1 ? 5 : (!SHARED && (REL ? STACK == kListStackRel : true)) ? 9 : 8;
}
// SHARED walk: the block's top-of-tree traversal keeps its stack and frontier
// in the warps' stack space (it ends before any warp walks)
constexpr int kCtaStack = 2048;    // warps 0 and 1's stacks
constexpr int kFrontier = 384;     // the start of warp 2's stack
static_assert(kCtaStack + kFrontier <= 3 * kListStack, "frontier inside warp 2's stack");

// Interaction-list walk.  The 32 Morton-consecutive targets of a warp share a
// traversal.  Each step the lanes pop up to 32 nodes from the warp's
// shared-memory stack and test them IN PARALLEL: a node is accepted when every
// target's own reference test (2h)^2 < theta^2 d^2 holds (d to the cell's
// centre of mass) — first tried in one shot against the group's bounding box
// (if the box's nearest point passes, every target does), then against the
// lane's own target (fails: opened), else for each remaining node in turn by
// the 32 lanes testing their own targets at once — so the accepted cells are
// exactly those of the stackless walk.  An accepted monopole cell is written,
// from the registers of the lane that tested it, straight into a 64-source
// shared tile that every lane evaluates on its own target with paired f32x2
// arithmetic whenever it is full.  Buckets that must be summed exactly are
// listed (first particle, count); whenever 32 have gathered, their particles
// are gathered into the same tile, one slot per lane located by binary search
// over the counts' prefix sums, so all loads of a tile are in flight together.
// A quadrupole cell goes into a QuadTile with its moments when it is accepted.
// A warp whose stack would overflow restarts with the stackless walk.
//
// CORR: the learned far-field correction, listed here and applied by the
// correction pipeline that runs after the walk (corr_rows_kernel on the
// tcgen05 tensor cores, then corr_apply_kernel).  An accepted monopole cell
// whose opening ratio side / |com - group centre| lies in the range the
// network saw in training, and that lies further than 1/kCorrGroup group radii
// from the group centre (so one evaluation there stands for all 32 targets),
// is appended to the group's list; the walk itself computes the plain
// monopole, exactly as without the correction.
// Register budgets: monopole walk 64 (8 blocks of 4 warps per SM), quadrupole
// walk 102 (5 blocks).
//
// SHARED: the top of the tree is traversed once for the block's 4 groups.  The
// 128 threads test up to 128 nodes at a time against the 4 group boxes: a node
// every group's box test accepts is staged once for all four (into every
// warp's source tile); an internal node whose opening test fails for every
// target of every group (the box's farthest point fails) is opened once for
// all; any other node goes to a frontier that each warp then walks on its own
// exactly as above.  Every group accepts, opens and sums exactly the nodes it
// would alone (the same interactions; only the order of the FP32 sums moves).
// A block whose shared stack or frontier would overflow starts every group
// from the root instead.
template <int ORDER, int STACK, bool CORR, bool REL, bool SHARED = false>
__global__ void __launch_bounds__(kListThreads, (list_walk_blocks<ORDER, STACK, CORR, REL, SHARED>())) walk_lists_kernel(
    const float4* __restrict__ pos, const float* __restrict__ tol, int n, Tree t, float eps2,
    const uint32_t* __restrict__ perm, double4* __restrict__ acc,
    unsigned long long* __restrict__ counters, int* status,
    const nbsp_mlp::Net* __restrict__ net, NbspCorrectionLists lists) {
  static_assert(!SHARED || (ORDER == 1 && !CORR && STACK == kListStack), "shared top: monopole walk");
  __shared__ int s_stack[kListThreads / 32][STACK];
  __shared__ float s_probe_k[kListThreads / 32][REL ? 32 : 1];  // their M side^2
  // nodes awaiting per-target tests during a step; the same words hold the
  // exclusive prefix of the bucket counts during a bucket flush (the two
  // phases of an iteration never overlap: a __syncwarp ends each)
  __shared__ float4 s_probe[kListThreads / 32][32];
  static_assert(sizeof(s_probe[0]) >= kListCap * sizeof(int), "prefix fits the probe words");
  __shared__ int2 s_leaves[kListThreads / 32][kListCap];  // (first particle, count)
  // ORDER 1: accepted cells are point masses in the source tile; ORDER 2:
  // cells fill a QuadTile
  static_assert(!(CORR && ORDER == 2), "the network corrects the monopole");
  __shared__ __align__(16) SourceTile s_src[kListThreads / 32];
  __shared__ __align__(16) QuadTile s_quad[ORDER == 2 ? kListThreads / 32 : 1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  SourceTile& src = s_src[wib];
  int staged = 0;   // sources waiting in src (warp-uniform)
  int listed = 0;   // corrected walk: cells listed for the network (warp-uniform)
  int qstaged = 0;  // cells waiting in the QuadTile (ORDER 2)
  const int warp = (blockIdx.x * kListThreads + threadIdx.x) >> 5;
  const bool live = warp * 32 < n;  // (a SHARED block's idle warps join its shared phase)
  if (!SHARED && !live) return;
  int* stack = s_stack[wib];
  int2* leaves = s_leaves[wib];
  const int s = warp * 32 + lane;
  const bool active = s < n;
  const float4 p = pos[active ? s : n - 1];
  const unsigned lt = (1u << lane) - 1u;
  const bool guard = !__all_sync(kFull, !active || self_term_is_finite(p.w, eps2));
  // relative test: this lane's tolerance and the group's smallest (the box
  // test stands for every target only with the least tolerant one)
  float tl = REL && active ? tol[s] : INFINITY, tmin = tl;
  if (REL)
    for (int off = 16; off > 0; off >>= 1) tmin = fminf(tmin, __shfl_xor_sync(kFull, tmin, off));

  // group bounding box
  float bx0 = p.x, bx1 = p.x, by0 = p.y, by1 = p.y, bz0 = p.z, bz1 = p.z;
  for (int off = 16; off > 0; off >>= 1) {
    bx0 = fminf(bx0, __shfl_xor_sync(kFull, bx0, off));
    bx1 = fmaxf(bx1, __shfl_xor_sync(kFull, bx1, off));
    by0 = fminf(by0, __shfl_xor_sync(kFull, by0, off));
    by1 = fmaxf(by1, __shfl_xor_sync(kFull, by1, off));
    bz0 = fminf(bz0, __shfl_xor_sync(kFull, bz0, off));
    bz1 = fmaxf(bz1, __shfl_xor_sync(kFull, bz1, off));
  }
  const float gx = 0.5f * (bx0 + bx1), gy = 0.5f * (by0 + by1), gz = 0.5f * (bz0 + bz1);
  const float ex = 0.5f * (bx1 - bx0), ey = 0.5f * (by1 - by0), ez = 0.5f * (bz1 - bz0);
  const float rg2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));  // group radius^2
  if (CORR && lane == 0) reinterpret_cast<float4*>(lists.centre)[warp] = make_float4(gx, gy, gz, rg2);

  const int total = (int)t.offset[n];
  float hx = 0.f, hy = 0.f, hz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
  unsigned approx = 0, exact = 0;
  int top = 1, nleaf = 0, iters = 0;
  bool overflow = false;
  if (SHARED) {
    constexpr int kGroups = kListThreads / 32;
    __shared__ float s_box[kGroups][8];  // centre, half extents, least and most tolerant
    __shared__ int s_live[kGroups];
    __shared__ int s_sum[kGroups][3];    // per warp: accepted, children, frontier nodes
    __shared__ int s_ctop, s_nfront, s_abort;
    int* cstack = &s_stack[0][0];
    int* front = &s_stack[0][0] + kCtaStack;
    float tmax = REL && active ? tl : -INFINITY;
    if (REL)
      for (int off = 16; off > 0; off >>= 1) tmax = fmaxf(tmax, __shfl_xor_sync(kFull, tmax, off));
    if (lane == 0) {
      s_box[wib][0] = gx;
      s_box[wib][1] = gy;
      s_box[wib][2] = gz;
      s_box[wib][3] = ex;
      s_box[wib][4] = ey;
      s_box[wib][5] = ez;
      s_box[wib][6] = tmin;
      s_box[wib][7] = tmax;
      s_live[wib] = live;
    }
    if (threadIdx.x == 0) {
      s_ctop = 1;
      cstack[0] = 0;
      s_nfront = 0;
      s_abort = 0;
    }
    __syncthreads();
    for (int csteps = 0;; ++csteps) {
      const int ctop = s_ctop;  // block-uniform: read after a barrier
      if (ctop == 0 || s_abort) break;
      if (csteps > total + 64) {  // every node is popped at most once
        if (threadIdx.x == 0) atomicOr(status, NBSP_DEVICE_ERROR_WALK_LIMIT);
        break;
      }
      const int take = min(kListThreads, ctop);
      int node = (int)threadIdx.x < take ? cstack[ctop - 1 - threadIdx.x] : -1;
      if (node >= total) {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        node = -1;
      }
      const bool valid = node >= 0;
      const int at = valid ? node : 0;
      const float4 w0 = t.wnode[2 * at], w1 = t.wnode[2 * at + 1];
      const int4 info = make_int4(0, __float_as_int(w1.z), __float_as_int(w1.w), 0);
      const float4 c = w0;
      const float ro = w1.x;
      const float km = REL ? w1.y : 0.f;
      const bool bad = valid && info.z > 0 && (info.y < 0 || info.y + info.z > n);
      if (bad) atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
      const bool ok = valid && !bad;
      bool all_accept = ok && info.z != 1, all_open = ok && info.z < 0;
#pragma unroll
      for (int w = 0; w < kGroups; ++w) {
        if (!s_live[w]) continue;
        const float ax = fabsf(c.x - s_box[w][0]), ay = fabsf(c.y - s_box[w][1]),
                    az = fabsf(c.z - s_box[w][2]);
        const float qx = fmaxf(ax - s_box[w][3], 0.f), qy = fmaxf(ay - s_box[w][4], 0.f),
                    qz = fmaxf(az - s_box[w][5], 0.f);
        const float fx = ax + s_box[w][3], fy = ay + s_box[w][4], fz = az + s_box[w][5];
        const float dmin2 = fmaf(qx, qx, fmaf(qy, qy, qz * qz));
        const float dmax2 = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
        all_accept = all_accept && opening_passes<REL>(dmin2, ro, km, s_box[w][6]);
        all_open = all_open && (dmax2 <= ro || (REL && dmax2 * dmax2 * s_box[w][7] < km));
      }
      const bool to_front = ok && !all_accept && !all_open;
      int4 ca = make_int4(-1, -1, -1, -1), cb = make_int4(-1, -1, -1, -1);
      if (all_open) {
        ca = reinterpret_cast<const int4*>(t.children)[2 * node];
        cb = reinterpret_cast<const int4*>(t.children)[2 * node + 1];
      }
      const int kids = (ca.x >= 0) + (ca.y >= 0) + (ca.z >= 0) + (ca.w >= 0) + (cb.x >= 0) +
                       (cb.y >= 0) + (cb.z >= 0) + (cb.w >= 0);
      // block-wide exclusive prefixes of the three counts
      int ia = all_accept, ik = kids, ifr = to_front;
      for (int off = 1; off < 32; off <<= 1) {
        const int ua = __shfl_up_sync(kFull, ia, off), uk = __shfl_up_sync(kFull, ik, off),
                  uf = __shfl_up_sync(kFull, ifr, off);
        if (lane >= off) {
          ia += ua;
          ik += uk;
          ifr += uf;
        }
      }
      if (lane == 31) {
        s_sum[wib][0] = ia;
        s_sum[wib][1] = ik;
        s_sum[wib][2] = ifr;
      }
      __syncthreads();  // (every entry popped above has been read)
      int ba = 0, bk = 0, bf = 0, na = 0, nk = 0, nf = 0;
#pragma unroll
      for (int w = 0; w < kGroups; ++w) {
        if (w < wib) {
          ba += s_sum[w][0];
          bk += s_sum[w][1];
          bf += s_sum[w][2];
        }
        na += s_sum[w][0];
        nk += s_sum[w][1];
        nf += s_sum[w][2];
      }
      const int ra = ba + ia - (int)all_accept, rk = bk + ik - kids, rf = bf + ifr - (int)to_front;
      const int cbase = ctop - take, front0 = s_nfront;
      const bool abort = cbase + nk > kCtaStack || front0 + nf > kFrontier;  // block-uniform
      if (!abort) {
        const int kid[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (k < kids) cstack[cbase + rk + k] = kid[k];
        if (to_front) front[front0 + rf] = node;
        // cells every group accepts: into every live warp's source tile, in
        // rounds of what fits before the tiles are evaluated
        approx += (unsigned)na;
        for (int done = 0; done < na;) {
          const int put = min(kStage - staged, na - done);
          const int r = ra - done;
          if (all_accept && r >= 0 && r < put)
#pragma unroll
            for (int w = 0; w < kGroups; ++w)
              if (s_live[w]) stage_source(s_src[w], staged + r, c);
          staged += put;
          done += put;
          __syncthreads();
          if (staged == kStage) {
            if (live) source_tile(src, p, eps2, guard, hx, hy, hz, lx, ly, lz);
            staged = 0;
            __syncthreads();
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        if (abort) {
          s_abort = 1;
        } else {
          s_ctop = cbase + nk;
          s_nfront = front0 + nf;
        }
      }
      __syncthreads();
    }
    const int nfront = s_nfront;
    const bool restart = s_abort != 0;
    __syncthreads();  // the shared stack's last reads
    if (restart) {  // start every group from the root, discarding the shared phase
      hx = hy = hz = lx = ly = lz = 0.f;
      approx = 0;
      staged = 0;
      top = 1;
      if (lane == 0) stack[0] = 0;
    } else {
      for (int k = lane; k < nfront; k += 32) stack[k] = front[k];
      top = nfront;
    }
    __syncthreads();  // warp 2's copy is in place before any warp walks
    if (!live) return;
  } else if (lane == 0) {
    stack[0] = 0;
  }
  __syncwarp();
  // (staged > 0 with nothing left to walk: cells the shared phase staged; the
  // draining iteration evaluates them)
  for (;;) {  // until the stack, the bucket list and the tiles are drained
    if (top > 0) {
      if (++iters > total + 64) {  // every node is popped at most once
        if (lane == 0) atomicOr(status, NBSP_DEVICE_ERROR_WALK_LIMIT);
        break;
      }
      const int take = min(32, top);
      int node = lane < take ? stack[top - 1 - lane] : -1;
      top -= take;
      __syncwarp();
      bool is_leaf = false, accept = false, test = false;
      int kids = 0;
      int4 info = make_int4(0, 0, 0, 0);
      float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
      float ro = 0.f, km = 0.f;
      int4 ca = make_int4(-1, -1, -1, -1), cb = make_int4(-1, -1, -1, -1);
      if (node >= total) {
        atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        node = -1;
      }
      {  // every lane loads a node (idle lanes the root) so no branch diverges
        const bool valid = node >= 0;
        const int at = valid ? node : 0;
        // one 32-byte record: the centre of mass and mass, the opening terms
        // and the particle range (the node's next and parent links are not read)
        const float4 w0 = __ldg(&t.wnode[2 * at]), w1 = __ldg(&t.wnode[2 * at + 1]);
        c = w0;
        ro = w1.x;
        if (REL) km = w1.y;
        info.y = __float_as_int(w1.z);
        info.z = __float_as_int(w1.w);
        const bool bad = valid && info.z > 0 && (info.y < 0 || info.y + info.z > n);
        if (bad) atomicOr(status, NBSP_DEVICE_ERROR_TREE_INCONSISTENT);
        const bool ok = valid && !bad;
        is_leaf = ok && info.z == 1;
        const float qx = fmaxf(fabsf(c.x - gx) - ex, 0.f);
        const float qy = fmaxf(fabsf(c.y - gy) - ey, 0.f);
        const float qz = fmaxf(fabsf(c.z - gz) - ez, 0.f);
        const float dmin2 = fmaf(qx, qx, fmaf(qy, qy, qz * qz));
        const bool cellish = ok && info.z != 1;
        const bool box = opening_passes<REL>(dmin2, ro, km, tmin);
        accept = cellish && box;
        test = cellish && !box;
      }
      // Nodes the box could not accept: a node that fails this lane's own
      // target is opened at once; for the rest every target's own test
      // decides, one node at a time with the 32 targets tested in parallel.
      const float d2own = fmaf(c.x - p.x, c.x - p.x, fmaf(c.y - p.y, c.y - p.y, (c.z - p.z) * (c.z - p.z)));
      const bool opened = test && active && !opening_passes<REL>(d2own, ro, km, tl);
      test = test && !opened;
      float4* probe = s_probe[wib];
      if (test) probe[lane] = make_float4(c.x, c.y, c.z, ro);
      if (REL && test) s_probe_k[wib][lane] = km;
      __syncwarp();
      for (unsigned pend = __ballot_sync(kFull, test); pend != 0u; pend &= pend - 1u) {
        const int from = __ffs(pend) - 1;
        const float4 q = probe[from];
        const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        const bool fail = active && !opening_passes<REL>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), q.w,
                                                         REL ? s_probe_k[wib][from] : 0.f, tl);
        const bool any = __any_sync(kFull, fail);
        if (lane == from) accept = !any;
      }
      const bool open = (test || opened) && !accept;
      is_leaf = is_leaf || (open && info.z > 0);  // a failing bucket is summed exactly
      if (open && info.z < 0) {                    // an opened cell pushes its -info.z children
        ca = __ldg(reinterpret_cast<const int4*>(t.children) + 2 * node);
        cb = __ldg(reinterpret_cast<const int4*>(t.children) + 2 * node + 1);
        kids = min(-info.z, 8);
      }
      unsigned m = __ballot_sync(kFull, is_leaf);
      if (is_leaf) leaves[nleaf + __popc(m & lt)] = make_int2(info.y, info.z);
      nleaf += __popc(m);
      {  // targets whose own particle is in one of these buckets: one term fewer
        // (only the group's own buckets overlap its targets: a vote first)
        const int lo = max(info.y - warp * 32, 0), hi = min(info.y + info.z - warp * 32, 32);
        if (__any_sync(kFull, is_leaf && hi > lo)) {
          const unsigned span = hi >= 32 ? kFull : (1u << max(hi, 0)) - 1u;
          const unsigned own = __reduce_or_sync(
              kFull, is_leaf && hi > lo ? span & ~((1u << min(lo, 31)) - 1u) : 0u);
          if (active && ((own >> lane) & 1u)) exact -= 1u;
        }
      }
      m = __ballot_sync(kFull, accept);
      if (ORDER == 1) {
        // A monopole cell is a point mass at its centre of mass, already in
        // this lane's registers from the opening test: it goes straight into
        // the source tile (evaluated whenever 64 sources have gathered).  The
        // corrected walk also lists the cell for its network evaluation.
        if (CORR) {
          bool listme = false;
          if (accept) {
            const float side = t.side[node];
            const float gdx = c.x - gx, gdy = c.y - gy, gdz = c.z - gz;
            const float dg2 = fmaf(gdx, gdx, fmaf(gdy, gdy, gdz * gdz));
            const float lo = __ldg(&net->x_min[3]), hi = __ldg(&net->x_max[3]);
            listme = kCorrGroup * kCorrGroup * dg2 > rg2 && side * side >= lo * lo * dg2 &&
                     side * side <= hi * hi * dg2;
          }
          const unsigned lm = __ballot_sync(kFull, listme);
          const int at = listed + __popc(lm & lt);
          if (listme && at < lists.capacity) lists.cells[(size_t)warp * lists.capacity + at] = node;
          listed += __popc(lm);
        }
        const int nacc = __popc(m), rank = __popc(m & lt), room = kStage - staged;
        if (accept && rank < room) stage_source(src, staged + rank, c);
        if (nacc >= room) {
          __syncwarp();
          source_tile(src, p, eps2, guard, hx, hy, hz, lx, ly, lz);
          __syncwarp();
          if (accept && rank >= room) stage_source(src, rank - room, c);
          staged = nacc - room;
        } else {
          staged += nacc;
        }
        approx += (unsigned)nacc;  // (warp-uniform; an idle lane's is dropped at the end)
      } else {  // a quadrupole cell goes into the QuadTile with its moments
        QuadTile& qt = s_quad[ORDER == 2 ? wib : 0];
        float4 qa = make_float4(0.f, 0.f, 0.f, 0.f);
        float qyz = 0.f;
        if (accept) {
          qa = t.quad[2 * node];
          qyz = t.quad[2 * node + 1].x;
        }
        const int nacc = __popc(m), rank = __popc(m & lt), room = kStage - qstaged;
        if (accept && rank < room) stage_cell(qt, qstaged + rank, c, qa, qyz);
        if (nacc >= room) {
          __syncwarp();
          quad_tile(qt, p, eps2, hx, hy, hz, lx, ly, lz);
          __syncwarp();
          if (accept && rank >= room) stage_cell(qt, rank - room, c, qa, qyz);
          qstaged = nacc - room;
        } else {
          qstaged += nacc;
        }
        approx += (unsigned)nacc;  // (warp-uniform; an idle lane's is dropped at the end)
      }
      int incl = kids;
      for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(kFull, incl, off);
        if (lane >= off) incl += v;
      }
      const int pushed = __shfl_sync(kFull, incl, 31);
      if (top + pushed > STACK) {
        overflow = true;
        break;
      }
      const int base = top + incl - kids;
      const int kid[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k < kids) stack[base + k] = kid[k];
      top += pushed;
      __syncwarp();
    }
    const bool drain = top == 0;
    if (nleaf >= 32 || (drain && nleaf > 0)) {
      // The buckets' particles, concatenated, fill the tile: each lane finds
      // the bucket of its slot by binary search over the exclusive prefix of
      // the counts and loads its particles, all loads of a tile in flight at
      // once.  The target's own particle adds exactly 0 (d = 0).
      int* pref = reinterpret_cast<int*>(s_probe[wib]);
      const int c0 = lane < nleaf ? leaves[lane].y : 0;
      const int c1 = lane + 32 < nleaf ? leaves[lane + 32].y : 0;
      int i0 = c0, i1 = c1;
      for (int off = 1; off < 32; off <<= 1) {
        const int v0 = __shfl_up_sync(kFull, i0, off), v1 = __shfl_up_sync(kFull, i1, off);
        if (lane >= off) {
          i0 += v0;
          i1 += v1;
        }
      }
      i1 += __shfl_sync(kFull, i0, 31);
      const int total_src = __shfl_sync(kFull, i1, 31);
      if (lane < nleaf) pref[lane] = i0 - c0;
      if (lane + 32 < nleaf) pref[lane + 32] = i1 - c1;
      __syncwarp();
      exact += active ? (unsigned)total_src : 0u;  // own particles were taken off above
      for (int f0 = 0; f0 < total_src;) {
        const int take = min(total_src - f0, kStage - staged);
        const bool h0 = lane < take, h1 = lane + 32 < take;
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = q0;
        if (h0) q0 = pos[bucket_source(pref, leaves, nleaf, f0 + lane)];
        if (h1) q1 = pos[bucket_source(pref, leaves, nleaf, f0 + lane + 32)];
        if (h0) stage_source(src, staged + lane, q0);
        if (h1) stage_source(src, staged + lane + 32, q1);
        staged += take;
        f0 += take;
        if (staged == kStage) {
          __syncwarp();
          source_tile(src, p, eps2, guard, hx, hy, hz, lx, ly, lz);
          staged = 0;
          __syncwarp();
        }
      }
      nleaf = 0;
    }
    if (drain && staged > 0) {  // the last, partial tile: pad with massless far sources
      for (int k = staged + lane; k < kStage; k += 32)
        stage_source(src, k, make_float4(kFarAway, kFarAway, kFarAway, 0.f));
      __syncwarp();
      source_tile(src, p, eps2, guard, hx, hy, hz, lx, ly, lz);
      staged = 0;
    }
    if (ORDER == 2 && drain && qstaged > 0) {  // the same for the last cells
      QuadTile& qt = s_quad[ORDER == 2 ? wib : 0];
      for (int k = qstaged + lane; k < kStage; k += 32)
        stage_cell(qt, k, make_float4(kFarAway, kFarAway, kFarAway, 0.f),
                   make_float4(0.f, 0.f, 0.f, 0.f), 0.f);
      __syncwarp();
      quad_tile(qt, p, eps2, hx, hy, hz, lx, ly, lz);
      qstaged = 0;
    }
    __syncwarp();
    if (drain) break;
  }
  if (CORR && lane == 0) {  // a group walked again keeps the plain monopole
    lists.count[warp] = overflow ? 0 : min(listed, lists.capacity);
    if (!overflow && listed > lists.capacity)
      atomicAdd(&counters[7], (unsigned long long)(listed - lists.capacity));
  }
  WalkAcc a;
  if (overflow) {
    if (lane == 0) atomicAdd(&counters[5], 1ull);  // groups walked again
    stackless_walk<ORDER, REL>(pos, n, t, eps2, s, active, p, tl, lane, status, a);
  } else {
    a.hx = hx;
    a.hy = hy;
    a.hz = hz;
    a.lx = lx;
    a.ly = ly;
    a.lz = lz;
    a.approx = active ? approx : 0u;
    a.exact = exact;
  }
  store_walk(a, s, active, lane, perm, n, acc, counters);
}

// ---- the correction pipeline after a corrected walk ------------------------
//
// 1. corr_scan_kernel: exclusive prefix of the per-group list lengths (one
//    row per listed (cell, group) pair, groups in order);
// 2. corr_rows_kernel: every row's 10 features at its group centre, the
//    network on 128-row tiles on the tcgen05 tensor cores, the de-standardised
//    output (zero for features outside the training range: the plain
//    monopole, the fallback);
// 3. corr_apply_kernel: one warp per group adds (M / |d|^2) * y of its rows,
//    in list order, to each target's walk result (deterministic).

__global__ void __launch_bounds__(1024) corr_scan_kernel(NbspCorrectionLists lists, int groups,
                                                         unsigned long long* counters) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < groups; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < groups ? lists.count[i] : 0;
    int x = v;
    for (int off = 1; off < 32; off <<= 1) {
      const int u = __shfl_up_sync(kFull, x, off);
      if (lane >= off) x += u;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = warp_sums[lane];
      for (int off = 1; off < 32; off <<= 1) {
        const int u = __shfl_up_sync(kFull, w, off);
        if (lane >= off) w += u;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const int incl = x + (wid > 0 ? warp_sums[wid - 1] : 0);
    const int c = carry;
    if (i < groups) lists.offset[i] = c + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = c + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    lists.offset[groups] = carry;
    atomicAdd(&counters[6], (unsigned long long)carry);  // network evaluations
  }
}

// Row r -> (its group, its cell), one warp per group: the rows kernel reads
// both with one 8-byte load and needs no search.
__global__ void __launch_bounds__(128) corr_rowmap_kernel(NbspCorrectionLists lists, int groups) {
  const int lane = threadIdx.x & 31;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= groups) return;
  const int cnt = lists.count[g], off = lists.offset[g];
  int2* rows = reinterpret_cast<int2*>(lists.row);
  for (int k = lane; k < cnt; k += 32)
    rows[off + k] = make_int2(g, lists.cells[(size_t)g * lists.capacity + k]);
}

// What the features of one row are computed from, loaded one tile ahead so the
// loads are in flight while the tensor cores run the current tile.
struct RowData {
  float4 c;    // cell centre of mass, mass
  float4 g;    // group centre, radius^2
  float4 qa;   // quadrupole xx, xy, xz, yy
  float qyz, side, spread;
  bool valid;
};

__device__ __forceinline__ RowData load_row(const Tree& t, const float4* centre, int2 gn,
                                            bool valid) {
  RowData d;
  d.valid = valid;
  const int node = valid ? gn.y : 0, grp = valid ? gn.x : 0;
  d.c = t.com[node];
  d.g = centre[grp];
  d.qa = t.quad[2 * node];
  d.qyz = t.quad[2 * node + 1].x;
  d.side = t.side[node];
  d.spread = t.spread[node];
  return d;
}

__global__ void __launch_bounds__(nbsp_umma::kThreads) corr_rows_kernel(
    const nbsp_mlp::Net* __restrict__ net, Tree t, NbspCorrectionLists lists, int groups,
    int* status) {
  extern __shared__ __align__(128) unsigned char umma_smem[];
  nbsp_umma::Smem& sm = *reinterpret_cast<nbsp_umma::Smem*>(umma_smem);
  nbsp_umma::setup(sm, nbsp_umma::weights_of(net), net);
  const uint32_t tmem = sm.tmem;
  uint32_t phase = 0;
  const int rows = lists.offset[groups];
  const int tiles = (rows + nbsp_umma::kRows - 1) / nbsp_umma::kRows;
  const float4* centre = reinterpret_cast<const float4*>(lists.centre);
  const int2* rowmap = reinterpret_cast<const int2*>(lists.row);
  const int stride = gridDim.x * nbsp_umma::kRows;
  // pipeline: the row map two tiles ahead, the row data one tile ahead
  int r = blockIdx.x * nbsp_umma::kRows + threadIdx.x;
  RowData cur = load_row(t, centre, r < rows ? rowmap[r] : make_int2(0, 0), r < rows);
  int2 ahead = r + stride < rows ? rowmap[r + stride] : make_int2(0, 0);
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, r += stride) {
    float v[nbsp_mlp::kIn];
    bool ok = false;
    if (cur.valid) {
      float f[nbsp_mlp::kIn];
      ok = features_of(cur.c, cur.side, cur.qa, cur.qyz, cur.spread, cur.g.x, cur.g.y, cur.g.z,
                       f);
#pragma unroll
      for (int q = 0; q < nbsp_mlp::kIn; ++q) {
        ok = ok && f[q] >= net->x_min[q] && f[q] <= net->x_max[q];
        v[q] = (f[q] - net->x_mean[q]) * net->x_inv_std[q];
      }
    }
    if (!ok)
#pragma unroll
      for (int q = 0; q < nbsp_mlp::kIn; ++q) v[q] = 0.f;
    nbsp_umma::put_inputs(sm, v);
    nbsp_umma::fence_async_smem();
    __syncthreads();
    const RowData next = load_row(t, centre, ahead, r + stride < rows);
    ahead = r + 2 * stride < rows ? rowmap[r + 2 * stride] : make_int2(0, 0);
    float y[3];
    if (!nbsp_umma::forward(sm, tmem, phase, y)) {
      if (threadIdx.x == 0) atomicOr(status, NBSP_DEVICE_ERROR_MMA_TIMEOUT);
      break;
    }
    if (r < rows)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        lists.y[(size_t)r * 3 + c] = ok ? fmaf(y[c], net->y_std[c], net->y_mean[c]) : 0.f;
    cur = next;
  }
  nbsp_umma::teardown(sm, tmem);
}

__global__ void __launch_bounds__(128) corr_apply_kernel(const float4* __restrict__ pos, int n,
                                                         Tree t, NbspCorrectionLists lists,
                                                         const uint32_t* __restrict__ perm,
                                                         double4* __restrict__ acc) {
  const int lane = threadIdx.x & 31;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g * 32 >= n) return;
  const int s = g * 32 + lane;
  const bool active = s < n;
  const float4 p = pos[active ? s : n - 1];
  const int cnt = lists.count[g], off = lists.offset[g];
  float hx = 0.f, hy = 0.f, hz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
  for (int i0 = 0; i0 < cnt; i0 += 32) {
    const int k = i0 + lane;
    float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
    float yx = 0.f, yy = 0.f, yz = 0.f;
    if (k < cnt) {
      c = t.com[lists.cells[(size_t)g * lists.capacity + k]];
      const float* y = &lists.y[(size_t)(off + k) * 3];
      yx = c.w * y[0];
      yy = c.w * y[1];
      yz = c.w * y[2];
    }
    float ax = 0.f, ay = 0.f, az = 0.f;
    const int take = min(32, cnt - i0);
    for (int j = 0; j < take; ++j) {
      const float cx = __shfl_sync(kFull, c.x, j), cy = __shfl_sync(kFull, c.y, j);
      const float cz = __shfl_sync(kFull, c.z, j);
      const float Yx = __shfl_sync(kFull, yx, j), Yy = __shfl_sync(kFull, yy, j);
      const float Yz = __shfl_sync(kFull, yz, j);
      const float dx = cx - p.x, dy = cy - p.y, dz = cz - p.z;
      const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      const float r = d2 > 0.f ? rsqrt_mufu(d2) : 0.f;
      const float w = r * r;
      ax = fmaf(w, Yx, ax);
      ay = fmaf(w, Yy, ay);
      az = fmaf(w, Yz, az);
    }
    fold(hx, lx, ax);
    fold(hy, ly, ay);
    fold(hz, lz, az);
  }
  if (active && cnt > 0) {  // the walk stored the target at its input index
    const uint32_t i = perm[s];
    if (i < (uint32_t)n) {
      double4 a = acc[i];
      a.x += (double)hx + (double)lx;
      a.y += (double)hy + (double)ly;
      a.z += (double)hz + (double)lz;
      acc[i] = a;
    }
  }
}

__global__ void tree_counts_kernel(Tree t, unsigned long long* counters) {
  if (threadIdx.x != 0) return;
  counters[2] = t.offset[t.n];
  counters[3] = *t.leaves;
  counters[4] = (unsigned long long)t.height[0];
}

int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return (int)b;
}

template <bool REL>
void launch_walk(const float4* p, const float* tol, size_t n, Tree t, int order, int mode,
                 const nbsp_mlp::Net* net, const NbspCorrectionLists* lists, float eps2,
                 const uint32_t* perm, double4* out, unsigned long long* counters, int* status,
                 cudaStream_t stream) {
  if (mode == NBSP_BH_WALK_LISTS || mode == NBSP_BH_WALK_SHARED || net != nullptr) {
    const unsigned blocks = (unsigned)((n + kListThreads - 1) / kListThreads);
    NbspCorrectionLists none{};
    if (net != nullptr && lists != nullptr) {  // the network corrects the monopole term
      NBSP_COUNT_LAUNCH(1), walk_lists_kernel<1, kListStack, true, REL><<<blocks, kListThreads, 0, stream>>>(
          p, tol, (int)n, t, eps2, perm, out, counters, status, net, *lists);
    } else if (order == 1 && mode == NBSP_BH_WALK_SHARED) {
      NBSP_COUNT_LAUNCH(1), walk_lists_kernel<1, kListStack, false, REL, true><<<blocks, kListThreads, 0, stream>>>(
          p, tol, (int)n, t, eps2, perm, out, counters, status, nullptr, none);
    } else if (order == 2) {
      NBSP_COUNT_LAUNCH(1), walk_lists_kernel<2, kListStack, false, REL><<<blocks, kListThreads, 0, stream>>>(
          p, tol, (int)n, t, eps2, perm, out, counters, status, nullptr, none);
    } else {
      constexpr int kStack = REL ? kListStackRel : kListStack;
      NBSP_COUNT_LAUNCH(1), walk_lists_kernel<1, kStack, false, REL><<<blocks, kListThreads, 0, stream>>>(
          p, tol, (int)n, t, eps2, perm, out, counters, status, nullptr, none);
    }
    return;
  }
  const unsigned blocks = (unsigned)((n + kWalkThreads - 1) / kWalkThreads);
  if (order == 2) {
    NBSP_COUNT_LAUNCH(1), walk_kernel<2, REL><<<blocks, kWalkThreads, 0, stream>>>(
        p, tol, (int)n, t, eps2, perm, out, counters, status);
  } else {
    NBSP_COUNT_LAUNCH(1), walk_kernel<1, REL><<<blocks, kWalkThreads, 0, stream>>>(
        p, tol, (int)n, t, eps2, perm, out, counters, status);
  }
}

}  // namespace

extern "C" {

void nbsp_bh_bounds(double* x, double* y, double* z, const double* m, size_t n, double* partial,
                    double* geometry, int* status, const double* ax, const double* ay,
                    const double* az, int rms_of_a, const NbspLeapfrogFusion* leapfrog,
                    cudaStream_t stream) {
  size_t blocks = (n + kBoundsThreads - 1) / kBoundsThreads;
  if (blocks < 1) blocks = 1;
  if (blocks > (size_t)kBoundsBlocks) blocks = kBoundsBlocks;
  if (leapfrog != nullptr && leapfrog->vx != nullptr) {
    NBSP_COUNT_LAUNCH(1), bounds_kernel<true><<<(unsigned)blocks, kBoundsThreads, 0, stream>>>(
        x, y, z, m, n, partial, status, ax, ay, az, rms_of_a != 0, leapfrog->vx, leapfrog->vy,
        leapfrog->vz, leapfrog->half_dt, leapfrog->dt);
  } else {
    NBSP_COUNT_LAUNCH(1), bounds_kernel<false><<<(unsigned)blocks, kBoundsThreads, 0, stream>>>(
        x, y, z, m, n, partial, status, ax, ay, az, rms_of_a != 0, nullptr, nullptr, nullptr,
        0.0, 0.0);
  }
  NBSP_COUNT_LAUNCH(1), bounds_final_kernel<<<1, kBoundsThreads, 0, stream>>>(partial, (int)blocks,
                                                                            n, geometry);
}

size_t nbsp_bh_sort_scratch_words(size_t n) { return sort_scratch_words(n); }

void nbsp_bh_keys(const double* x, const double* y, const double* z, const double* m, size_t n,
                  const double* geometry, uint64_t* keys, uint32_t* index, void* unsorted,
                  uint32_t* scratch, const double* ax, const double* ay, const double* az,
                  double tol_scale, float* unsorted_tol, cudaStream_t stream) {
  cudaMemsetAsync(scratch, 0, sort_scratch_words(n) * sizeof(uint32_t), stream);
  const SortScratch sc = sort_scratch(scratch, n);
  size_t blocks = (n + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > (size_t)kKeysBlocks) blocks = kKeysBlocks;
  NBSP_COUNT_LAUNCH(1), keys_kernel<<<(unsigned)blocks, 256, 0, stream>>>(
      x, y, z, m, n, geometry, keys, index, (float4*)unsorted, sc.hist, ax, ay, az, tol_scale,
      unsorted_tol);
}

void nbsp_bh_sort(uint64_t* keys, uint32_t* index, uint64_t* keys_alt, uint32_t* index_alt,
                  size_t n, uint32_t* scratch, int* status, cudaStream_t stream) {
  cudaFuncSetAttribute(sort_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)kDownsweepSmem);
  const SortScratch sc = sort_scratch(scratch, n);
  const size_t tiles = sort_tiles(n);
  NBSP_COUNT_LAUNCH(1), sort_bases_kernel<<<1, kRadix, 0, stream>>>(sc.hist, sc.base);
  uint64_t* kin = keys;
  uint32_t* vin = index;
  uint64_t* kout = keys_alt;
  uint32_t* vout = index_alt;
  for (int pass = 0; pass < kSortPasses; ++pass) {
    NBSP_COUNT_LAUNCH(1), sort_pass_kernel<<<(unsigned)tiles, kSortThreads, kDownsweepSmem, stream>>>(
        kin, vin, kout, vout, n, 8 * pass, sc.base + pass * kRadix, sc.ticket + pass,
        sc.status + (size_t)pass * tiles * kRadix, status);
    uint64_t* tk = kin;
    kin = kout;
    kout = tk;
    uint32_t* tv = vin;
    vin = vout;
    vout = tv;
  }
  // kSortPasses = 8 (even): the result is back in (keys, index)
}

void nbsp_bh_duplicates(const uint64_t* keys, const uint32_t* perm, const double* x,
                        const double* y, const double* z, size_t n, int* status,
                        cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), duplicates_kernel<<<grid_for(n, 256), 256, 0, stream>>>(keys, perm, x, y, z, n, status);
}

void nbsp_bh_gather(const void* unsorted, const uint32_t* perm, size_t n, void* pos4,
                    const float* unsorted_tol, float* tol, int* status, cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), gather_kernel<<<grid_for(n, 256), 256, 0, stream>>>(
      (const float4*)unsorted, perm, n, (float4*)pos4, unsorted_tol, tol, status);
}

size_t nbsp_bh_tree_bytes(size_t n) { return tree_bytes(n); }

void nbsp_bh_build(const uint64_t* keys, size_t n, int leaf_capacity, void* tree, int* status,
                   cudaStream_t stream) {
  Tree t = tree_view(tree, n);
  cudaMemsetAsync(t.mask, 0, n * sizeof(uint32_t), stream);
  cudaMemsetAsync(t.leaves, 0, sizeof(unsigned long long), stream);
  if (n >= 2)
    NBSP_COUNT_LAUNCH(1), radix_tree_kernel<<<(unsigned)((n - 1 + 255) / 256), 256, 0, stream>>>(keys, t, status);
  // keep and place: one thread per internal binary node (n >= 2: the caller
  // handles a lone particle without a tree)
  const unsigned internal_blocks = (unsigned)((n - 1 + 255) / 256);
  if (internal_blocks > 0)
    NBSP_COUNT_LAUNCH(1), keep_kernel<<<internal_blocks, 256, 0, stream>>>(t, leaf_capacity, status);
  const int blocks = (int)((n + kScanItems - 1) / kScanItems);
  NBSP_COUNT_LAUNCH(1), scan_reduce_kernel<<<blocks, 256, 0, stream>>>(t);
  NBSP_COUNT_LAUNCH(1), scan_blocks_kernel<<<1, 1024, 0, stream>>>(t, blocks);
  NBSP_COUNT_LAUNCH(1), scan_apply_kernel<<<blocks, 256, 0, stream>>>(t);
  if (internal_blocks > 0)
    NBSP_COUNT_LAUNCH(1), place_kernel<<<internal_blocks, 256, 0, stream>>>(t, leaf_capacity, status);
}

void nbsp_bh_moments(const void* pos4, const uint64_t* keys, size_t n, const double* geometry,
                     double theta, double start_theta, int opening, int quadrupoles, void* tree,
                     int* status, cudaStream_t stream) {
  Tree t = tree_view(tree, n);
  const size_t nb = 2 * n - 1;
  Opening o;
  o.keys = keys;
  o.geometry = geometry;
  o.inv_theta = theta > 0.0 ? 1.0 / theta : INFINITY;
  o.inv_theta2 = theta > 0.0 ? 1.0 / (theta * theta) : INFINITY;
  o.relative = start_theta > 0.0;
  o.start_inv_theta = o.relative ? 1.0 / start_theta : o.inv_theta;
  o.start_inv_theta2 = o.relative ? 1.0 / (start_theta * start_theta) : o.inv_theta2;
  o.criterion = opening;
  size_t blocks = (nb + 255) / 256;  // grid-stride over the octree nodes (<= 2n - 1)
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (quadrupoles)
    NBSP_COUNT_LAUNCH(1), moments_kernel<true><<<(unsigned)blocks, 256, 0, stream>>>(
                              (const float4*)pos4, t, o, status);
  else
    NBSP_COUNT_LAUNCH(1), moments_kernel<false><<<(unsigned)blocks, 256, 0, stream>>>(
                              (const float4*)pos4, t, o, status);
}

void nbsp_bh_walk(const void* pos4, const float* tol, size_t n, const void* tree, int order,
                  int mode, const void* correction, const NbspCorrectionLists* lists, float eps2,
                  const uint32_t* perm, void* acc, unsigned long long* counters, int* status,
                  cudaStream_t stream) {
  Tree t = tree_view(const_cast<void*>(tree), n);
  const nbsp_mlp::Net* net = (const nbsp_mlp::Net*)correction;
  const float4* p = (const float4*)pos4;
  double4* out = (double4*)acc;
  if (tol != nullptr)
    launch_walk<true>(p, tol, n, t, order, mode, net, lists, eps2, perm, out, counters, status,
                      stream);
  else
    launch_walk<false>(p, nullptr, n, t, order, mode, net, lists, eps2, perm, out, counters,
                       status, stream);
}

void nbsp_bh_correct(const void* pos4, size_t n, const void* tree, const void* correction,
                     const NbspCorrectionLists* lists, const uint32_t* perm, void* acc,
                     unsigned long long* counters, int* status, cudaStream_t stream) {
  Tree t = tree_view(const_cast<void*>(tree), n);
  const nbsp_mlp::Net* net = (const nbsp_mlp::Net*)correction;
  const int groups = (int)((n + 31) / 32);
  NBSP_COUNT_LAUNCH(1), corr_scan_kernel<<<1, 1024, 0, stream>>>(*lists, groups, counters);
  NBSP_COUNT_LAUNCH(1), corr_rowmap_kernel<<<(unsigned)((groups + 3) / 4), 128, 0, stream>>>(
      *lists, groups);
  const int smem = (int)sizeof(nbsp_umma::Smem);
  cudaFuncSetAttribute(corr_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  // persistent: kCtasPerSm CTAs per SM, each holding 64 of the 512 TMEM columns
  NBSP_COUNT_LAUNCH(1), corr_rows_kernel<<<148 * nbsp_umma::kCtasPerSm, nbsp_umma::kThreads, smem, stream>>>(
      net, t, *lists, groups, status);
  NBSP_COUNT_LAUNCH(1), corr_apply_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(
      (const float4*)pos4, (int)n, t, *lists, perm, (double4*)acc);
}

void nbsp_bh_unsort(const void* acc, size_t n, double g, double* ax, double* ay, double* az,
                    const NbspLeapfrogFusion* leapfrog, cudaStream_t stream) {
  if (leapfrog != nullptr && leapfrog->vx != nullptr) {
    NBSP_COUNT_LAUNCH(1), unsort_kernel<true><<<grid_for(n, 256), 256, 0, stream>>>(
        (const double4*)acc, n, g, ax, ay, az, leapfrog->vx, leapfrog->vy, leapfrog->vz,
        leapfrog->half_dt);
  } else {
    NBSP_COUNT_LAUNCH(1), unsort_kernel<false><<<grid_for(n, 256), 256, 0, stream>>>(
        (const double4*)acc, n, g, ax, ay, az, nullptr, nullptr, nullptr, 0.0);
  }
}

void nbsp_bh_mlp_pairs(const void* pos4, size_t n, const void* tree, float theta, int opening,
                       unsigned long long seed, int samples, int* target, int* cell, int* status,
                       cudaStream_t stream) {
  Tree t = tree_view(const_cast<void*>(tree), n);
  NBSP_COUNT_LAUNCH(1), mlp_pairs_kernel<<<(samples + 127) / 128, 128, 0, stream>>>(
      (const float4*)pos4, (int)n, t, theta, opening, seed, samples, target, cell, status);
}

void nbsp_bh_mlp_labels(const void* pos4, size_t n, const void* tree, const int* target,
                        const int* cell, int samples, float eps2, float* feat, float* lab, int* ok,
                        cudaStream_t stream) {
  Tree t = tree_view(const_cast<void*>(tree), n);
  const long long threads = (long long)samples * 32;
  NBSP_COUNT_LAUNCH(1), mlp_labels_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(
      (const float4*)pos4, (int)n, t, target, cell, samples, eps2, feat, lab, ok);
}

void nbsp_bh_mlp_stats(const float* feat, const float* lab, const int* ok, int rows, void* net,
                       cudaStream_t stream) {
  NBSP_COUNT_LAUNCH(1), mlp_stats_kernel<<<nbsp_mlp::kIn + nbsp_mlp::kOut, 256, 0, stream>>>(
      feat, lab, ok, rows, (nbsp_mlp::Net*)net);
}

void nbsp_bh_tree_counts(const void* tree, size_t n, unsigned long long* counters,
                         cudaStream_t stream) {
  Tree t = tree_view(const_cast<void*>(tree), n);
  NBSP_COUNT_LAUNCH(1), tree_counts_kernel<<<1, 32, 0, stream>>>(t, counters);
}

}  // extern "C"
