// All-pairs accelerations for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code that runs while a CUDA graph
// is being captured (an allocation there breaks the capture), plugins living
// inside a host framework that owns every device allocation through its own
// pool, and real-time loops that must not touch the allocator after start-up.
// They own their input and output buffers already; what they cannot provide
// is the all-pairs path's working memory.  This entry point therefore keeps
// that working memory in one file-scope __device__ array of fixed size, which
// the CUDA module reserves on every GPU that loads this library, for as long as
// the process lives.
//
// Limits and sharing rules (also in include/n_body_sim_pro_cuda.h):
//   * at most kNoAllocMaxParticles (16384) particles; larger counts are
//     rejected with INVALID_ARGUMENT before any GPU work;
//   * the array (about 4.3 MiB) is shared by every call in the process on that
//     device and keeps the last call's contents; each call rewrites all of it
//     that it reads, and clears the one word that must start at zero;
//   * two calls whose GPU work overlaps (different streams, no ordering
//     between them) race on the array and produce wrong results;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress; make that first call before any stream capture.
#include "internal.h"
#include "n_body_sim_pro_cuda.h"

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

namespace {

constexpr size_t kNoAllocMaxParticles = 16384;  // multiple of 256: no padding beyond it
constexpr int kNoAllocMaxChunks = 8;
constexpr int kNoAllocBlock = 128;
constexpr int kNoAllocPerThread = 4;

// Byte offsets of the sub-buffers inside the static array.
constexpr size_t kOffCentre = 0;        // 3 doubles
constexpr size_t kOffStatus = 256;      // 1 int
constexpr size_t kOffSums = 512;        // centre-of-mass partials: 11 doubles x <= 64 blocks
constexpr size_t kOffPacked = 8192;     // float4[kNoAllocMaxParticles]
constexpr size_t kOffHi = kOffPacked + kNoAllocMaxParticles * 16;
constexpr size_t kOffLo = kOffHi + (size_t)kNoAllocMaxChunks * kNoAllocMaxParticles * 16;
constexpr size_t kScratchBytes = kOffLo + (size_t)kNoAllocMaxChunks * kNoAllocMaxParticles * 16;
static_assert(kOffSums + 11 * 64 * sizeof(double) <= kOffPacked, "partials overlap");

}  // namespace

// The working memory: about 4.3 MiB on every device that loads the library.
// Host code must not pass this name to a kernel (on the host it is only a
// stand-in); the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
// Host-side cache of the array's device address, one slot per device.
unsigned char* g_scratch_address[kMaxDevices];

NBodySimProStatus report(NBodySimProError* error, NBodySimProStatus status, int line,
                         const char* message) {
  if (error != nullptr) {
    error->status = status;
    error->source_file = __FILE__;
    error->source_line = line;
    snprintf(error->message, sizeof(error->message), "%s", message);
  }
  return status;
}

NBodySimProStatus report_cuda(NBodySimProError* error, cudaError_t code, int line,
                              const char* what) {
  char text[256];
  snprintf(text, sizeof(text), "%s: %s", what, cudaGetErrorString(code));
  const NBodySimProStatus status =
      (code == cudaErrorNoDevice || code == cudaErrorInsufficientDriver ||
       code == cudaErrorNoKernelImageForDevice)
          ? N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM
          : N_BODY_SIM_PRO_STATUS_INVALID_STATE;
  return report(error, status, line, text);
}

// True when `p` may be dereferenced by a kernel on `device` (the current one):
// managed memory, or device memory that lives on that same device (a buffer of
// another GPU would be a peer access, or a fault without peer access).
bool device_accessible(const void* p, int device) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (attr.type == cudaMemoryTypeManaged) return true;
  return attr.type == cudaMemoryTypeDevice && attr.device == device;
}

}  // namespace

extern "C" N_BODY_SIM_PRO_CUDA_API NBodySimProStatus
n_body_sim_pro_cuda_allpairs_acceleration_noalloc(
    const double* positions_x, const double* positions_y, const double* positions_z,
    const double* masses, double* accelerations_x, double* accelerations_y,
    double* accelerations_z, size_t particle_count, double gravitational_constant,
    double softening_length, void* stream, NBodySimProError* error) {
  if (particle_count > kNoAllocMaxParticles) {
    return report(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                  "particle_count exceeds the 16384-particle limit of the static scratch "
                  "array (use n_body_sim_pro_gravity_compute_acceleration_cuda)");
  }
  const double eps2 = softening_length * softening_length;
  if (!(eps2 >= 0.0) || eps2 == INFINITY || gravitational_constant != gravitational_constant) {
    return report(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                  "gravity parameters must be finite");
  }
  if (particle_count == 0) return N_BODY_SIM_PRO_STATUS_OK;
  const void* arrays[] = {positions_x, positions_y, positions_z, masses,
                          accelerations_x, accelerations_y, accelerations_z};
  int device = 0;
  cudaError_t code = cudaGetDevice(&device);
  if (code != cudaSuccess) return report_cuda(error, code, __LINE__, "cudaGetDevice");
  if (device < 0 || device >= kMaxDevices) {
    return report(error, N_BODY_SIM_PRO_STATUS_UNSUPPORTED_PLATFORM, __LINE__,
                  "device ordinal beyond the scratch address table");
  }
  for (const void* a : arrays) {
    if (a == nullptr || !device_accessible(a, device)) {
      return report(error, N_BODY_SIM_PRO_STATUS_INVALID_ARGUMENT, __LINE__,
                    "all seven arrays must be non-null pointers to the current device's memory");
    }
  }

  // One-time set-up on this device: the array's address as the device sees it.
  unsigned char* base = __atomic_load_n(&g_scratch_address[device], __ATOMIC_ACQUIRE);
  if (base == nullptr) {
    void* address = nullptr;
    code = cudaGetSymbolAddress(&address, g_noalloc_scratch);
    if (code != cudaSuccess || address == nullptr) {
      return report_cuda(error, code != cudaSuccess ? code : cudaErrorInvalidSymbol, __LINE__,
                         "cudaGetSymbolAddress of the static scratch array");
    }
    base = static_cast<unsigned char*>(address);
    __atomic_store_n(&g_scratch_address[device], base, __ATOMIC_RELEASE);
  }

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n = particle_count;
  const size_t n_padded = (n + 255) / 256 * 256;
  double* centre = reinterpret_cast<double*>(base + kOffCentre);
  int* status = reinterpret_cast<int*>(base + kOffStatus);
  double* sums = reinterpret_cast<double*>(base + kOffSums);
  void* packed = base + kOffPacked;
  void* hi = base + kOffHi;
  void* lo = base + kOffLo;

  NbspAllPairsShape shape;
  shape.block = kNoAllocBlock;
  shape.per_thread = kNoAllocPerThread;
  shape.paired = 0;
  shape.min_blocks = 0;
  const size_t target_blocks = (n + kNoAllocBlock * kNoAllocPerThread - 1) /
                               (kNoAllocBlock * kNoAllocPerThread);
  size_t chunks = (148 * 8 + target_blocks - 1) / target_blocks;
  if (chunks > (size_t)kNoAllocMaxChunks) chunks = kNoAllocMaxChunks;
  if (chunks < 1) chunks = 1;
  shape.chunks = (int)chunks;

  code = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (code != cudaSuccess) return report_cuda(error, code, __LINE__, "status clear");
  nbsp_centre_of_mass(positions_x, positions_y, positions_z, masses, n, sums, centre, s);
  nbsp_pack_relative(positions_x, positions_y, positions_z, masses, n, n_padded, centre, packed,
                     status, s);
  nbsp_allpairs_force(packed, n, n_padded, (float)eps2, shape, hi, lo, s);
  nbsp_allpairs_finalize(hi, lo, n, shape.chunks, gravitational_constant, accelerations_x,
                         accelerations_y, accelerations_z, s);
  code = cudaGetLastError();
  if (code != cudaSuccess) return report_cuda(error, code, __LINE__, "kernel launch");
  return N_BODY_SIM_PRO_STATUS_OK;
}
