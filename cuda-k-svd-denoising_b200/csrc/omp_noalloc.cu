// ksvd_omp_noalloc: the OMP sparse-coding step for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code running inside a CUDA
// graph that is being captured or replayed (allocation is not a capturable
// operation), plugins hosted by a framework that owns every device allocation
// through its own pool and forbids others, and real-time loops that must not
// risk an allocation stall or failure once running.  ksvd_omp() needs a
// context, whose creation and first use allocate, and it keeps the dictionary
// Gram matrix in context memory.  This entry point instead keeps the Gram in
// a fixed array compiled into the library, so it allocates nothing: the
// caller passes the patches, the dictionary and the output code buffers.
//
// Limits and sharing:
//   * at most kNoAllocMaxAtoms atoms (the array holds a 512 x 512 FP64 Gram,
//     2 MiB, present on every GPU that loads this library until the process
//     exits); larger dictionaries are rejected with KSVD_ERR_TOO_LARGE;
//   * every call on a device uses the same array; the Gram kernel writes all
//     K x K entries it uses before the OMP kernel reads them, so nothing has
//     to start at zero, but two calls whose work overlaps on the GPU (for
//     example on two streams) overwrite each other's Gram and give wrong
//     codes: serialise them;
//   * the OMP kernel is the one ksvd_omp's FP32 form would run: the
//     dictionary resident in shared memory when it fits, else streamed through
//     it (so every patch size that ksvd_omp accepts works up to 512 atoms);
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before starting any stream capture.  The cached address
//     belongs to the device's primary context: after cudaDeviceReset() it is
//     stale and this entry point must not be called again in that process.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>

#include "ksvd_internal.cuh"

namespace {

constexpr int kNoAllocMaxAtoms = 512;
constexpr int kNoAllocMaxDevices = 64;

// The Gram scratch.  In host code this name is only a stand-in for the
// symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_gram[kNoAllocMaxAtoms * kNoAllocMaxAtoms];

std::atomic<double*> g_gram_ptr[kNoAllocMaxDevices];
std::mutex g_setup_mutex;

// Device address of the scratch on `device` (the current device), looked up
// once per device.
ksvd_status gram_scratch(int device, double** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return KSVD_ERR_INVALID;
  double* p = g_gram_ptr[device].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_gram_ptr[device].load(std::memory_order_relaxed);
    if (!p) {
      void* addr = nullptr;
      if (cudaGetSymbolAddress(&addr, g_noalloc_gram) != cudaSuccess || addr == nullptr) {
        cudaGetLastError();
        return KSVD_ERR_CUDA;
      }
      p = static_cast<double*>(addr);
      g_gram_ptr[device].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return KSVD_OK;
}

}  // namespace

extern "C" ksvd_status ksvd_omp_noalloc(const ksvd_params* p, const float* d_patches, int64_t num_patches,
                                        const float* d_dict, int32_t* d_idx, float* d_coef, void* stream) {
  if (!p || !d_patches || !d_dict || !d_idx || !d_coef || num_patches < 1) return KSVD_ERR_INVALID;
  if (p->patch_width_dim < 1 || p->patch_height_dim < 1) return KSVD_ERR_INVALID;
  const int64_t n64 = int64_t(p->patch_width_dim) * p->patch_height_dim;  // bounded before it becomes an int
  if (n64 > (int64_t(1) << 20)) return KSVD_ERR_INVALID;
  const int n = int(n64), K = p->atoms, L = p->omp_iter;
  if (K < 1 || L < 1 || L > 32) return KSVD_ERR_INVALID;
  if (K > kNoAllocMaxAtoms) return KSVD_ERR_TOO_LARGE;
  const bool resident = ksvd::omp_fp32_supported(n, K, L);
  if (!resident && !ksvd::omp_stream_supported(n, K, L)) return KSVD_ERR_INVALID;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return KSVD_ERR_NO_DEVICE;
  }
  double* gram = nullptr;
  ksvd_status st = gram_scratch(device, &gram);
  if (st != KSVD_OK) return st;
  int num_sms = 0;
  if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    cudaGetLastError();
    return KSVD_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = ksvd::launch_gram_f64(d_dict, K, n, gram, s);
  if (e == cudaSuccess)
    e = resident ? ksvd::launch_omp_fp32(d_patches, num_patches, n, d_dict, gram, K, L, d_idx, d_coef, num_sms,
                                         nullptr, s)
                 : ksvd::launch_omp_stream(d_patches, num_patches, n, d_dict, gram, K, L, d_idx, d_coef, num_sms,
                                           nullptr, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return KSVD_ERR_CUDA;
  }
  return KSVD_OK;
}
