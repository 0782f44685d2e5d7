// Fixed scratch for xs_run_path_device_noalloc: the resident path's
// observable partial sums (one row per CTA and output time) live in a
// file-scope device array instead of memory from cudaMalloc, so that callers
// that must not allocate device memory can still run the path.  Every GPU
// that loads this library holds the array until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "xs_noalloc.hpp"

// 16 MiB: XS_NOALLOC_SCRATCH_DOUBLE2 complex FP64 values.
static __device__ __align__(256) double2 xs_noalloc_scratch[XS_NOALLOC_SCRATCH_DOUBLE2];

namespace {
std::mutex g_mu;
void* g_addr[XS_NOALLOC_MAX_DEVICES] = {};
}  // namespace

// Device address of the scratch array on the current device.  Host code may
// not use the array's name as a device pointer, so the address is looked up
// once per device with that device current and cached.  The cache assumes the
// device's primary context lives as long as the process: after a
// cudaDeviceReset (or a MATLAB gpuDevice reset) the module is loaded again and
// the cached address is stale, so a caller that resets a device must not call
// xs_run_path_device_noalloc on it again in the same process.  Returns the
// CUDA error of the lookup (cudaSuccess when *out is valid).
cudaError_t xs_noalloc_scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= XS_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, xs_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}
