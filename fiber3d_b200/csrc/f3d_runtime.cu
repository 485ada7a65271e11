// Library-level plumbing: version, status strings, the per-device error word.
#include <mutex>

#include "f3d_common.cuh"

namespace f3d {

// One error word per device that loads the library; kernels record the first
// failing status here (atomicCAS from 0), f3d_get_device_error reads+clears.
static __device__ int g_device_error;

int *device_error_word() {
  static std::mutex mu;
  static int *addr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_device_error) != cudaSuccess) return nullptr;
    addr[dev] = static_cast<int *>(p);
  }
  return addr[dev];
}

}  // namespace f3d

extern "C" {

const char *f3d_version(void) { return "fiber3d_b200 0.1.0 (sm_100a)"; }

const char *f3d_status_string(int status) {
  switch (status) {
    case F3D_OK: return "ok";
    case F3D_ERR_NULL: return "a required pointer is NULL";
    case F3D_ERR_SHAPE: return "negative or inconsistent sizes";
    case F3D_ERR_ALIGN: return "a pointer is not suitably aligned";
    case F3D_ERR_WORKSPACE: return "workspace missing or too small";
    case F3D_ERR_ARG: return "invalid argument";
    case F3D_ERR_CUDA: return "CUDA runtime error";
    case F3D_ERR_NONFINITE: return "non-finite input";
    case F3D_ERR_TIMEOUT: return "device-side bounded wait ran out";
    case F3D_ERR_SINGULAR: return "zero pivot in LU factorisation";
    case F3D_ERR_TOO_LARGE: return "size beyond the documented maximum";
    default: return "unknown status";
  }
}

int f3d_get_device_error(void *stream) {
  int *w = f3d::device_error_word();
  if (!w) return F3D_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int h = 0;
  if (cudaMemcpyAsync(&h, w, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return F3D_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return F3D_ERR_CUDA;
  if (h != 0) {
    if (cudaMemsetAsync(w, 0, sizeof(int), s) != cudaSuccess) return F3D_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return F3D_ERR_CUDA;
  }
  return h;
}

}  // extern "C"
