// Library-level plumbing: version, status strings, the per-device error
// word, the bounded-wait limit and a self-test of the bounded wait.
#include <atomic>
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

static std::atomic<uint64_t> g_wait_limit_ns{kWaitLimitNs};

uint64_t wait_limit_ns() { return g_wait_limit_ns.load(std::memory_order_relaxed); }

// One CTA waits on an mbarrier that nothing ever arrives on, for at most
// limit_ns, then records F3D_ERR_TIMEOUT like a kernel whose copy never
// landed.  No copy is issued, so nothing is in flight when the CTA exits.
__global__ void bounded_wait_selftest_kernel(uint64_t limit_ns, int *err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0, limit_ns)) record_error(err, F3D_ERR_TIMEOUT);
}

}  // namespace f3d

extern "C" {

int f3d_set_wait_limit_ns(uint64_t limit_ns) {
  f3d::g_wait_limit_ns.store(limit_ns ? limit_ns : f3d::kWaitLimitNs, std::memory_order_relaxed);
  return F3D_OK;
}

uint64_t f3d_wait_limit_ns(void) { return f3d::wait_limit_ns(); }

int f3d_selftest_bounded_wait(uint64_t limit_ns, void *stream) {
  if (limit_ns == 0 || limit_ns > f3d::kWaitLimitNs) return F3D_ERR_ARG;
  int *err = f3d::device_error_word();
  if (!err) return F3D_ERR_CUDA;
  f3d::bounded_wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limit_ns, err);
  return f3d::launch_status();
}

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

int f3d_peek_device_error_async(int *host_dst, void *stream) {
  if (!host_dst) return F3D_ERR_NULL;
  int *w = f3d::device_error_word();
  if (!w) return F3D_ERR_CUDA;
  if (cudaMemcpyAsync(host_dst, w, sizeof(int), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)) !=
      cudaSuccess)
    return F3D_ERR_CUDA;
  return F3D_OK;
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
