// The all-pairs sum without a caller workspace.
//
// f3d_pair_sum needs scratch memory when it splits the sources over several
// CTAs (per-split partial sums and their counters) and, in FP32C, for the
// packed float sources.  Normally the caller allocates that workspace.  Some
// callers cannot: code that runs where device allocation is forbidden or
// unavailable (a host that hands over only pre-registered buffers, a
// real-time loop that must not call cudaMalloc and so risk an implicit device
// synchronisation or an out-of-memory failure mid-run, or a plugin whose host
// owns all memory).  f3d_pair_sum_noalloc serves them: its scratch is the
// file-scope device array below, which every GPU that loads the library holds
// for the life of the process.
//
// Host code must not use the array's name as a device address: on the host it
// names a shadow object.  The device address is fetched once per device with
// cudaGetSymbolAddress (with that device current) and passed to the kernels.
#include <mutex>

#include "f3d_common.cuh"

namespace f3d {

int pair_sum_impl(int kernel, int precision, int self_mode, const double *rs, const double *rt,
                  const double *dens, const double *nrm, const int32_t *gs, const int32_t *gt,
                  double *out, int64_t ns, int64_t nt, double eta, double reg, double eps,
                  int accumulate, const f3d_pair_shape *shape, void *ws, size_t ws_bytes,
                  cudaStream_t st);

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of this device's scratch array, looked up on first use.
static int noalloc_scratch(void **addr) {
  static std::mutex mu;
  static void *cached[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return F3D_ERR_CUDA;
  std::lock_guard<std::mutex> lock(mu);
  if (!cached[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return F3D_ERR_CUDA;
    cached[dev] = p;
  }
  *addr = cached[dev];
  return F3D_OK;
}

}  // namespace f3d

extern "C" {

int f3d_pair_sum_noalloc(int kernel, int precision, int self_mode, const double *r_source,
                         const double *r_target, const double *density, const double *normal,
                         const int32_t *src_group, const int32_t *trg_group, double *out,
                         int64_t ns, int64_t nt, double eta, double reg, double epsilon_distance,
                         int accumulate, void *stream) {
  size_t need = 0;
  int rc = f3d_pair_workspace_bytes(kernel, precision, ns, nt, nullptr, &need);
  if (rc) return rc;
  if (need > f3d::kNoAllocScratchBytes) return F3D_ERR_TOO_LARGE;
  void *scratch = nullptr;
  if (need > 0) {
    if ((rc = f3d::noalloc_scratch(&scratch))) return rc;
    // The array keeps whatever the previous call left; the split counters
    // must start at zero, so clear them on this call's stream.
    const size_t clear = need < f3d::kCounterBytes ? need : f3d::kCounterBytes;
    if (cudaMemsetAsync(scratch, 0, clear, static_cast<cudaStream_t>(stream)) != cudaSuccess)
      return F3D_ERR_CUDA;
  }
  return f3d::pair_sum_impl(kernel, precision, self_mode, r_source, r_target, density, normal,
                            src_group, trg_group, out, ns, nt, eta, reg, epsilon_distance,
                            accumulate, nullptr, scratch, scratch ? f3d::kNoAllocScratchBytes : 0,
                            static_cast<cudaStream_t>(stream));
}

}  // extern "C"
