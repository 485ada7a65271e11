// The all-pairs sums for host callers: one entry point that brings the
// inputs from host memory into a caller-provided device buffer, runs the sum,
// brings the result back and waits, so that a host-side binding (fiber3d's
// kernels.kernels functions take and return numpy arrays) makes one call per
// sum instead of a sequence of allocations, copies and launches.  The kernel
// is the one f3d_pair_sum runs; only the staging differs.
//
// Page-locked host memory that the device can address (cudaHostAlloc'd or
// registered memory under unified addressing) is read and written by
// kernels directly: one staging kernel reads every such input over the host
// link (one launch instead of a copy per array), and the pair kernel writes
// its result straight into such an `out` (each element is written exactly
// once, so nothing is read back over the link).  Other host memory goes
// through cudaMemcpyAsync.
#include <algorithm>

#include "f3d_common.cuh"

namespace f3d {

int pair_sum_impl(int kernel, int precision, int self_mode, const double *rs, const double *rt,
                  const double *dens, const double *nrm, const int32_t *gs, const int32_t *gt,
                  double *out, int64_t ns, int64_t nt, double eta, double reg, double eps,
                  int accumulate, const f3d_pair_shape *shape, void *ws, size_t ws_bytes,
                  cudaStream_t st);

struct HostLayout {
  size_t rs, rt, dens, nrm, out, bytes;
};

// Device staging of one host sum: [r_source][r_target unless the same
// points][density][normal if any][out], each 256-byte aligned.  With the
// same points (one array holding the sources as its first ns points) the
// points region holds max(ns, nt) points.
static HostLayout host_layout(int kernel, int64_t ns, int64_t nt, bool same) {
  HostLayout L{};
  size_t o = 0;
  auto take = [&](size_t n) {
    const size_t at = o;
    o += round_up(n * sizeof(double), 256);
    return at;
  };
  L.rs = take(3 * static_cast<size_t>(same ? std::max(ns, nt) : ns));
  L.rt = same ? L.rs : take(3 * static_cast<size_t>(nt));
  L.dens = take(3 * static_cast<size_t>(ns));
  L.nrm = (kernel == F3D_KERNEL_STRESSLET) ? take(3 * static_cast<size_t>(ns))
          : (kernel == F3D_KERNEL_TRACTION) ? take(3 * static_cast<size_t>(nt))
                                             : 0;
  L.out = take(3 * static_cast<size_t>(nt));
  L.bytes = o;
  return L;
}

// Device address of page-locked host memory the current device can access
// directly, or null (pageable memory, device memory, or an error, which is
// cleared).
static void *mapped_host(const void *p) {
  if (!p) return nullptr;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

// Up to four host-to-device copies in one launch: blockIdx.y picks the
// array, each CTA moves 16 KB of it (16-byte loads when both ends are
// 16-byte aligned, else 8-byte ones; sizes are whole doubles).  All loads of
// a thread are issued before its stores, so a CTA keeps 16 KB of reads in
// flight over the host link.
struct StageSeg {
  const char *src;
  char *dst;
  int64_t bytes;
};
struct StageArgs {
  StageSeg seg[4];
};
constexpr int kStageThreads = 256;
constexpr int kStageBytesPerCta = 16384;

__global__ void __launch_bounds__(kStageThreads) stage_in_kernel(const StageArgs a) {
  const StageSeg s = a.seg[blockIdx.y];
  const int64_t first = static_cast<int64_t>(blockIdx.x) * kStageBytesPerCta;
  if (first >= s.bytes) return;
  if (((reinterpret_cast<uintptr_t>(s.src) | reinterpret_cast<uintptr_t>(s.dst)) & 15) == 0) {
    constexpr int kU = kStageBytesPerCta / (16 * kStageThreads);
    const int64_t n = s.bytes / 16;
    const uint4 *src = reinterpret_cast<const uint4 *>(s.src);
    uint4 *dst = reinterpret_cast<uint4 *>(s.dst);
    const int64_t base = first / 16 + threadIdx.x;
    uint4 r[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (base + u * kStageThreads < n) r[u] = src[base + u * kStageThreads];
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (base + u * kStageThreads < n) dst[base + u * kStageThreads] = r[u];
    // an odd last double
    if ((s.bytes & 15) && blockIdx.x == 0 && threadIdx.x == 0) {
      const int64_t last = s.bytes / 8 - 1;
      reinterpret_cast<double *>(s.dst)[last] = reinterpret_cast<const double *>(s.src)[last];
    }
  } else {
    constexpr int kU = kStageBytesPerCta / (8 * kStageThreads);
    const int64_t n = s.bytes / 8;
    const double *src = reinterpret_cast<const double *>(s.src);
    double *dst = reinterpret_cast<double *>(s.dst);
    const int64_t base = first / 8 + threadIdx.x;
    double r[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (base + u * kStageThreads < n) r[u] = src[base + u * kStageThreads];
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (base + u * kStageThreads < n) dst[base + u * kStageThreads] = r[u];
  }
}

// A page-locked word per host thread and device that the device error word
// is copied into asynchronously (read after the call's one wait).
static int *pinned_error_slot() {
  constexpr int kMaxDevices = 64;
  thread_local int *slot[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  if (!slot[dev] && cudaHostAlloc(reinterpret_cast<void **>(&slot[dev]), 64, cudaHostAllocDefault) != cudaSuccess) {
    (void)cudaGetLastError();
    slot[dev] = nullptr;
  }
  return slot[dev];
}

}  // namespace f3d

extern "C" {

int f3d_pair_host_bytes(int kernel, int64_t ns, int64_t nt, int same_points, size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  if (kernel < 0 || kernel > 3) return F3D_ERR_ARG;
  if (ns < 0 || nt < 0) return F3D_ERR_SHAPE;
  *bytes = f3d::host_layout(kernel, ns, nt, same_points != 0).bytes;
  return F3D_OK;
}

int f3d_pair_sum_host(int kernel, int precision, int self_mode, const double *r_source,
                      const double *r_target, const double *density, const double *normal, double *out,
                      int64_t ns, int64_t nt, double eta, double reg, double epsilon_distance,
                      const f3d_pair_shape *shape, void *device_buffer, size_t device_bytes,
                      void *workspace, size_t workspace_bytes, void *stream) {
  if (kernel < 0 || kernel > 3) return F3D_ERR_ARG;
  if (self_mode == F3D_SELF_SKIP_GROUP) return F3D_ERR_ARG;  // no group ids on this path
  if (ns < 0 || nt < 0) return F3D_ERR_SHAPE;
  if (nt == 0) return F3D_OK;
  if (!r_target || !out || (ns > 0 && (!r_source || !density))) return F3D_ERR_NULL;
  const bool has_nrm = kernel == F3D_KERNEL_STRESSLET || kernel == F3D_KERNEL_TRACTION;
  if (has_nrm && !normal) return F3D_ERR_NULL;
  const bool same = (r_source == r_target);
  const f3d::HostLayout L = f3d::host_layout(kernel, ns, nt, same);
  if (!device_buffer || device_bytes < L.bytes) return F3D_ERR_WORKSPACE;
  if (!f3d::aligned(device_buffer, 256)) return F3D_ERR_ALIGN;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char *b = static_cast<char *>(device_buffer);
  double *d_rs = reinterpret_cast<double *>(b + L.rs), *d_rt = reinterpret_cast<double *>(b + L.rt);
  double *d_dens = reinterpret_cast<double *>(b + L.dens), *d_out = reinterpret_cast<double *>(b + L.out);
  double *d_nrm = has_nrm ? reinterpret_cast<double *>(b + L.nrm) : nullptr;
  const size_t sb = 3 * sizeof(double) * static_cast<size_t>(ns), tb = 3 * sizeof(double) * static_cast<size_t>(nt);
  // inputs: one staging launch when every host array is device-addressable,
  // else one copy per array
  const size_t nb_rs = same ? std::max(sb, tb) : sb, nb_nrm = kernel == F3D_KERNEL_TRACTION ? tb : sb;
  const void *srcs[4] = {r_source, same ? nullptr : r_target, density, has_nrm ? normal : nullptr};
  void *dsts[4] = {d_rs, d_rt, d_dens, d_nrm};
  const size_t sizes[4] = {nb_rs, same ? 0 : tb, sb, has_nrm ? nb_nrm : 0};
  f3d::StageArgs sa{};
  bool zero_copy = true;
  int nseg = 0;
  int64_t most = 0;
  for (int i = 0; i < 4 && zero_copy; ++i) {
    if (sizes[i] == 0) continue;
    void *m = f3d::mapped_host(srcs[i]);
    if (!m || !f3d::aligned(m, 8)) zero_copy = false;
    sa.seg[nseg++] = {static_cast<const char *>(m), static_cast<char *>(dsts[i]), static_cast<int64_t>(sizes[i])};
    most = std::max(most, static_cast<int64_t>(sizes[i]));
  }
  if (zero_copy && nseg > 0) {
    const dim3 grid(static_cast<unsigned>((most + f3d::kStageBytesPerCta - 1) / f3d::kStageBytesPerCta), nseg);
    f3d::stage_in_kernel<<<grid, f3d::kStageThreads, 0, st>>>(sa);
    if (f3d::launch_status() != F3D_OK) return F3D_ERR_CUDA;
  } else {
    for (int i = 0; i < 4; ++i)
      if (sizes[i] > 0 && cudaMemcpyAsync(dsts[i], srcs[i], sizes[i], cudaMemcpyHostToDevice, st) != cudaSuccess)
        return F3D_ERR_CUDA;
  }
  // output: written by the kernel into a device-addressable `out` directly
  double *direct = ns > 0 ? static_cast<double *>(f3d::mapped_host(out)) : nullptr;
  if (direct && !f3d::aligned(direct, 8)) direct = nullptr;
  int rc = f3d::pair_sum_impl(kernel, precision, self_mode, d_rs, d_rt, d_dens, d_nrm, nullptr, nullptr,
                              direct ? direct : d_out, ns, nt, eta, reg, epsilon_distance, 0, shape, workspace,
                              workspace_bytes, st);
  if (rc) return rc;
  if (!direct && cudaMemcpyAsync(out, d_out, tb, cudaMemcpyDeviceToHost, st) != cudaSuccess) return F3D_ERR_CUDA;
  // the kernels' error word, read after the same wait
  int *w = f3d::device_error_word();
  int *slot = f3d::pinned_error_slot();
  int local = 0;
  int *dst = slot ? slot : &local;
  if (!w || cudaMemcpyAsync(dst, w, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return F3D_ERR_CUDA;
  const int err = *dst;
  if (err != 0) {
    if (cudaMemsetAsync(w, 0, sizeof(int), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return F3D_ERR_CUDA;
    return err;
  }
  return F3D_OK;
}

}  // extern "C"
