// The all-pairs sums for host callers: one entry point that copies the
// inputs from host memory into a caller-provided device buffer, runs the sum,
// copies the result back and waits, so that a host-side binding (fiber3d's
// kernels.kernels functions take and return numpy arrays) makes one call per
// sum instead of a sequence of allocations, copies and launches.  The kernel
// is the one f3d_pair_sum runs; only the staging differs.
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
  auto h2d = [&](void *dst, const void *src, size_t n) {
    return n == 0 || cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) == cudaSuccess;
  };
  if (!h2d(d_rs, r_source, same ? std::max(sb, tb) : sb) || (!same && !h2d(d_rt, r_target, tb)) ||
      !h2d(d_dens, density, sb) ||
      (has_nrm && !h2d(d_nrm, normal, kernel == F3D_KERNEL_TRACTION ? tb : sb)))
    return F3D_ERR_CUDA;
  int rc = f3d::pair_sum_impl(kernel, precision, self_mode, d_rs, d_rt, d_dens, d_nrm, nullptr, nullptr, d_out, ns,
                              nt, eta, reg, epsilon_distance, 0, shape, workspace, workspace_bytes, st);
  if (rc) return rc;
  if (cudaMemcpyAsync(out, d_out, tb, cudaMemcpyDeviceToHost, st) != cudaSuccess) return F3D_ERR_CUDA;
  // the kernels' error word, read after the same wait
  int *w = f3d::device_error_word();
  int err = 0;
  if (!w || cudaMemcpyAsync(&err, w, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return F3D_ERR_CUDA;
  if (err != 0) {
    if (cudaMemsetAsync(w, 0, sizeof(int), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return F3D_ERR_CUDA;
    return err;
  }
  return F3D_OK;
}

}  // extern "C"
