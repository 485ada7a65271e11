// Velocity field at grid points (fiber3d's compute_velocity, tstep/tstep.py
// :1273-1381, and its post-processing :1414-1448).  The sums themselves --
// periphery and body double layers, the fibers' Oseen flow -- are the pair
// kernels' source -> target sums; this file holds the three pieces around
// them:
//   * each fiber's self-flow at its own nodes with upsampled quadrature
//     (P_kerUp, weights_0_up: tstep/fiber_matrices.py:84-92; the dense
//     oseen_tensor_source_target of kernels.py:119-200 applied to it);
//   * the replacement, at grid points within `near` of a fiber node, of the
//     fibers' flow by that self-flow at the nearest node of the last such
//     fiber (tstep.py:1341-1365);
//   * rigid motion U + W x (g - c) at grid points inside a body
//     (tstep.py:1438-1448).
#include "f3d_common.cuh"

namespace f3d {

// One CTA per fiber.  up_mats + up_off[f]: P_up (M x n, row-major) then the
// unit-length trapezoid weights w_up (M) of the M = uprate * n equispaced
// upsampling nodes; the weights are scaled by L/2 here.
__global__ void fiber_self_flow_up_kernel(const int32_t *__restrict__ npts, const int64_t *__restrict__ pt_off,
                                          const double *__restrict__ length, const double *__restrict__ x,
                                          const double *__restrict__ f, const double *__restrict__ up_mats,
                                          const int64_t *__restrict__ up_off, int uprate, double eta,
                                          double reg, double eps, double *__restrict__ vself) {
  const int k = blockIdx.x;
  const int n = npts[k];
  const int M = uprate * n;
  const int64_t p0 = pt_off[k];
  const double *P = up_mats + up_off[k];
  const double *w = P + static_cast<int64_t>(M) * n;
  const double half_l = 0.5 * length[k];
  extern __shared__ double sm[];
  double *xs = sm;             // n x 3
  double *fs = xs + 3 * n;     // n x 3
  double *xu = fs + 3 * n;     // M x 3
  double *fu = xu + 3 * M;     // M x 3
  for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
    xs[i] = x[3 * p0 + i];
    fs[i] = f[3 * p0 + i];
  }
  __syncthreads();
  for (int u = threadIdx.x; u < M; u += blockDim.x) {
    double a[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i) {
      const double pui = P[static_cast<int64_t>(u) * n + i];
      for (int c = 0; c < 3; ++c) {
        a[c] = fma(pui, xs[3 * i + c], a[c]);
        b[c] = fma(pui, fs[3 * i + c], b[c]);
      }
    }
    const double wu = w[u] * half_l;
    for (int c = 0; c < 3; ++c) {
      xu[3 * u + c] = a[c];
      fu[3 * u + c] = b[c] * wu;
    }
  }
  __syncthreads();
  const double c8 = 1.0 / (8.0 * kPi * eta);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double tx = xs[3 * i], ty = xs[3 * i + 1], tz = xs[3 * i + 2];
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int u = 0; u < M; ++u) {
      const double dx = xu[3 * u] - tx, dy = xu[3 * u + 1] - ty, dz = xu[3 * u + 2] - tz;
      const double dr = sqrt(dx * dx + dy * dy + dz * dz);
      // r > epsilon_distance: 1/r, 1/r^3; else r -> sqrt(r^2 + reg^2)
      const double re = (dr > eps) ? dr : sqrt(dr * dr + reg * reg);
      const double fr = 1.0 / re, gr = 1.0 / (re * re * re);
      const double f0 = fu[3 * u], f1 = fu[3 * u + 1], f2 = fu[3 * u + 2];
      const double df = dx * f0 + dy * f1 + dz * f2;
      v0 += fr * f0 + gr * df * dx;
      v1 += fr * f1 + gr * df * dy;
      v2 += fr * f2 + gr * df * dz;
    }
    vself[3 * (p0 + i)] = c8 * v0;
    vself[3 * (p0 + i) + 1] = c8 * v1;
    vself[3 * (p0 + i) + 2] = c8 * v2;
  }
}

// One thread per grid point.  Distances as fiber3d forms them:
// sqrt(((g_x - x)^2 + (g_y - y)^2) + (g_z - z)^2), rounded operation by
// operation (no contraction), so the <= near test and the first-minimum
// node are the reference's.  A fiber is skipped without looking at its
// nodes when |g - x_0| - R > near (1 + 2^-40), R = max_i |x_i - x_0| (the
// CTA forms every fiber's x_0 and R first): every node is then farther than
// near, so the fiber can be neither the hit nor the nearest-node source.
constexpr int kNearMaxFibers = 2048;

__global__ void grid_near_fiber_kernel(const double *__restrict__ grid, int64_t ngrid,
                                       const double *__restrict__ x, const int64_t *__restrict__ pt_off,
                                       int nfib, const double *__restrict__ vself, double near,
                                       double *__restrict__ vfib) {
  __shared__ double s_rad[kNearMaxFibers];
  const bool bounded = nfib <= kNearMaxFibers;
  if (bounded) {
    for (int k = threadIdx.x; k < nfib; k += blockDim.x) {
      const int64_t p0 = pt_off[k], p1 = pt_off[k + 1];
      double r2 = 0.0;
      for (int64_t p = p0 + 1; p < p1; ++p) {
        const double dx = x[3 * p] - x[3 * p0], dy = x[3 * p + 1] - x[3 * p0 + 1], dz = x[3 * p + 2] - x[3 * p0 + 2];
        r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
      }
      s_rad[k] = sqrt(r2);
    }
    __syncthreads();
  }
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= ngrid) return;
  const double gx = grid[3 * g], gy = grid[3 * g + 1], gz = grid[3 * g + 2];
  const double reach = near * (1.0 + 0x1p-40) + 0x1p-40;
  int64_t best = -1;
  for (int k = 0; k < nfib; ++k) {
    const int64_t p0 = pt_off[k], p1 = pt_off[k + 1];
    if (bounded) {
      const double ax = gx - x[3 * p0], ay = gy - x[3 * p0 + 1], az = gz - x[3 * p0 + 2];
      const double d0 = sqrt(ax * ax + ay * ay + az * az);
      if (d0 - s_rad[k] * (1.0 + 0x1p-40) > reach) continue;
    }
    double dmin = 0.0;
    int64_t imin = p0;
    bool hit = false;
    for (int64_t p = p0; p < p1; ++p) {
      const double dx = __dsub_rn(gx, x[3 * p]), dy = __dsub_rn(gy, x[3 * p + 1]),
                   dz = __dsub_rn(gz, x[3 * p + 2]);
      const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
      hit |= (d <= near);
      if (p == p0 || d < dmin) { dmin = d; imin = p; }
    }
    if (hit) best = imin;
  }
  if (best >= 0) {
    vfib[3 * g] = vself[3 * best];
    vfib[3 * g + 1] = vself[3 * best + 1];
    vfib[3 * g + 2] = vself[3 * best + 2];
  }
}

// One thread per grid point: inside the sphere of radius `radius` about c
// (the test of tstep.py:1439), v = U + W x (g - c), uw = (U, W).
__global__ void grid_rigid_override_kernel(const double *__restrict__ grid, int64_t ngrid,
                                           const double *__restrict__ c, const double *__restrict__ uw,
                                           double radius, double *__restrict__ v) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= ngrid) return;
  const double gx = grid[3 * g], gy = grid[3 * g + 1], gz = grid[3 * g + 2];
  const double a = __dsub_rn(gx, c[0]), b = __dsub_rn(c[1], gy), e = __dsub_rn(c[2], gz);
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(e, e));
  if (!(d2 <= __dmul_rn(radius, radius))) return;
  const double r0 = __dsub_rn(gx, c[0]), r1 = __dsub_rn(gy, c[1]), r2 = __dsub_rn(gz, c[2]);
  v[3 * g] = __dadd_rn(uw[0], __dsub_rn(__dmul_rn(uw[4], r2), __dmul_rn(uw[5], r1)));
  v[3 * g + 1] = __dadd_rn(uw[1], __dsub_rn(__dmul_rn(uw[5], r0), __dmul_rn(uw[3], r2)));
  v[3 * g + 2] = __dadd_rn(uw[2], __dsub_rn(__dmul_rn(uw[3], r1), __dmul_rn(uw[4], r0)));
}

}  // namespace f3d

extern "C" {

int f3d_fiber_self_flow_up(const int32_t *npts, const int64_t *pt_off, const double *length, int32_t nfib,
                           int32_t max_n, const double *x, const double *f, const double *up_mats,
                           const int64_t *up_off, int32_t uprate, double eta, double reg,
                           double epsilon_distance, double *vself, void *stream) {
  if (nfib < 0 || max_n < 0 || uprate < 1) return F3D_ERR_SHAPE;
  if (nfib == 0) return F3D_OK;
  if (!npts || !pt_off || !length || !x || !f || !up_mats || !up_off || !vself) return F3D_ERR_NULL;
  const size_t smem = static_cast<size_t>(6) * max_n * (1 + uprate) * sizeof(double);
  if (smem > 48 * 1024) return F3D_ERR_TOO_LARGE;
  f3d::fiber_self_flow_up_kernel<<<nfib, 128, smem, static_cast<cudaStream_t>(stream)>>>(
      npts, pt_off, length, x, f, up_mats, up_off, uprate, eta, reg, epsilon_distance, vself);
  return f3d::launch_status();
}

int f3d_grid_near_fiber(const double *grid, int64_t ngrid, const double *x, const int64_t *pt_off,
                        int32_t nfib, const double *vself, double near, double *vfib, void *stream) {
  if (ngrid < 0 || nfib < 0) return F3D_ERR_SHAPE;
  if (ngrid == 0 || nfib == 0) return F3D_OK;
  if (!grid || !x || !pt_off || !vself || !vfib) return F3D_ERR_NULL;
  f3d::grid_near_fiber_kernel<<<static_cast<unsigned>((ngrid + 127) / 128), 128, 0,
                                static_cast<cudaStream_t>(stream)>>>(grid, ngrid, x, pt_off, nfib, vself, near,
                                                                     vfib);
  return f3d::launch_status();
}

int f3d_grid_rigid_override(const double *grid, int64_t ngrid, const double *center, const double *uw,
                            double radius, double *v, void *stream) {
  if (ngrid < 0) return F3D_ERR_SHAPE;
  if (ngrid == 0) return F3D_OK;
  if (!grid || !center || !uw || !v) return F3D_ERR_NULL;
  f3d::grid_rigid_override_kernel<<<static_cast<unsigned>((ngrid + 127) / 128), 128, 0,
                                    static_cast<cudaStream_t>(stream)>>>(grid, ngrid, center, uw, radius, v);
  return f3d::launch_status();
}

}  // extern "C"
