// Surface operators: the periphery (shell) double layer with singularity
// subtraction and its null-space correction, rigid-body rows, and their
// dense preconditioner blocks.
//
// Reference (fiber3d, python/):
//   singularity-subtraction vectors e_x, e_y, e_z   periphery/periphery.py:75-98,
//                                                   body/body.py:325-346
//   shell operator M = S - I_E - diag(1/w) (+ n n^T) tstep/tstep.py:327-351
//   its application in the matvec                   tstep/tstep.py:1097-1104
//   body rows: -E mu - K U + v ; -K^T lambda + U    tstep/tstep.py:1118-1143
//   body preconditioner block                       tstep/tstep_utils.py:1341-1386
// Unknown q = the weighted double-layer density (x_all slice); mu = q / w.
// E is stored per node as a 3x3 row-major matrix E[i][a][c] = e_c(i)_a.
#include <algorithm>

#include "f3d_common.cuh"

namespace f3d {

int pair_sum_impl(int kernel, int precision, int self_mode, const double *rs, const double *rt,
                  const double *dens, const double *nrm, const int32_t *gs, const int32_t *gt,
                  double *out, int64_t ns, int64_t nt, double eta, double reg, double eps,
                  int accumulate, const f3d_pair_shape *shape, void *ws, size_t ws_bytes,
                  cudaStream_t st);

__global__ void unit_density_kernel(const double *w, double *dens, int64_t n, int c) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dens[3 * i + 0] = (c == 0) ? w[i] : 0.0;
  dens[3 * i + 1] = (c == 1) ? w[i] : 0.0;
  dens[3 * i + 2] = (c == 2) ? w[i] : 0.0;
}

__global__ void scatter_column_kernel(const double *col, double *E, int64_t n, int c) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int a = 0; a < 3; ++a) E[9 * i + 3 * a + c] = col[3 * i + a];
}

// s = sum_j n_j . q_j, one CTA, fixed reduction order.
__global__ void __launch_bounds__(1024) normal_dot_kernel(const double *nrm, const double *q,
                                                          int64_t n, double *s) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
    acc += nrm[3 * i] * q[3 * i] + nrm[3 * i + 1] * q[3 * i + 1] + nrm[3 * i + 2] * q[3 * i + 2];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) *s = v;
  }
}

// y_i = B_i x_i for n row-major 3 x 3 blocks B (9 doubles per node).
__global__ void block3_gemv_kernel(const double *__restrict__ B, const double *__restrict__ x, double *y,
                                   int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *b = B + 9 * i;
  const double x0 = x[3 * i], x1 = x[3 * i + 1], x2 = x[3 * i + 2];
  y[3 * i] = fma(b[0], x0, fma(b[1], x1, b[2] * x2));
  y[3 * i + 1] = fma(b[3], x0, fma(b[4], x1, b[5] * x2));
  y[3 * i + 2] = fma(b[6], x0, fma(b[7], x1, b[8] * x2));
}

// Binv_i = B_i^-1, B_i = -(E_i + I) / w_i + n_i n_i^T: the 3 x 3 diagonal
// blocks of the dense shell operator.  The inverse is the adjugate over the
// determinant (cofactor expansion with fused products); a block whose
// determinant is zero or not finite is counted in *info.
__global__ void shell_block_inverse_kernel(const double *__restrict__ E, const double *__restrict__ w,
                                           const double *__restrict__ nrm, double *Binv, int64_t n,
                                           int32_t *info) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double inv_w = 1.0 / w[i];
  const double n0 = nrm[3 * i], n1 = nrm[3 * i + 1], n2 = nrm[3 * i + 2];
  const double nn[3] = {n0, n1, n2};
  double b[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) b[r][c] = fma(nn[r], nn[c], -(E[9 * i + 3 * r + c] + (r == c ? 1.0 : 0.0)) * inv_w);
  const double c00 = fma(b[1][1], b[2][2], -b[1][2] * b[2][1]);
  const double c01 = fma(b[1][2], b[2][0], -b[1][0] * b[2][2]);
  const double c02 = fma(b[1][0], b[2][1], -b[1][1] * b[2][0]);
  const double det = fma(b[0][0], c00, fma(b[0][1], c01, b[0][2] * c02));
  if (!(det != 0.0) || !isfinite(det)) {
    if (info) atomicAdd(info, 1);
  }
  const double id = 1.0 / det;
  double *o = Binv + 9 * i;
  o[0] = c00 * id;
  o[1] = fma(b[0][2], b[2][1], -b[0][1] * b[2][2]) * id;
  o[2] = fma(b[0][1], b[1][2], -b[0][2] * b[1][1]) * id;
  o[3] = c01 * id;
  o[4] = fma(b[0][0], b[2][2], -b[0][2] * b[2][0]) * id;
  o[5] = fma(b[0][2], b[1][0], -b[0][0] * b[1][2]) * id;
  o[6] = c02 * id;
  o[7] = fma(b[0][1], b[2][0], -b[0][0] * b[2][1]) * id;
  o[8] = fma(b[0][0], b[1][1], -b[0][1] * b[1][0]) * id;
}

// res_i = v_i - E_i mu_i - mu_i + n_i s   (mu = q / w)
__global__ void shell_residual_kernel(const double *__restrict__ v, const double *__restrict__ E,
                                      const double *__restrict__ w, const double *__restrict__ nrm,
                                      const double *__restrict__ q, const double *__restrict__ s,
                                      double *res, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double inv = 1.0 / w[i];
  const double mu[3] = {q[3 * i] * inv, q[3 * i + 1] * inv, q[3 * i + 2] * inv};
  const double ss = *s;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double *e = E + 9 * i + 3 * a;
    res[3 * i + a] = v[3 * i + a] - (e[0] * mu[0] + e[1] * mu[1] + e[2] * mu[2]) - mu[a] + nrm[3 * i + a] * ss;
  }
}

// One CTA per body.  x_b = [lambda (3nb), U (3), Omega (3)].
__global__ void __launch_bounds__(256) body_residual_kernel(
    const int64_t *node_off, const int64_t *x_off, const double *__restrict__ nodes,
    const double *__restrict__ center, const double *__restrict__ E, const double *__restrict__ w,
    const double *__restrict__ v, const double *__restrict__ x, double *res) {
  const int b = blockIdx.x;
  const int64_t i0 = node_off[b], i1 = node_off[b + 1];
  const int64_t xo = x_off[b];
  const int64_t nb = i1 - i0;
  const double *lam = x + xo;
  const double *U = x + xo + 3 * nb;
  const double cx = center[3 * b], cy = center[3 * b + 1], cz = center[3 * b + 2];
  double f[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t k = threadIdx.x; k < nb; k += blockDim.x) {
    const int64_t i = i0 + k;
    const double r[3] = {nodes[3 * i] - cx, nodes[3 * i + 1] - cy, nodes[3 * i + 2] - cz};
    const double l[3] = {lam[3 * k], lam[3 * k + 1], lam[3 * k + 2]};
    const double inv = 1.0 / w[i];
    const double mu[3] = {l[0] * inv, l[1] * inv, l[2] * inv};
    // K U = U + Omega x r
    const double ku[3] = {U[0] + U[4] * r[2] - U[5] * r[1], U[1] + U[5] * r[0] - U[3] * r[2],
                          U[2] + U[3] * r[1] - U[4] * r[0]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double *e = E + 9 * i + 3 * a;
      res[xo + 3 * k + a] = v[3 * i + a] - (e[0] * mu[0] + e[1] * mu[1] + e[2] * mu[2]) - ku[a];
    }
    // K^T lambda = [sum lambda, sum r x lambda]
    f[0] += l[0]; f[1] += l[1]; f[2] += l[2];
    f[3] += r[1] * l[2] - r[2] * l[1];
    f[4] += r[2] * l[0] - r[0] * l[2];
    f[5] += r[0] * l[1] - r[1] * l[0];
  }
  __shared__ double red[6][8];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double a = f[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = a;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double a = 0.0;
    for (int wi = 0; wi < static_cast<int>(blockDim.x >> 5); ++wi) a += red[threadIdx.x][wi];
    res[xo + 3 * nb + threadIdx.x] = -a + U[threadIdx.x];
  }
}

// Dense surface operator block: rows/cols 3n (+6 for a rigid body).
// mode 0 (shell): M = S - blockdiag(E_i/w_i + I/w_i) + n n^T
// mode 1 (body):  [[S - blockdiag(E_i/w_i), -K], [-K^T, I6]]
__global__ void surface_dense_kernel(const double *__restrict__ x, const double *__restrict__ nrm,
                                     const double *__restrict__ E, const double *__restrict__ w,
                                     const double *center, double *M, int64_t n, int64_t ld,
                                     double factor, double eps2, double reg2, int mode) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  const int64_t nc = (mode == 1) ? n + 2 : n;  // column blocks (2 extra for U, Omega)
  if (j >= nc) return;
  if (i >= n) {
    // rigid-body rows: -K^T for column blocks j < n, identity on U, Omega
    const int64_t rb = i - n;  // 0: force rows (U), 1: torque rows (Omega)
    double *row = M + 3 * i * ld + 3 * j;
    if (j < n) {
      const double r[3] = {x[3 * j] - center[0], x[3 * j + 1] - center[1], x[3 * j + 2] - center[2]};
      // -K^T: force rows -I; torque rows -(r x .) as a matrix
      const double T[3][3] = {{0.0, -r[2], r[1]}, {r[2], 0.0, -r[0]}, {-r[1], r[0], 0.0}};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) row[a * ld + b] = (rb == 0) ? -(a == b ? 1.0 : 0.0) : -T[a][b];
    } else {
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) row[a * ld + b] = (j - n == rb && a == b) ? 1.0 : 0.0;
    }
    return;
  }
  double *row = M + 3 * i * ld + 3 * j;
  if (j >= n) {
    // -K columns: U columns -I, Omega columns -(Omega x r) = -rot_i
    const double r[3] = {x[3 * i] - center[0], x[3 * i + 1] - center[1], x[3 * i + 2] - center[2]};
    const double rot[3][3] = {{0.0, r[2], -r[1]}, {-r[2], 0.0, r[0]}, {r[1], -r[0], 0.0}};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) row[a * ld + b] = (j == n) ? -(a == b ? 1.0 : 0.0) : -rot[a][b];
    return;
  }
  double blk[3][3];
  if (i == j) {
    const double inv = 1.0 / w[i];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        blk[a][b] = -E[9 * i + 3 * a + b] * inv - ((mode == 0 && a == b) ? inv : 0.0);
  } else {
    const double r[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
    double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (r2 < eps2) r2 += reg2;
    const double rn = sqrt(r2);
    const double rdn = r[0] * nrm[3 * j] + r[1] * nrm[3 * j + 1] + r[2] * nrm[3 * j + 2];
    const double s = factor * rdn / (rn * rn * rn * rn * rn);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) blk[a][b] = s * r[a] * r[b];
  }
  if (mode == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) blk[a][b] += nrm[3 * i + a] * nrm[3 * j + b];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) row[a * ld + b] = blk[a][b];
}

// dst[seg_dst[s] + k] = src[seg_src[s] + k], k < seg_len[s]
__global__ void gather_segments_kernel(const double *__restrict__ src, double *dst,
                                       const int64_t *seg_src, const int64_t *seg_dst,
                                       const int64_t *seg_len, int nseg) {
  const int s = blockIdx.y;
  if (s >= nseg) return;
  const int64_t len = seg_len[s];
  for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < len;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[seg_dst[s] + k] = src[seg_src[s] + k];
}

// Per body b: the nvec[b] 3-vectors at x + off[b] are multiplied by R_b
// (transpose = 0) or R_b^T (transpose = 1), R_b row-major at R + 9 b.
// Rigid-body surfaces at a new location/orientation: node i of body b
// (body_of[i]) gets x = R_b x_ref + c_b, n = R_b n_ref and, for the 3 x 3
// singularity-vector map E_i (E[9i + 3a + c] = e_c(i)_a), E = R_b E_ref R_b^T.
// One thread per node.
__global__ void rigid_body_update_kernel(const int32_t *__restrict__ body_of,
                                         const double *__restrict__ R, const double *__restrict__ loc,
                                         const double *__restrict__ ref_nodes,
                                         const double *__restrict__ ref_normals,
                                         const double *__restrict__ ref_E, int64_t nnodes,
                                         double *__restrict__ nodes, double *__restrict__ normals,
                                         double *__restrict__ E) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nnodes) return;
  const int b = body_of[i];
  double r[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) r[q] = R[9 * b + q];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double x = loc[3 * b + a], nn = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      x = fma(r[3 * a + c], ref_nodes[3 * i + c], x);
      nn = fma(r[3 * a + c], ref_normals[3 * i + c], nn);
    }
    nodes[3 * i + a] = x;
    normals[3 * i + a] = nn;
  }
  if (ref_E && E) {
    double t[9];  // t = R E_ref
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double v = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) v = fma(r[3 * a + m], ref_E[9 * i + 3 * m + c], v);
        t[3 * a + c] = v;
      }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double v = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) v = fma(t[3 * a + m], r[3 * c + m], v);
        E[9 * i + 3 * a + c] = v;
      }
  }
}

// One thread per rigid body: the time-step update of tstep.py:1403-1407
// from the body's velocities in the solution (U at sol[vel_off[b]], Omega at
// sol[vel_off[b] + 3]): loc += dt U; q <- q_dt q with q_dt = (cos(a/2),
// sin(a/2) phi/a), phi = dt Omega, a = |phi| (the identity when a == 0;
// quaternion.py:14-38); then R(q) (quaternion.py:41-53) into R.
__global__ void body_advance_kernel(const double *__restrict__ sol, const int64_t *__restrict__ vel_off,
                                    int nbody, double dt, double *__restrict__ loc,
                                    double *__restrict__ quat, double *__restrict__ R) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbody) return;
  const double *u = sol + vel_off[b];
  for (int c = 0; c < 3; ++c) loc[3 * b + c] = __dadd_rn(loc[3 * b + c], __dmul_rn(dt, u[c]));
  const double f0 = u[3] * dt, f1 = u[4] * dt, f2 = u[5] * dt;
  const double a = sqrt(f0 * f0 + f1 * f1 + f2 * f2);
  double qs = 1.0, q0 = 0.0, q1 = 0.0, q2 = 0.0;
  if (a != 0.0) {
    double sh, ch;
    sincos(0.5 * a, &sh, &ch);
    qs = ch;
    q0 = sh * (f0 / a); q1 = sh * (f1 / a); q2 = sh * (f2 / a);
  }
  const double rs = quat[4 * b], r0 = quat[4 * b + 1], r1 = quat[4 * b + 2], r2 = quat[4 * b + 3];
  const double s = qs * rs - (q0 * r0 + q1 * r1 + q2 * r2);
  const double p0 = qs * r0 + rs * q0 + (q1 * r2 - q2 * r1);
  const double p1 = qs * r1 + rs * q1 + (q2 * r0 - q0 * r2);
  const double p2 = qs * r2 + rs * q2 + (q0 * r1 - q1 * r0);
  quat[4 * b] = s; quat[4 * b + 1] = p0; quat[4 * b + 2] = p1; quat[4 * b + 3] = p2;
  const double d = s * s - 0.5;
  double *m = R + 9 * b;
  m[0] = 2.0 * (p0 * p0 + d); m[1] = 2.0 * (p0 * p1 - s * p2); m[2] = 2.0 * (p0 * p2 + s * p1);
  m[3] = 2.0 * (p1 * p0 + s * p2); m[4] = 2.0 * (p1 * p1 + d); m[5] = 2.0 * (p1 * p2 - s * p0);
  m[6] = 2.0 * (p2 * p0 - s * p1); m[7] = 2.0 * (p2 * p1 + s * p0); m[8] = 2.0 * (p2 * p2 + d);
}

__global__ void rotate_blocks_kernel(double *x, const int64_t *off, const int32_t *nvec,
                                     const double *R, int transpose) {
  const int b = blockIdx.x;
  double r[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = R[9 * b + i];
  double *v = x + off[b];
  for (int k = threadIdx.x; k < nvec[b]; k += blockDim.x) {
    const double a0 = v[3 * k], a1 = v[3 * k + 1], a2 = v[3 * k + 2];
    if (transpose) {
      v[3 * k] = r[0] * a0 + r[3] * a1 + r[6] * a2;
      v[3 * k + 1] = r[1] * a0 + r[4] * a1 + r[7] * a2;
      v[3 * k + 2] = r[2] * a0 + r[5] * a1 + r[8] * a2;
    } else {
      v[3 * k] = r[0] * a0 + r[1] * a1 + r[2] * a2;
      v[3 * k + 1] = r[3] * a0 + r[4] * a1 + r[5] * a2;
      v[3 * k + 2] = r[6] * a0 + r[7] * a1 + r[8] * a2;
    }
  }
}

}  // namespace f3d

extern "C" {

int f3d_rigid_body_update(const int32_t *body_of, const double *R, const double *loc,
                          const double *ref_nodes, const double *ref_normals, const double *ref_E,
                          int64_t nnodes, double *nodes, double *normals, double *E, void *stream) {
  if (nnodes < 0) return F3D_ERR_SHAPE;
  if (nnodes == 0) return F3D_OK;
  if (!body_of || !R || !loc || !ref_nodes || !ref_normals || !nodes || !normals) return F3D_ERR_NULL;
  if ((ref_E == nullptr) != (E == nullptr)) return F3D_ERR_NULL;
  const unsigned grid = static_cast<unsigned>((nnodes + 127) / 128);
  f3d::rigid_body_update_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      body_of, R, loc, ref_nodes, ref_normals, ref_E, nnodes, nodes, normals, E);
  return f3d::launch_status();
}

int f3d_body_advance(const double *sol, const int64_t *vel_off, int32_t nbody, double dt, double *loc,
                     double *quat, double *R, void *stream) {
  if (nbody < 0) return F3D_ERR_SHAPE;
  if (nbody == 0) return F3D_OK;
  if (!sol || !vel_off || !loc || !quat || !R) return F3D_ERR_NULL;
  const unsigned grid = static_cast<unsigned>((nbody + 127) / 128);
  f3d::body_advance_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(sol, vel_off, nbody, dt, loc,
                                                                               quat, R);
  return f3d::launch_status();
}

int f3d_rotate_blocks(double *x, const int64_t *offsets, const int32_t *nvec, const double *R,
                      int32_t nbody, int transpose, void *stream) {
  if (nbody < 0) return F3D_ERR_SHAPE;
  if (nbody == 0) return F3D_OK;
  if (!x || !offsets || !nvec || !R) return F3D_ERR_NULL;
  f3d::rotate_blocks_kernel<<<nbody, 256, 0, static_cast<cudaStream_t>(stream)>>>(x, offsets, nvec, R,
                                                                                  transpose);
  return f3d::launch_status();
}


int f3d_singularity_vectors_workspace_bytes(int64_t n, size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  if (n < 0) return F3D_ERR_SHAPE;
  size_t pw = 0;
  int rc = f3d_pair_workspace_bytes(F3D_KERNEL_STRESSLET, F3D_FP64, n, n, nullptr, &pw);
  if (rc) return rc;
  *bytes = f3d::round_up(static_cast<size_t>(n) * 6 * sizeof(double), 256) + pw;
  return F3D_OK;
}

int f3d_singularity_vectors(const double *nodes, const double *normals, const double *weights,
                            double *E, int64_t n, double eta, double reg, double epsilon_distance,
                            void *workspace, size_t workspace_bytes, void *stream) {
  if (n < 0) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  if (!nodes || !normals || !weights || !E) return F3D_ERR_NULL;
  size_t need = 0;
  int rc = f3d_singularity_vectors_workspace_bytes(n, &need);
  if (rc) return rc;
  if (!workspace || workspace_bytes < need) return F3D_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double *dens = static_cast<double *>(workspace);
  double *col = dens + 3 * n;
  const size_t head = f3d::round_up(static_cast<size_t>(n) * 6 * sizeof(double), 256);
  unsigned char *pws = static_cast<unsigned char *>(workspace) + head;
  const unsigned nb = static_cast<unsigned>((n + 255) / 256);
  for (int c = 0; c < 3; ++c) {
    f3d::unit_density_kernel<<<nb, 256, 0, st>>>(weights, dens, n, c);
    if ((rc = f3d::launch_status())) return rc;
    rc = f3d::pair_sum_impl(F3D_KERNEL_STRESSLET, F3D_FP64, F3D_SELF_SKIP_INDEX, nodes, nodes, dens,
                            normals, nullptr, nullptr, col, n, n, eta, reg, epsilon_distance, 0,
                            nullptr, pws, workspace_bytes - head, st);
    if (rc) return rc;
    f3d::scatter_column_kernel<<<nb, 256, 0, st>>>(col, E, n, c);
    if ((rc = f3d::launch_status())) return rc;
  }
  return F3D_OK;
}

int f3d_shell_residual(const double *v, const double *E, const double *weights,
                       const double *normals, const double *q, double *res, int64_t n,
                       double *scratch, void *stream) {
  if (n < 0) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  if (!v || !E || !weights || !normals || !q || !res || !scratch) return F3D_ERR_NULL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  f3d::normal_dot_kernel<<<1, 1024, 0, st>>>(normals, q, n, scratch);
  int rc = f3d::launch_status();
  if (rc) return rc;
  f3d::shell_residual_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
      v, E, weights, normals, q, scratch, res, n);
  return f3d::launch_status();
}

int f3d_block3_gemv(const double *B, const double *x, double *y, int64_t n, void *stream) {
  if (n < 0) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  if (!B || !x || !y) return F3D_ERR_NULL;
  if (x == y) return F3D_ERR_ARG;
  f3d::block3_gemv_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      B, x, y, n);
  return f3d::launch_status();
}

int f3d_shell_block_inverse(const double *E, const double *weights, const double *normals, double *Binv,
                            int64_t n, int32_t *info, void *stream) {
  if (n < 0) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  if (!E || !weights || !normals || !Binv) return F3D_ERR_NULL;
  f3d::shell_block_inverse_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0,
                                    static_cast<cudaStream_t>(stream)>>>(E, weights, normals, Binv, n, info);
  return f3d::launch_status();
}

int f3d_body_residual(int32_t nbody, const int64_t *node_off, const int64_t *x_off,
                      const double *nodes, const double *centers, const double *E,
                      const double *weights, const double *v, const double *x, double *res,
                      void *stream) {
  if (nbody < 0) return F3D_ERR_SHAPE;
  if (nbody == 0) return F3D_OK;
  if (!node_off || !x_off || !nodes || !centers || !E || !weights || !v || !x || !res)
    return F3D_ERR_NULL;
  f3d::body_residual_kernel<<<nbody, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      node_off, x_off, nodes, centers, E, weights, v, x, res);
  return f3d::launch_status();
}

int f3d_surface_dense(int mode, const double *nodes, const double *normals, const double *E,
                      const double *weights, const double *center, double *M, int64_t n,
                      int64_t ld, double eta, double reg, double epsilon_distance, void *stream) {
  if (mode != 0 && mode != 1) return F3D_ERR_ARG;
  const int64_t dim = (mode == 1) ? 3 * n + 6 : 3 * n;
  if (n < 0 || ld < dim) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  if (!nodes || !normals || !E || !weights || !M || (mode == 1 && !center)) return F3D_ERR_NULL;
  const int64_t rows = (mode == 1) ? n + 2 : n;
  if (rows > 65535) return F3D_ERR_TOO_LARGE;
  const int64_t cols = rows;
  dim3 grid(static_cast<unsigned>((cols + 127) / 128), static_cast<unsigned>(rows));
  f3d::surface_dense_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      nodes, normals, E, weights, center, M, n, ld, -3.0 / (4.0 * f3d::kPi * eta),
      epsilon_distance * epsilon_distance, reg * reg, mode);
  return f3d::launch_status();
}

int f3d_gather_segments(const double *src, double *dst, const int64_t *seg_src,
                        const int64_t *seg_dst, const int64_t *seg_len, int32_t nseg,
                        int64_t max_len, void *stream) {
  if (nseg < 0 || max_len < 0) return F3D_ERR_SHAPE;
  if (nseg == 0 || max_len == 0) return F3D_OK;
  if (!src || !dst || !seg_src || !seg_dst || !seg_len) return F3D_ERR_NULL;
  if (nseg > 65535) return F3D_ERR_TOO_LARGE;
  const unsigned gx = static_cast<unsigned>(std::min<int64_t>((max_len + 255) / 256, 1024));
  dim3 grid(gx, static_cast<unsigned>(nseg));
  f3d::gather_segments_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      src, dst, seg_src, seg_dst, seg_len, nseg);
  return f3d::launch_status();
}

}  // extern "C"
