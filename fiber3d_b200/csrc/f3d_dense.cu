// Dense 3n x 3n operator builders (set-up work: the periphery and body
// preconditioners factor these matrices once).  HBM-write bound: one thread
// writes one 3x3 block; a warp covers 32 consecutive column blocks of one
// row block, so each of the three rows is written as a contiguous run.
//
//   stresslet_kernel_times_normal_numba  python/kernels/kernels.py:1063-1120
//   oseen_tensor (input_format 'r')      python/kernels/kernels.py:31-116
//   complementary_kernel                 python/kernels/kernels.py:1286-1295
//   stresslet_kernel (input_format 'r')  python/kernels/kernels.py:911-992
#include "f3d_common.cuh"

namespace f3d {

__global__ void stresslet_normal_dense_kernel(const double *__restrict__ x,
                                              const double *__restrict__ nrm, double *M,
                                              int64_t n, int64_t ld, double factor, double eps2,
                                              double reg2) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  if (j >= n) return;
  double *row = M + 3 * i * ld + 3 * j;
  if (i == j) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) row[a * ld + b] = 0.0;
    return;
  }
  const double r[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
  double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  if (r2 < eps2) r2 += reg2;
  const double rn = sqrt(r2);
  const double rdn = r[0] * nrm[3 * j] + r[1] * nrm[3 * j + 1] + r[2] * nrm[3 * j + 2];
  const double s = factor * rdn / (rn * rn * rn * rn * rn);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) row[a * ld + b] = s * r[a] * r[b];
}

// Row block i = target, column block j = source.
__global__ void oseen_tensor_dense_kernel(const double *__restrict__ xs,
                                          const double *__restrict__ xt, double *G, int64_t ns,
                                          int64_t ld, double factor, double eps2, double reg2) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  if (j >= ns) return;
  // oseen_tensor uses r = x_j - x_i; only r r^T enters, so the sign is moot.
  const double r[3] = {xs[3 * j] - xt[3 * i], xs[3 * j + 1] - xt[3 * i + 1],
                       xs[3 * j + 2] - xt[3 * i + 2]};
  double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  // kernels.py:86-93: dr > eps is plain, dr <= eps is regularised.
  if (!(r2 > eps2)) r2 += reg2;
  const double d = sqrt(r2);
  const double fr = factor / d;
  const double gr = factor / (d * d * d);
  double *row = G + 3 * i * ld + 3 * j;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) row[a * ld + b] = (a == b ? fr : 0.0) + gr * r[a] * r[b];
}

// The 3-index stresslet tensor: S[3i+a, 3j+b, c] = fr dr_a dr_b dr_c with
// dr = x_j - x_i, fr = -3/(4 pi eta dr^5) for dr > eps and
// -3/(4 pi eta (dr^2 + reg^2)^(5/2)) otherwise (the diagonal blocks are then
// zero because dr = 0).  One thread writes the 27 entries of pair (i, j):
// for each a, nine consecutive doubles, so a warp writes 32 x 72 contiguous
// bytes per row.
__global__ void stresslet_tensor_dense_kernel(const double *__restrict__ x, double *S, int64_t n,
                                              double factor, double eps, double reg2) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  if (j >= n) return;
  const double dr[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
  const double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
  const double d = sqrt(r2);
  const double fr = (d > eps) ? factor / pow(d, 5.0) : factor / pow(r2 + reg2, 2.5);
  const int64_t ld = 9 * n;  // doubles per row (3n columns x 3)
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double *row = S + (3 * i + a) * ld + 9 * j;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) row[3 * b + c] = fr * dr[a] * dr[b] * dr[c];
  }
}

__global__ void complementary_dense_kernel(const double *__restrict__ nrm, double *C, int64_t m,
                                           int64_t ld) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t r = blockIdx.y;
  if (c >= m) return;
  C[r * ld + c] = nrm[r] * nrm[c];
}

static int check_dense(const void *a, const void *b, int64_t n, int64_t ld) {
  if (n < 0 || ld < 3 * n) return F3D_ERR_SHAPE;
  if (n > 0 && (!a || !b)) return F3D_ERR_NULL;
  if (!aligned(a, 8) || !aligned(b, 8)) return F3D_ERR_ALIGN;
  if (n > 65535) return F3D_ERR_TOO_LARGE;  // grid.y carries the row block
  return F3D_OK;
}

}  // namespace f3d

extern "C" {

int f3d_stresslet_times_normal_dense(const double *r_vectors, const double *normal, double *M,
                                     int64_t n, int64_t ld, double eta, double reg,
                                     double epsilon_distance, void *stream) {
  int rc = f3d::check_dense(r_vectors, M, n, ld);
  if (rc) return rc;
  if (n > 0 && !normal) return F3D_ERR_NULL;
  if (n == 0) return F3D_OK;
  dim3 grid(static_cast<unsigned>((n + 127) / 128), static_cast<unsigned>(n));
  f3d::stresslet_normal_dense_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      r_vectors, normal, M, n, ld, -3.0 / (4.0 * f3d::kPi * eta),
      epsilon_distance * epsilon_distance, reg * reg);
  return f3d::launch_status();
}

int f3d_oseen_tensor_dense(const double *r_vectors, double *G, int64_t n, int64_t ld, double eta,
                           double reg, double epsilon_distance, void *stream) {
  int rc = f3d::check_dense(r_vectors, G, n, ld);
  if (rc) return rc;
  if (n == 0) return F3D_OK;
  dim3 grid(static_cast<unsigned>((n + 127) / 128), static_cast<unsigned>(n));
  f3d::oseen_tensor_dense_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      r_vectors, r_vectors, G, n, ld, 1.0 / (8.0 * f3d::kPi * eta),
      epsilon_distance * epsilon_distance, reg * reg);
  return f3d::launch_status();
}

int f3d_oseen_tensor_source_target_dense(const double *r_source, const double *r_target,
                                         double *G, int64_t ns, int64_t nt, int64_t ld,
                                         double eta, double reg, double epsilon_distance,
                                         void *stream) {
  if (ns < 0 || nt < 0 || ld < 3 * ns) return F3D_ERR_SHAPE;
  if (ns == 0 || nt == 0) return F3D_OK;
  if (!r_source || !r_target || !G) return F3D_ERR_NULL;
  if (!f3d::aligned(r_source, 8) || !f3d::aligned(r_target, 8) || !f3d::aligned(G, 8))
    return F3D_ERR_ALIGN;
  if (nt > 65535) return F3D_ERR_TOO_LARGE;
  dim3 grid(static_cast<unsigned>((ns + 127) / 128), static_cast<unsigned>(nt));
  f3d::oseen_tensor_dense_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      r_source, r_target, G, ns, ld, 1.0 / (8.0 * f3d::kPi * eta),
      epsilon_distance * epsilon_distance, reg * reg);
  return f3d::launch_status();
}

int f3d_stresslet_tensor_dense(const double *r_vectors, double *S, int64_t n, double eta, double reg,
                               double epsilon_distance, void *stream) {
  int rc = f3d::check_dense(r_vectors, S, n, 3 * n);
  if (rc) return rc;
  if (n == 0) return F3D_OK;
  dim3 grid(static_cast<unsigned>((n + 127) / 128), static_cast<unsigned>(n));
  f3d::stresslet_tensor_dense_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      r_vectors, S, n, -3.0 / (4.0 * f3d::kPi * eta), epsilon_distance, reg * reg);
  return f3d::launch_status();
}

int f3d_complementary_dense(const double *normal, double *C, int64_t n, int64_t ld,
                            void *stream) {
  int rc = f3d::check_dense(normal, C, n, ld);
  if (rc) return rc;
  if (n == 0) return F3D_OK;
  const int64_t m = 3 * n;
  if (m > 65535) return F3D_ERR_TOO_LARGE;
  dim3 grid(static_cast<unsigned>((m + 255) / 256), static_cast<unsigned>(m));
  f3d::complementary_dense_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(normal, C,
                                                                                       m, ld);
  return f3d::launch_status();
}

}  // extern "C"
