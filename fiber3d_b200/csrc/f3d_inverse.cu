// Batched explicit inverses of small dense FP64 blocks, and the batched
// block-diagonal matrix-vector product that applies them.
//
// fiber3d's block-diagonal preconditioner (P_inv, tstep/tstep.py:950-994)
// factors every fiber block with scipy.linalg.lu_factor
// (tstep/tstep_utils.py:1405-1419) and applies lu_solve once per GMRES
// iteration.  A substitution is a chain of 2n dependent steps; a product
// with the explicit inverse is one streaming pass over the block, so for the
// fiber blocks (4N <= 128) this file forms P_b^-1 once per time step and
// applies it as a block GEMV.  The preconditioner is the same linear
// operator as fiber3d's (to rounding); only how it is evaluated changes.
//
// Inverse: Gauss-Jordan with partial (row) pivoting, in place.  Step k picks
// a row p >= k of (to 2^-20) largest |a_pk|, swaps rows k and p, and pivots
// on (k, k):
//   a_kk <- 1/a_kk,  a_kj <- a_kj / a_kk,  a_ik <- -a_ik / a_kk,
//   a_ij <- a_ij - a_ik a_kj / a_kk      (i != k, j != k, old values).
// After n steps the array holds (PA)^-1; swapping columns k and p_k for
// k = n-1 .. 0 gives A^-1.
//
// One CTA per block holds the whole NMAX x NMAX matrix in registers: thread
// t owns an 8 x 4 tile (rows 8*(t/(NMAX/4)) .., columns 4*(t%(NMAX/4)) ..),
// so a warp covers whole rows.  Per step the owners of column k publish it to
// shared memory (the pivot search is then done redundantly by every warp, no
// extra barrier), the owners of rows k and p publish those rows, and every
// thread applies the rank-1 sweep to its tile: two barriers per step.
// Blocks smaller than NMAX are padded with the identity, which the sweeps
// leave untouched.
#include <algorithm>

#include "f3d_common.cuh"

namespace f3d {

constexpr int kInvTR = 8;  // tile rows per thread
constexpr int kInvTC = 4;  // tile columns per thread

template <int NMAX>
struct InvShape {
  static constexpr int kColTiles = NMAX / kInvTC;
  static constexpr int kRowTiles = NMAX / kInvTR;
  static constexpr int kThreads = kColTiles * kRowTiles;
};

// 1/x for the pivot: the hardware approximation (rcp.approx.ftz.f64, about
// 2^-22 relative error) refined by one third-order Newton step
// y1 = y0 (1 + e + e^2), e = 1 - x y0, whose error is O(e^3): within an ulp
// or so of the correctly rounded quotient, in 4 dependent operations.
// Pivots below the normal range are reported as zero pivots by the caller.
__device__ __forceinline__ double reciprocal(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

// Step k = kb + M of the Gauss-Jordan sweep on the register tiles.
// Column k is published to shared memory and zeroed in the tiles; the pivot
// row is read back with its column-k entry taken as 1, so that one update
//   a_ij <- a_ij - (c_i / pv) u_j
// gives every entry: a_kj = u_j / pv on the pivot row (which is overwritten),
// a_ik = -c_i / pv in column k, and the elimination elsewhere.
template <int NMAX, int M>
__device__ __forceinline__ void inverse_step(double (&a)[kInvTR][kInvTC], int kb, int n, int r0,
                                             int c0, int ct, int rt, int lane, int tid,
                                             double (*s_col)[NMAX], double (*s_row)[2][NMAX],
                                             int *s_piv, int &first_zero) {
  constexpr int II = M % kInvTR;  // tile row of row k in its owner
  constexpr int JJ = M % kInvTC;  // tile column of column k in its owner
  const int k = kb + M;
  if (k >= NMAX) return;
  const int par = k & 1;
  // (a) publish column k, zero it in the tiles
  if (ct == k / kInvTC) {
#pragma unroll
    for (int i = 0; i < kInvTR; ++i) {
      s_col[par][r0 + i] = a[i][JJ];
      a[i][JJ] = 0.0;
    }
  }
  __syncthreads();
  // (b) pivot, found by every warp: the first row p >= k whose magnitude
  // has the largest leading 32 bits (sign, exponent, 20 mantissa bits), i.e.
  // a pivot within a factor 1 - 2^-20 of the column maximum -- threshold
  // partial pivoting, as stable as the exact maximum.  Two warp reductions.
  unsigned key = 0u, row = 0xFFFFFFFFu;
#pragma unroll
  for (int q = 0; q < NMAX / 32; ++q) {
    const int r = lane + 32 * q;
    if (r >= k && r < n) {
      const unsigned kq =
          static_cast<unsigned>(static_cast<unsigned long long>(__double_as_longlong(fabs(s_col[par][r]))) >> 32);
      if (row == 0xFFFFFFFFu || kq > key) { key = kq; row = static_cast<unsigned>(r); }
    }
  }
  const unsigned kmax = __reduce_max_sync(0xffffffffu, row != 0xFFFFFFFFu ? key : 0u);
  const unsigned pmin = __reduce_min_sync(0xffffffffu, (row != 0xFFFFFFFFu && key == kmax) ? row : 0xFFFFFFFFu);
  const int p = pmin < static_cast<unsigned>(n) ? static_cast<int>(pmin) : k;
  // (c) publish rows k and p (column k already zero); 16-byte stores
  if (rt == k / kInvTR) {
    double2 *dst = reinterpret_cast<double2 *>(&s_row[par][0][c0]);
    dst[0] = make_double2(a[II][0], a[II][1]);
    dst[1] = make_double2(a[II][2], a[II][3]);
  }
  if (rt == p / kInvTR) {
    const int ip = p % kInvTR;
    double v[kInvTC];
#pragma unroll
    for (int j = 0; j < kInvTC; ++j) {
      v[j] = a[0][j];
#pragma unroll
      for (int i = 1; i < kInvTR; ++i) v[j] = (ip == i) ? a[i][j] : v[j];
    }
    double2 *dst = reinterpret_cast<double2 *>(&s_row[par][1][c0]);
    dst[0] = make_double2(v[0], v[1]);
    dst[1] = make_double2(v[2], v[3]);
  }
  if (tid == 0) s_piv[k] = p;
  __syncthreads();
  // (d) swap rows k and p, then the update
  const double pv = s_col[par][p];
  const bool zero_pivot = !(fabs(pv) >= 2.2250738585072014e-308);  // zero, subnormal or NaN
  if (zero_pivot && first_zero == 0) first_zero = k + 1;
  const double pinv = zero_pivot ? 0.0 : reciprocal(pv);
  double u[kInvTC];
  {
    const double2 *src = reinterpret_cast<const double2 *>(&s_row[par][1][c0]);
    const double2 u01 = src[0], u23 = src[1];
    u[0] = u01.x; u[1] = u01.y; u[2] = u23.x; u[3] = u23.y;
  }
  if (ct == k / kInvTC) u[JJ] = 1.0;
  double c[kInvTR];
  {
    const double2 *src = reinterpret_cast<const double2 *>(&s_col[par][r0]);
#pragma unroll
    for (int i = 0; i < kInvTR / 2; ++i) {
      const double2 cc = src[i];
      c[2 * i] = cc.x;
      c[2 * i + 1] = cc.y;
    }
  }
#pragma unroll
  for (int i = 0; i < kInvTR; ++i) {
    const int r = r0 + i;
    if (r == k) {
#pragma unroll
      for (int j = 0; j < kInvTC; ++j) a[i][j] = u[j] * pinv;
    } else {
      double ci;
      if (r == p) {
        const double2 *src = reinterpret_cast<const double2 *>(&s_row[par][0][c0]);
        const double2 w01 = src[0], w23 = src[1];
        a[i][0] = w01.x; a[i][1] = w01.y; a[i][2] = w23.x; a[i][3] = w23.y;
        ci = s_col[par][k];
      } else {
        ci = c[i];
      }
      const double f = ci * pinv;
#pragma unroll
      for (int j = 0; j < kInvTC; ++j) a[i][j] = fma(-f, u[j], a[i][j]);
    }
  }
}

template <int NMAX>
__global__ void __launch_bounds__(InvShape<NMAX>::kThreads, 1)
    batched_inverse_kernel(double *__restrict__ A, const int64_t *__restrict__ moff,
                           const int32_t *__restrict__ sizes, int count, float *__restrict__ A32,
                           int32_t *__restrict__ info) {
  using S = InvShape<NMAX>;
  __shared__ __align__(16) double s_col[2][NMAX];
  __shared__ __align__(16) double s_row[2][2][NMAX];  // [parity][0: old row k, 1: old row p][col]
  __shared__ int s_piv[NMAX];
  __shared__ int s_dest[NMAX];
  const int b = blockIdx.x;
  if (b >= count) return;
  const int n = sizes[b];
  if (n <= 0 || n > NMAX) return;
  double *M = A + moff[b];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int ct = tid % S::kColTiles, rt = tid / S::kColTiles;
  const int c0 = ct * kInvTC, r0 = rt * kInvTR;

  double a[kInvTR][kInvTC];
#pragma unroll
  for (int i = 0; i < kInvTR; ++i) {
    const int r = r0 + i;
#pragma unroll
    for (int j = 0; j < kInvTC; ++j) {
      const int c = c0 + j;
      a[i][j] = (r < n && c < n) ? M[static_cast<int64_t>(r) * n + c] : (r == c ? 1.0 : 0.0);
    }
  }
  int first_zero = 0;
  // Steps run in groups of kInvTR so that k % kInvTR and k % kInvTC are
  // compile-time constants inside a step (no runtime register indexing).
  // Steps past n pivot on the identity padding and change nothing.
  for (int kb = 0; kb < n; kb += kInvTR) {
    inverse_step<NMAX, 0>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 1>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 2>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 3>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 4>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 5>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 6>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
    inverse_step<NMAX, 7>(a, kb, n, r0, c0, ct, rt, lane, tid, s_col, s_row, s_piv, first_zero);
  }
  // column unscramble: X P, swaps (k, p_k) for k = n-1 .. 0
  __syncthreads();
  if (tid == 0) {
    for (int j = 0; j < n; ++j) s_dest[j] = j;  // s_dest[j] = source column of final column j
    for (int k = n - 1; k >= 0; --k) {
      const int p = s_piv[k];
      const int t = s_dest[k];
      s_dest[k] = s_dest[p];
      s_dest[p] = t;
    }
    // invert: final position of source column c
    for (int j = 0; j < n; ++j) s_piv[s_dest[j]] = j;
    info[b] = first_zero;
  }
  __syncthreads();
  float *M32 = A32 ? A32 + moff[b] : nullptr;
#pragma unroll
  for (int i = 0; i < kInvTR; ++i) {
    const int r = r0 + i;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < kInvTC; ++j) {
      const int c = c0 + j;
      if (c >= n) continue;
      const int64_t o = static_cast<int64_t>(r) * n + s_piv[c];
      M[o] = a[i][j];
      if (M32) M32[o] = static_cast<float>(a[i][j]);
    }
  }
}

// y_b = M_b x_b for every block b (M row-major n_b x n_b at moff[b], x and y
// at voff[b]).  One CTA per block, 8 lanes per row (16-byte loads where the
// block is aligned), FP64 accumulation.
template <typename T>
__global__ void __launch_bounds__(128) block_gemv_kernel(const T *__restrict__ M,
                                                         const int64_t *__restrict__ moff,
                                                         const int64_t *__restrict__ voff,
                                                         const int32_t *__restrict__ sizes,
                                                         int count, const double *__restrict__ x,
                                                         double *__restrict__ y) {
  extern __shared__ __align__(16) double xs[];
  const int b = blockIdx.x;
  if (b >= count) return;
  const int n = sizes[b];
  const T *Mb = M + moff[b];
  const double *xb = x + voff[b];
  for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = xb[i];
  __syncthreads();
  constexpr int kVec = 16 / sizeof(T);
  const bool vec = ((reinterpret_cast<uintptr_t>(Mb) & 15) == 0) && (n % kVec == 0);
  const int sub = threadIdx.x & 7;          // lane within the row group
  const int grp = threadIdx.x >> 3;         // 16 row groups per CTA
  for (int r = grp; r < n; r += 16) {
    const T *row = Mb + static_cast<int64_t>(r) * n;
    double s = 0.0;
    if (vec) {
      for (int c = sub * kVec; c < n; c += 8 * kVec) {
        if constexpr (sizeof(T) == 8) {
          const double2 v = *reinterpret_cast<const double2 *>(row + c);
          s = fma(v.x, xs[c], s);
          s = fma(v.y, xs[c + 1], s);
        } else {
          const float4 v = *reinterpret_cast<const float4 *>(row + c);
          s = fma(static_cast<double>(v.x), xs[c], s);
          s = fma(static_cast<double>(v.y), xs[c + 1], s);
          s = fma(static_cast<double>(v.z), xs[c + 2], s);
          s = fma(static_cast<double>(v.w), xs[c + 3], s);
        }
      }
    } else {
      for (int c = sub; c < n; c += 8) s = fma(static_cast<double>(row[c]), xs[c], s);
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    if (sub == 0) y[voff[b] + r] = s;
  }
}

}  // namespace f3d

extern "C" {

int f3d_batched_inverse(double *A, const int64_t *matrix_offsets, const int32_t *sizes,
                        int32_t count, int32_t max_n, float *A32, int32_t *info, void *stream) {
  if (count < 0 || max_n < 0) return F3D_ERR_SHAPE;
  if (count == 0) return F3D_OK;
  if (!A || !matrix_offsets || !sizes || !info) return F3D_ERR_NULL;
  if (max_n > 128) return F3D_ERR_TOO_LARGE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (max_n <= 32) {
    f3d::batched_inverse_kernel<32><<<count, f3d::InvShape<32>::kThreads, 0, st>>>(
        A, matrix_offsets, sizes, count, A32, info);
  } else if (max_n <= 64) {
    f3d::batched_inverse_kernel<64><<<count, f3d::InvShape<64>::kThreads, 0, st>>>(
        A, matrix_offsets, sizes, count, A32, info);
  } else {
    f3d::batched_inverse_kernel<128><<<count, f3d::InvShape<128>::kThreads, 0, st>>>(
        A, matrix_offsets, sizes, count, A32, info);
  }
  return f3d::launch_status();
}

int f3d_block_gemv(int precision, const void *M, const int64_t *matrix_offsets,
                   const int64_t *vector_offsets, const int32_t *sizes, int32_t count,
                   int32_t max_n, const double *x, double *y, void *stream) {
  if (count < 0 || max_n < 0) return F3D_ERR_SHAPE;
  if (count == 0) return F3D_OK;
  if (!M || !matrix_offsets || !vector_offsets || !sizes || !x || !y) return F3D_ERR_NULL;
  if (x == y) return F3D_ERR_ARG;
  const size_t smem = static_cast<size_t>(max_n) * sizeof(double);
  if (smem > 48 * 1024) return F3D_ERR_TOO_LARGE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (precision == F3D_FP64) {
    f3d::block_gemv_kernel<double><<<count, 128, smem, st>>>(
        static_cast<const double *>(M), matrix_offsets, vector_offsets, sizes, count, x, y);
  } else if (precision == F3D_FP32C) {
    f3d::block_gemv_kernel<float><<<count, 128, smem, st>>>(
        static_cast<const float *>(M), matrix_offsets, vector_offsets, sizes, count, x, y);
  } else {
    return F3D_ERR_ARG;
  }
  return f3d::launch_status();
}

}  // extern "C"
