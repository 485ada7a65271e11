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
// Blocks of up to 32 rows (batched_inverse_kernel<32>): one CTA per block
// holds the whole NMAX x NMAX matrix in registers, thread t an 8 x 4 tile
// (rows 8*(t/(NMAX/4)) .., columns 4*(t%(NMAX/4)) ..), so a warp covers
// whole rows.  Per step the owners of column k publish it to
// shared memory (the pivot search is then done redundantly by every warp, no
// extra barrier), the owners of rows k and p publish those rows, and every
// thread applies the rank-1 sweep to its tile: two barriers per step.
// Blocks smaller than NMAX are padded with the identity, which the sweeps
// leave untouched.  Blocks of 33..128 rows take the blocked form
// (batched_inverse_tc_kernel): 16-column panels, no row exchanges, and the
// rank-16 updates on the FP64 tensor cores.
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

// Blocked Gauss-Jordan for blocks of 33..128 rows (NMAX 64 or 128): one CTA
// per block, the block in shared memory (padded with the identity), 16
// pivots per panel.
//  * Panel: NMAX threads, one row each with the row's 16 panel entries in
//    registers, run the 16 sweeps restricted to the panel columns.  Partial
//    pivoting: the pivot of step k is the first row whose |a_ik|, rounded
//    toward zero to float with its last 8 mantissa bits cleared, is largest
//    among the rows not yet pivoted (a pivot within 2^-16 of the column
//    maximum).  The key (those bits, then 128 - row) makes the search one
//    warp max-reduction and a max over the warps; each warp's winner posts
//    its row with its key, so a step needs one barrier (posts double
//    buffered by step parity).  Rows are never exchanged: the pivot rows are
//    recorded instead (perm).
//  * Update: every other column moves by W R (W the panel after its sweeps,
//    R the old entries of the panel's 16 pivot rows), the pivot rows
//    themselves starting from zero: one m16n8k16 step on the FP64 tensor
//    cores per 16 x 8 tile.
// Sweeping pivot (perm[k], k) for every k leaves X with X[perm[k], j] =
// (PA)^-1 (k, j), so A^-1 (k, perm[j]) = X[perm[k], j].
template <int NMAX>
struct TcInv {
  static constexpr int kS = NMAX + 4;  // block row stride (doubles): B-fragment reads 4t + g apart
  static constexpr int kWS = 20;       // W panel row stride: A-fragment reads 4g + t apart
  static constexpr int kPanels = NMAX / 16;
  static constexpr int kThreads = 256;
  static constexpr size_t kSmem =
      (static_cast<size_t>(NMAX) * kS + static_cast<size_t>(NMAX) * kWS + 16 * static_cast<size_t>(kS)) *
      sizeof(double);
};

template <int NMAX>
__global__ void __launch_bounds__(256, 1)
    batched_inverse_tc_kernel(double *__restrict__ A, const int64_t *__restrict__ moff,
                              const int32_t *__restrict__ sizes, int count, float *__restrict__ A32,
                              int32_t *__restrict__ info) {
  using T = TcInv<NMAX>;
  constexpr int S = T::kS;
  extern __shared__ __align__(16) unsigned char tc_smem[];
  double *X = reinterpret_cast<double *>(tc_smem);  // [NMAX][S]
  double *Ws = X + NMAX * S;                         // [NMAX][kWS]
  double *Rs = Ws + NMAX * T::kWS;                   // [16][S]
  __shared__ unsigned s_key[2][NMAX / 32];
  __shared__ __align__(16) double s_cand[2][NMAX / 32][16];  // each warp's best row, by step parity
  __shared__ int s_perm[NMAX];   // pivot row of step k
  __shared__ int s_iperm[NMAX];  // step whose pivot is row r
  __shared__ int s_panel[NMAX];  // panel in which row r was a pivot (-1: not yet)
  const int b = blockIdx.x;
  if (b >= count) return;
  const int n = sizes[b];
  if (n <= 0 || n > NMAX) return;
  double *M = A + moff[b];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < NMAX * NMAX; e += T::kThreads) {
    const int r = e / NMAX, c = e % NMAX;
    X[r * S + c] = (r < n && c < n) ? M[static_cast<int64_t>(r) * n + c] : (r == c ? 1.0 : 0.0);
  }
  for (int r = tid; r < NMAX; r += T::kThreads) s_panel[r] = -1;
  __syncthreads();
  int first_zero = 0;  // kept by thread 0
  for (int p = 0; p < T::kPanels; ++p) {
    const int c0 = 16 * p;
    if (tid < NMAX) {
      const int i = tid;
      double v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = X[i * S + c0 + j];
      bool done = s_panel[i] >= 0;
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        const int par = jj & 1;
        // pivot key: |a_ik| as a float rounded toward zero, last 8 mantissa
        // bits replaced by 128 - row (first row among equals; never 0 for a
        // row not yet pivoted); pivoted rows 0
        const unsigned key =
            done ? 0u : ((__float_as_uint(__double2float_rz(fabs(v[jj]))) & ~255u) | static_cast<unsigned>(128 - i));
        const unsigned wmax = __reduce_max_sync(0xffffffffu, key);
        if (key == wmax) {  // this warp's winner posts its row (live keys are distinct; a warp
                            // with no live row posts garbage under key 0, which never wins)
          s_key[par][warp] = wmax;
#pragma unroll
          for (int j = 0; j < 16; ++j) s_cand[par][warp][j] = v[j];
        }
        asm volatile("bar.sync 1, %0;" ::"r"(NMAX) : "memory");
        unsigned best = s_key[par][0];
        int bw = 0;
#pragma unroll
        for (int w = 1; w < NMAX / 32; ++w)
          if (s_key[par][w] > best) {
            best = s_key[par][w];
            bw = w;
          }
        const int pr = 128 - static_cast<int>(best & 255u);
        const double *prow = s_cand[par][bw];
        if (i == pr) {
          s_perm[c0 + jj] = i;
          s_panel[i] = p;
          done = true;
        }
        const double d = prow[jj];
        if (tid == 0 && first_zero == 0 && !(fabs(d) >= 2.2250738585072014e-308)) first_zero = c0 + jj + 1;
        const double inv = reciprocal(d);
        if (i == pr) {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = (j == jj) ? inv : v[j] * inv;
        } else {
          const double l = v[jj] * inv;
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = (j == jj) ? -l : fma(-l, prow[j], v[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        X[i * S + c0 + j] = v[j];
        Ws[i * T::kWS + j] = v[j];
      }
    }
    __syncthreads();
    // the panel's pivot rows as they were before the panel
    for (int e = tid; e < 16 * NMAX; e += T::kThreads) {
      const int jj = e / NMAX, c = e % NMAX;
      Rs[jj * S + c] = X[s_perm[c0 + jj] * S + c];
    }
    __syncthreads();
    // every column tile outside the panel: X <- [row not a pivot of this
    // panel] X + W R, on the tensor cores
    {
      constexpr int kRT = NMAX / 16, kCT = NMAX / 8, kStride = 8 / kRT;
      const int g = lane >> 2, t = lane & 3;
      const int rt = warp % kRT;
      const int r0 = 16 * rt + g, r1 = r0 + 8;
      double af[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) af[q] = Ws[(16 * rt + g + 8 * (q & 1)) * T::kWS + t + 4 * (q >> 1)];
      const bool keep0 = s_panel[r0] != p, keep1 = s_panel[r1] != p;
      for (int ct = warp / kRT; ct < kCT; ct += kStride) {
        if ((ct >> 1) == p) continue;  // the panel's own two column tiles
        const int c = 8 * ct;
        double bf[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = Rs[(t + 4 * j) * S + c + g];
        double2 *x0 = reinterpret_cast<double2 *>(X + r0 * S + c + 2 * t);
        double2 *x1 = reinterpret_cast<double2 *>(X + r1 * S + c + 2 * t);
        const double2 o0 = *x0, o1 = *x1;
        double dd[4] = {keep0 ? o0.x : 0.0, keep0 ? o0.y : 0.0, keep1 ? o1.x : 0.0, keep1 ? o1.y : 0.0};
        mma_f64_16816(dd, af, bf);
        *x0 = make_double2(dd[0], dd[1]);
        *x1 = make_double2(dd[2], dd[3]);
      }
    }
    __syncthreads();
  }
  // A^-1 (k, c) = X[perm[k], iperm[c]]: coalesced stores of the block's rows
  for (int k = tid; k < NMAX; k += T::kThreads) s_iperm[s_perm[k]] = k;
  __syncthreads();
  float *M32 = A32 ? A32 + moff[b] : nullptr;
  for (int e = tid; e < n * n; e += T::kThreads) {
    const int k = e / n, c = e % n;
    const double v = X[s_perm[k] * S + s_iperm[c]];
    M[e] = v;
    if (M32) M32[e] = static_cast<float>(v);
  }
  if (tid == 0) info[b] = first_zero;
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
    using T = f3d::TcInv<64>;
    if (cudaFuncSetAttribute(f3d::batched_inverse_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(T::kSmem)) != cudaSuccess)
      return F3D_ERR_CUDA;
    f3d::batched_inverse_tc_kernel<64><<<count, T::kThreads, T::kSmem, st>>>(A, matrix_offsets, sizes, count, A32,
                                                                             info);
  } else {
    using T = f3d::TcInv<128>;
    if (cudaFuncSetAttribute(f3d::batched_inverse_tc_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(T::kSmem)) != cudaSuccess)
      return F3D_ERR_CUDA;
    f3d::batched_inverse_tc_kernel<128><<<count, T::kThreads, T::kSmem, st>>>(A, matrix_offsets, sizes, count,
                                                                              A32, info);
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
