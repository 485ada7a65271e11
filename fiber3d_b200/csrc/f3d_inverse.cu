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
// One CTA per block holds the whole NMAX x NMAX matrix in registers.  Lane l
// of warp w owns rows l, l+32, .. (R = NMAX/32 of them) of columns 8w ..
// 8w+7, so a column lives in one warp and a row is spread over all warps;
// rows interleaved across lanes keep every shared-memory access of a column
// conflict-free.  That makes
// the pivot step cheap for everyone but one warp:
//   * the warp that owns column k+1 updates its tile for step k, then finds
//     pivot k+1 on its own (two warp reductions, no shared memory), computes
//     the reciprocal, and publishes column k+1, p and 1/a_pk to shared
//     memory (double buffered);
//   * one CTA barrier per step; after it every warp swaps rows k and p of its
//     own columns through a small per-warp buffer (one lane writes each row,
//     __syncwarp, all read) and applies the rank-1 sweep to its tile.
// Blocks smaller than NMAX are padded with the identity, which the sweeps
// leave untouched.
#include <algorithm>
#include <type_traits>

#include "f3d_common.cuh"

namespace f3d {

constexpr int kInvCPW = 8;  // columns per warp

template <int NMAX>
struct InvShape {
  static constexpr int kRPL = NMAX / 32;        // rows per lane
  static constexpr int kWarps = NMAX / kInvCPW;  // 4, 8, 16
  static constexpr int kThreads = 32 * kWarps;   // 128, 256, 512
};

template <int NMAX>
struct InvSmem {
  double col[2][NMAX];                           // published pivot column, by step parity
  double pinv[2];
  int piv[2];
  int zero[2];
  double rk[InvShape<NMAX>::kWarps][kInvCPW];    // per warp: old row k of its columns
  double rp[InvShape<NMAX>::kWarps][kInvCPW];    // per warp: old row p
  int pivots[NMAX];
  int dest[NMAX];
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

// Calls f(integral_constant<int, slot>) for a slot (< R) that is the same in
// every lane of the warp: a uniform branch to a body whose register index is
// a compile-time constant (no per-element selects, no local memory).
template <int R, typename F>
__device__ __forceinline__ void on_slot(int slot, F &&f) {
  if (slot == 0) f(std::integral_constant<int, 0>{});
  if constexpr (R > 1) {
    if (slot == 1) f(std::integral_constant<int, 1>{});
  }
  if constexpr (R > 2) {
    if (slot == 2) f(std::integral_constant<int, 2>{});
    if (slot == 3) f(std::integral_constant<int, 3>{});
  }
}

// Pivot search on column slot JJ of the owner warp for step k, and publication
// of that column, the pivot row index and the pivot's reciprocal (buffer par).
// The pivot is the first row p in [k, n) whose magnitude has the largest
// leading 32 bits (sign, exponent, 20 mantissa bits): a pivot within a factor
// 1 - 2^-20 of the column maximum -- threshold partial pivoting, as stable as
// the exact maximum.
template <int NMAX, int JJ>
__device__ __forceinline__ void inv_search_publish(const double (&a)[InvShape<NMAX>::kRPL][kInvCPW], int k,
                                                   int n, int lane, InvSmem<NMAX> &sm, int par) {
  constexpr int R = InvShape<NMAX>::kRPL;
  unsigned key = 0u, row = 0xFFFFFFFFu;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = i * 32 + lane;
    if (r >= k && r < n) {
      const unsigned kq = static_cast<unsigned>(
          static_cast<unsigned long long>(__double_as_longlong(fabs(a[i][JJ]))) >> 32);
      if (row == 0xFFFFFFFFu || kq > key) { key = kq; row = static_cast<unsigned>(r); }
    }
  }
  const unsigned kmax = __reduce_max_sync(0xffffffffu, row != 0xFFFFFFFFu ? key : 0u);
  const unsigned pmin = __reduce_min_sync(0xffffffffu, (row != 0xFFFFFFFFu && key == kmax) ? row : 0xFFFFFFFFu);
  const int p = pmin < static_cast<unsigned>(n) ? static_cast<int>(pmin) : k;
#pragma unroll
  for (int i = 0; i < R; ++i) sm.col[par][i * 32 + lane] = a[i][JJ];
  __syncwarp();
  if (lane == 0) {
    const double pv = sm.col[par][p];
    const bool zero = !(fabs(pv) >= 2.2250738585072014e-308);  // zero, subnormal or NaN
    sm.piv[par] = p;
    sm.zero[par] = zero ? 1 : 0;
    sm.pinv[par] = zero ? 0.0 : reciprocal(pv);
  }
}

// Step k = kb + M (M < 8, so the owner's column slot M is a compile-time
// register index).  Ends with the step's one CTA barrier.
template <int NMAX, int M>
__device__ __forceinline__ void inverse_step(double (&a)[InvShape<NMAX>::kRPL][kInvCPW], int kb, int n,
                                             int lane, int warp, int tid, InvSmem<NMAX> &sm,
                                             int &first_zero) {
  constexpr int R = InvShape<NMAX>::kRPL;
  const int k = kb + M;
  if (k >= n) return;  // uniform across the CTA
  const int par = k & 1;
  const int p = sm.piv[par];
  const double pinv = sm.pinv[par];
  if (tid == 0) {
    sm.pivots[k] = p;
    if (sm.zero[par] && first_zero == 0) first_zero = k + 1;
  }
  const bool own = (warp == kb / kInvCPW);
  // the owner's column k is now in sm.col: zero it in the tile, so that the
  // one update below also produces the new column k
  if (own) {
#pragma unroll
    for (int i = 0; i < R; ++i) a[i][M] = 0.0;
  }
  // rows k and p of this warp's columns, through the per-warp buffer (the
  // tile slot of a row, row / 32, is the same in every lane)
  on_slot<R>(k / 32, [&](auto q) {
    if (lane == k % 32) {
#pragma unroll
      for (int j = 0; j < kInvCPW; ++j) sm.rk[warp][j] = a[decltype(q)::value][j];
    }
  });
  on_slot<R>(p / 32, [&](auto q) {
    if (lane == p % 32) {
#pragma unroll
      for (int j = 0; j < kInvCPW; ++j) sm.rp[warp][j] = a[decltype(q)::value][j];
    }
  });
  __syncwarp();
  // One FMA per element on every row: a_ij <- a_ij - (a_ik / a_pk) u_j with
  // u = old row p (u_k = 1 in the owner's column k).  On row k this gives
  // old row k - (a_kk / a_pk) u, which is exactly the new row p; on row p it
  // gives nothing useful.  The two lanes holding rows k and p then put the
  // right values in place: row k <- u / a_pk, row p <- old row k - (a_kk /
  // a_pk) u.  (With p == k only the first.)  No per-element selects.
  double u[kInvCPW];
#pragma unroll
  for (int j = 0; j < kInvCPW; ++j) u[j] = sm.rp[warp][j];
  if (own) u[M] = 1.0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const double f = sm.col[par][i * 32 + lane] * pinv;
#pragma unroll
    for (int j = 0; j < kInvCPW; ++j) a[i][j] = fma(-f, u[j], a[i][j]);
  }
  on_slot<R>(k / 32, [&](auto q) {
    if (lane == k % 32) {
#pragma unroll
      for (int j = 0; j < kInvCPW; ++j) a[decltype(q)::value][j] = u[j] * pinv;
    }
  });
  if (p != k) {
    const double fk = sm.col[par][k] * pinv;
    on_slot<R>(p / 32, [&](auto q) {
      if (lane == p % 32) {
#pragma unroll
        for (int j = 0; j < kInvCPW; ++j) a[decltype(q)::value][j] = fma(-fk, u[j], sm.rk[warp][j]);
      }
    });
  }
  // the owner of column k + 1 finds the next pivot while the others finish
  const int k1 = k + 1;
  if (k1 < n && warp == k1 / kInvCPW) inv_search_publish<NMAX, (M + 1) % kInvCPW>(a, k1, n, lane, sm, par ^ 1);
  __syncthreads();
}

template <int NMAX>
__global__ void __launch_bounds__(InvShape<NMAX>::kThreads, 1)
    batched_inverse_kernel(double *__restrict__ A, const int64_t *__restrict__ moff,
                           const int32_t *__restrict__ sizes, int count, float *__restrict__ A32,
                           int32_t *__restrict__ info) {
  using S = InvShape<NMAX>;
  constexpr int R = S::kRPL;
  __shared__ __align__(16) InvSmem<NMAX> sm;
  const int b = blockIdx.x;
  if (b >= count) return;
  const int n = sizes[b];
  if (n <= 0 || n > NMAX) return;
  double *Mb = A + moff[b];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int c0 = warp * kInvCPW;

  double a[R][kInvCPW];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = i * 32 + lane;
#pragma unroll
    for (int j = 0; j < kInvCPW; ++j) {
      const int c = c0 + j;
      a[i][j] = (r < n && c < n) ? Mb[static_cast<int64_t>(r) * n + c] : (r == c ? 1.0 : 0.0);
    }
  }
  int first_zero = 0;
  if (warp == 0) inv_search_publish<NMAX, 0>(a, 0, n, lane, sm, 0);
  __syncthreads();
  // steps in groups of 8, so that the owner's column slot is a compile-time
  // index inside a step; steps past n return at once
  for (int kb = 0; kb < n; kb += kInvCPW) {
    inverse_step<NMAX, 0>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 1>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 2>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 3>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 4>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 5>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 6>(a, kb, n, lane, warp, tid, sm, first_zero);
    inverse_step<NMAX, 7>(a, kb, n, lane, warp, tid, sm, first_zero);
  }
  // column unscramble: X P, swaps (k, p_k) for k = n-1 .. 0
  __syncthreads();
  if (tid == 0) {
    for (int j = 0; j < n; ++j) sm.dest[j] = j;  // dest[j] = source column of final column j
    for (int k = n - 1; k >= 0; --k) {
      const int p = sm.pivots[k];
      const int t = sm.dest[k];
      sm.dest[k] = sm.dest[p];
      sm.dest[p] = t;
    }
    // invert: final position of source column c
    for (int j = 0; j < n; ++j) sm.pivots[sm.dest[j]] = j;
    info[b] = first_zero;
  }
  __syncthreads();
  float *M32 = A32 ? A32 + moff[b] : nullptr;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int r = i * 32 + lane;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < kInvCPW; ++j) {
      const int c = c0 + j;
      if (c >= n) continue;
      const int64_t o = static_cast<int64_t>(r) * n + sm.pivots[c];
      Mb[o] = a[i][j];
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
