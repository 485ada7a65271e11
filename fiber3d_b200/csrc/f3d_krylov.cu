// Device kernels of the GMRES solver that replaces scipy.sparse.linalg.gmres
// behind bpm_utilities/gmres.py:9-111 (right preconditioning), plus the dense
// matrix-vector product that applies the periphery preconditioner
// (the dense LU solve of tstep/tstep.py:957-958, here an explicit inverse).
//
// Krylov basis V is stored row-major, one basis vector of length n per row.
// The number of basis vectors in use, k, is read from device memory so that
// one captured CUDA graph serves every Arnoldi step.
//
//   multidot:   h[i] = V[i] . w, i < k            (two stages, fixed order)
//   multiaxpy:  w -= sum_{i<k} h[i] V[i]
//   norm/scale: beta = |w|, V[k] = w / beta, H column written to `hcol`
//   gemv:       y = M x for row-major M (FP64 or FP32 storage, FP64 sum)
//   gemv_f16:   the same product from FP16 storage with a power-of-two scale
//               per row and the diagonal blocks kept apart in FP64 (the
//               preconditioner of the mixed-precision inner solves)
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>

#include "f3d_common.cuh"

namespace f3d {

constexpr int kDotThreads = 256;
constexpr int kMaxBasis = 256;  // rows of V handled by one multidot launch

// Stage 1: CTA c sums rows i < k over its column chunk into part[c * kmax + i].
__global__ void __launch_bounds__(kDotThreads) multidot_stage1(const double *__restrict__ V,
                                                               const double *__restrict__ w,
                                                               const int *kptr, int64_t n,
                                                               int64_t ldv, double *part,
                                                               int kmax) {
  const int k = *kptr;
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t j0 = static_cast<int64_t>(blockIdx.x) * chunk;
  const int64_t j1 = min(n, j0 + chunk);
  __shared__ double red[kDotThreads / 32];
  for (int i = 0; i < k; ++i) {
    const double *v = V + static_cast<int64_t>(i) * ldv;
    double s = 0.0;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += kDotThreads) s = fma(v[j], w[j], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < kDotThreads / 32; ++q) t += red[q];
      part[static_cast<int64_t>(blockIdx.x) * kmax + i] = t;
    }
    __syncthreads();
  }
}

// Stage 2: h[i] (+)= sum_c part[c * kmax + i].  One warp per i: lane l sums
// c = l, l + 32, ... in order, then a fixed butterfly; the order is the same
// on every call.
__global__ void multidot_stage2(const double *part, int nparts, const int *kptr, int kmax,
                                double *h, int accumulate) {
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= *kptr) return;
  double s = 0.0;
  for (int c = lane; c < nparts; c += 32) s += part[static_cast<int64_t>(c) * kmax + i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) h[i] = accumulate ? h[i] + s : s;
}

// w[j] -= sum_{i<k} h[i] V[i][j]
__global__ void multiaxpy_kernel(const double *__restrict__ V, const double *__restrict__ h,
                                 const int *kptr, double *w, int64_t n, int64_t ldv) {
  __shared__ double hs[kMaxBasis];
  const int k = *kptr;
  for (int i = threadIdx.x; i < k; i += blockDim.x) hs[i] = h[i];
  __syncthreads();
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = w[j];
    for (int i = 0; i < k; ++i) s = fma(-hs[i], V[static_cast<int64_t>(i) * ldv + j], s);
    w[j] = s;
  }
}

// Combination y[j] = sum_{i<k} c[i] V[i][j] (+ y[j] if accumulate)
__global__ void combine_kernel(const double *__restrict__ V, const double *__restrict__ c,
                               int k, double *y, int64_t n, int64_t ldv, int accumulate) {
  __shared__ double cs[kMaxBasis];
  for (int i = threadIdx.x; i < k; i += blockDim.x) cs[i] = c[i];
  __syncthreads();
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = accumulate ? y[j] : 0.0;
    for (int i = 0; i < k; ++i) s = fma(cs[i], V[static_cast<int64_t>(i) * ldv + j], s);
    y[j] = s;
  }
}

// Stage 1 of a norm: part[c] = sum over chunk of w^2.
__global__ void __launch_bounds__(kDotThreads) sumsq_stage1(const double *__restrict__ w,
                                                            int64_t n, double *part) {
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t j0 = static_cast<int64_t>(blockIdx.x) * chunk;
  const int64_t j1 = min(n, j0 + chunk);
  __shared__ double red[kDotThreads / 32];
  double s = 0.0;
  for (int64_t j = j0 + threadIdx.x; j < j1; j += kDotThreads) s = fma(w[j], w[j], s);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < kDotThreads / 32; ++q) t += red[q];
    part[blockIdx.x] = t;
  }
}

// beta = sqrt(sum part); writes hcol[k] = beta (the subdiagonal entry of the
// Hessenberg column, whose first k entries the caller already holds).
__global__ void norm_stage2(const double *part, int nparts, const int *kptr, double *hcol,
                            double *beta_out) {
  // one warp: lane l sums parts l, l + 32, ... in order, then a fixed butterfly
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int c = lane; c < nparts; c += 32) s += part[c];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane != 0) return;
  const double b = sqrt(s);
  if (hcol) hcol[*kptr] = b;
  if (beta_out) *beta_out = b;
}

// V[k] = w / beta (beta > 0; else zero), also into `also` if non-null.
__global__ void scale_into_kernel(const double *__restrict__ w, const double *beta, int *kptr,
                                  double *V, int64_t n, int64_t ldv, double *also) {
  const int k = *kptr;
  const double b = *beta;
  const double inv = b > 0.0 ? 1.0 / b : 0.0;
  double *dst = V + static_cast<int64_t>(k) * ldv;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = w[j] * inv;
    dst[j] = v;
    if (also) also[j] = v;
  }
}

// dst[(*k + offset) * ld + j] = src[j]
__global__ void store_row_kernel(const double *__restrict__ src, const int *kptr, int offset,
                                 double *dst, int64_t n, int64_t ld) {
  const int row = *kptr + offset;
  if (row < 0) return;
  double *d = dst + static_cast<int64_t>(row) * ld;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x)
    d[j] = src[j];
}

__global__ void bump_kernel(int *kptr) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *kptr += 1;
}

// y = M x, M row-major rows x cols.  Each warp owns kRowsPerWarp rows of a
// group; x is staged through shared memory in chunks shared by the 32 rows of
// the CTA's group, so M streams from HBM once and x mostly from L2.  With
// VEC > 1 each lane loads VEC consecutive elements (16 bytes) per access; the
// caller guarantees 16-byte aligned rows (ld and cols multiples of VEC).
template <typename T, int VEC>
__device__ __forceinline__ void gemv_rows(const T *__restrict__ M, const double *__restrict__ x, double *y,
                                          int64_t rows, int64_t cols, int64_t ld, int64_t bx, int64_t gx) {
  constexpr int kXChunk = 4096;
  constexpr int kRowsPerWarp = 4;
  __shared__ __align__(16) double xs[kXChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const int64_t group = static_cast<int64_t>(warps) * kRowsPerWarp;
  for (int64_t rb = bx * group; rb < rows; rb += gx * group) {
    double acc[kRowsPerWarp];
#pragma unroll
    for (int q = 0; q < kRowsPerWarp; ++q) acc[q] = 0.0;
    const int64_t rw = rb + static_cast<int64_t>(warp) * kRowsPerWarp;
    for (int64_t c0 = 0; c0 < cols; c0 += kXChunk) {
      const int cw = static_cast<int>((cols - c0 < kXChunk) ? (cols - c0) : kXChunk);
      __syncthreads();
      for (int i = threadIdx.x; i < cw; i += blockDim.x) xs[i] = x[c0 + i];
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kRowsPerWarp; ++q) {
        const int64_t r = rw + q;
        if (r < rows) {
          const T *row = M + r * ld + c0;
          double a = acc[q];
          if (VEC == 1) {
#pragma unroll 4
            for (int i = lane; i < cw; i += 32) a = fma(static_cast<double>(row[i]), xs[i], a);
          } else if constexpr (sizeof(T) == 8) {
            const double2 *rv = reinterpret_cast<const double2 *>(row);
            const int nv = cw / 2;
#pragma unroll 2
            for (int i = lane; i < nv; i += 32) {
              const double2 d = rv[i];
              a = fma(d.x, xs[2 * i], a);
              a = fma(d.y, xs[2 * i + 1], a);
            }
          } else {
            const float4 *rv = reinterpret_cast<const float4 *>(row);
            const int nv = cw / 4;
#pragma unroll 2
            for (int i = lane; i < nv; i += 32) {
              const float4 f = rv[i];
              a = fma(static_cast<double>(f.x), xs[4 * i], a);
              a = fma(static_cast<double>(f.y), xs[4 * i + 1], a);
              a = fma(static_cast<double>(f.z), xs[4 * i + 2], a);
              a = fma(static_cast<double>(f.w), xs[4 * i + 3], a);
            }
          }
          acc[q] = a;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kRowsPerWarp; ++q) {
      double a = acc[q];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      if (lane == 0 && rw + q < rows) y[rw + q] = a;
    }
  }
}


template <typename T, int VEC>
__global__ void __launch_bounds__(256) gemv_kernel(const T *__restrict__ M,
                                                   const double *__restrict__ x, double *y,
                                                   int64_t rows, int64_t cols, int64_t ld) {
  gemv_rows<T, VEC>(M, x, y, rows, cols, ld, blockIdx.x, gridDim.x);
}

// count square FP64 matrices in one launch: matrix b (n[b] x n[b], row-major
// at M + m_off[b]) times x + x_off[b] into y + y_off[b]; blockIdx.y = b.
template <int VEC>
__global__ void __launch_bounds__(256) gemv_batched_kernel(const double *__restrict__ M,
                                                           const int64_t *__restrict__ m_off,
                                                           const int64_t *__restrict__ n,
                                                           const int64_t *__restrict__ x_off,
                                                           const int64_t *__restrict__ y_off,
                                                           const double *__restrict__ x, double *y) {
  const int b = blockIdx.y;
  const int64_t nb = n[b];
  gemv_rows<double, VEC>(M + m_off[b], x + x_off[b], y + y_off[b], nb, nb, nb, blockIdx.x, gridDim.x);
}

// Row r of M (cols entries) -> FP16 row of M16 scaled by row_scale[r] = 2^e,
// the smallest power of two >= max |M[r][c]| over the columns outside r's
// diagonal block; the block's entries (columns db*(r/db) .. +db-1) go to
// diag[r*db + c] in FP64 and are zero in M16.  One warp per row.
__global__ void quantize_rows_f16_kernel(const double *__restrict__ M, int64_t ld, int64_t rows,
                                         int64_t cols, int db, __half *__restrict__ M16,
                                         int64_t ld16, float *__restrict__ row_scale,
                                         double *__restrict__ diag) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    const double *row = M + r * ld;
    const int64_t b0 = db > 0 ? (r / db) * db : -1;
    const int64_t b1 = db > 0 ? b0 + db : -1;
    double mx = 0.0;
    for (int64_t c = lane; c < cols; c += 32)
      if (c < b0 || c >= b1) mx = fmax(mx, fabs(row[c]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);  // mx = m 2^e, m in [0.5, 1)
    const double s = ldexp(1.0, e);
    const double inv = 1.0 / s;  // exact: a power of two
    __half *out = M16 + r * ld16;
    for (int64_t c = lane; c < cols; c += 32) {
      const bool in_block = c >= b0 && c < b1;
      out[c] = __double2half(in_block ? 0.0 : row[c] * inv);
      if (in_block) diag[r * db + (c - b0)] = row[c];
    }
    if (lane == 0) row_scale[r] = static_cast<float>(s);
  }
}

// y = diag(row_scale) M16 x + blockdiag(diag) x.  Same row/warp layout as
// gemv_kernel; x chunk staged as FP32, products summed in FP32.
template <int VEC>
__global__ void __launch_bounds__(256) gemv_f16_kernel(const __half *__restrict__ M, int64_t ld,
                                                       const float *__restrict__ row_scale,
                                                       const double *__restrict__ diag, int db,
                                                       const double *__restrict__ x, double *y,
                                                       int64_t rows, int64_t cols) {
  constexpr int kXChunk = 8192;
  constexpr int kRowsPerWarp = 4;
  __shared__ __align__(16) float xs[kXChunk];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const int64_t group = static_cast<int64_t>(warps) * kRowsPerWarp;
  for (int64_t rb = static_cast<int64_t>(blockIdx.x) * group; rb < rows;
       rb += static_cast<int64_t>(gridDim.x) * group) {
    float acc[kRowsPerWarp];
#pragma unroll
    for (int q = 0; q < kRowsPerWarp; ++q) acc[q] = 0.0f;
    const int64_t rw = rb + static_cast<int64_t>(warp) * kRowsPerWarp;
    for (int64_t c0 = 0; c0 < cols; c0 += kXChunk) {
      const int cw = static_cast<int>((cols - c0 < kXChunk) ? (cols - c0) : kXChunk);
      __syncthreads();
      for (int i = threadIdx.x; i < cw; i += blockDim.x) xs[i] = static_cast<float>(x[c0 + i]);
      __syncthreads();
      if (VEC == 1) {
#pragma unroll
        for (int q = 0; q < kRowsPerWarp; ++q) {
          const int64_t r = rw + q;
          if (r < rows) {
            const __half *row = M + r * ld + c0;
            float a = acc[q];
#pragma unroll 4
            for (int i = lane; i < cw; i += 32) a = fmaf(__half2float(row[i]), xs[i], a);
            acc[q] = a;
          }
        }
      } else {
        // the kRowsPerWarp rows advance together: that many independent
        // 16-byte loads in flight per lane per iteration
        const uint4 *rv[kRowsPerWarp];
#pragma unroll
        for (int q = 0; q < kRowsPerWarp; ++q) {
          const int64_t r = rw + q < rows ? rw + q : rows - 1;  // clamped rows are not stored
          rv[q] = reinterpret_cast<const uint4 *>(M + r * ld + c0);
        }
        const int nv = cw / 8;
#pragma unroll 2
        for (int i = lane; i < nv; i += 32) {
          uint4 u[kRowsPerWarp];
#pragma unroll
          for (int q = 0; q < kRowsPerWarp; ++q) u[q] = rv[q][i];
          const float4 xa = *reinterpret_cast<const float4 *>(xs + 8 * i);
          const float4 xb = *reinterpret_cast<const float4 *>(xs + 8 * i + 4);
#pragma unroll
          for (int q = 0; q < kRowsPerWarp; ++q) {
            const float2 f0 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].x));
            const float2 f1 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].y));
            const float2 f2 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].z));
            const float2 f3 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].w));
            float a = acc[q];
            a = fmaf(f0.x, xa.x, a);
            a = fmaf(f0.y, xa.y, a);
            a = fmaf(f1.x, xa.z, a);
            a = fmaf(f1.y, xa.w, a);
            a = fmaf(f2.x, xb.x, a);
            a = fmaf(f2.y, xb.y, a);
            a = fmaf(f3.x, xb.z, a);
            a = fmaf(f3.y, xb.w, a);
            acc[q] = a;
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kRowsPerWarp; ++q) {
      float a = acc[q];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      const int64_t r = rw + q;
      if (lane == 0 && r < rows) {
        double v = static_cast<double>(a) * static_cast<double>(row_scale[r]);
        if (db > 0) {
          const int64_t b0 = (r / db) * db;
          for (int c = 0; c < db && b0 + c < cols; ++c) v = fma(diag[r * db + c], x[b0 + c], v);
        }
        y[r] = v;
      }
    }
  }
}

// gemv_f16_kernel with all of x staged once (FP32, cols <= kGemvF16FullX)
// in a persistent CTA of 1024 threads per SM: no restaging barriers inside
// the row loop, and 32 warps x 4 rows of 16-byte loads (64 KB) in flight per
// SM.  Each lane sums its columns in the same order as
// gemv_f16_kernel<8> (whose x chunks are whole multiples of 32 lanes x 8
// columns), so the two give the same results.
constexpr int64_t kGemvF16FullX = 45056;

__global__ void __launch_bounds__(1024, 1) gemv_f16_fullx_kernel(const __half *__restrict__ M, int64_t ld,
                                                                 const float *__restrict__ row_scale,
                                                                 const double *__restrict__ diag, int db,
                                                                 const double *__restrict__ x, double *y,
                                                                 int64_t rows, int64_t cols) {
  constexpr int kRowsPerWarp = 4;
  extern __shared__ __align__(16) float xs_all[];
  for (int64_t i = threadIdx.x; i < cols; i += blockDim.x) xs_all[i] = static_cast<float>(x[i]);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  const int nv = static_cast<int>(cols / 8);
  for (int64_t grp = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp; grp * kRowsPerWarp < rows;
       grp += nwarps) {
    const int64_t rw = grp * kRowsPerWarp;
    float acc[kRowsPerWarp];
    const uint4 *rv[kRowsPerWarp];
#pragma unroll
    for (int q = 0; q < kRowsPerWarp; ++q) {
      acc[q] = 0.0f;
      const int64_t r = rw + q < rows ? rw + q : rows - 1;  // clamped rows are not stored
      rv[q] = reinterpret_cast<const uint4 *>(M + r * ld);
    }
#pragma unroll 1
    for (int i = lane; i < nv; i += 32) {
      uint4 u[kRowsPerWarp];
#pragma unroll
      for (int q = 0; q < kRowsPerWarp; ++q) u[q] = rv[q][i];
      const float4 xa = *reinterpret_cast<const float4 *>(xs_all + 8 * i);
      const float4 xb = *reinterpret_cast<const float4 *>(xs_all + 8 * i + 4);
#pragma unroll
      for (int q = 0; q < kRowsPerWarp; ++q) {
        const float2 f0 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].x));
        const float2 f1 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].y));
        const float2 f2 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].z));
        const float2 f3 = __half22float2(*reinterpret_cast<const __half2 *>(&u[q].w));
        float a = acc[q];
        a = fmaf(f0.x, xa.x, a);
        a = fmaf(f0.y, xa.y, a);
        a = fmaf(f1.x, xa.z, a);
        a = fmaf(f1.y, xa.w, a);
        a = fmaf(f2.x, xb.x, a);
        a = fmaf(f2.y, xb.y, a);
        a = fmaf(f3.x, xb.z, a);
        a = fmaf(f3.y, xb.w, a);
        acc[q] = a;
      }
    }
#pragma unroll
    for (int q = 0; q < kRowsPerWarp; ++q) {
      float a = acc[q];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      const int64_t r = rw + q;
      if (lane == 0 && r < rows) {
        double v = static_cast<double>(a) * static_cast<double>(row_scale[r]);
        if (db > 0) {
          const int64_t b0 = (r / db) * db;
          for (int c = 0; c < db && b0 + c < cols; ++c) v = fma(diag[r * db + c], x[b0 + c], v);
        }
        y[r] = v;
      }
    }
  }
}

__global__ void cast_to_float_kernel(const double *__restrict__ a, float *b, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    b[i] = static_cast<float>(a[i]);
}

static unsigned grid_for(int64_t n, int threads) {
  const int64_t g = (n + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(sm_count()) * 8;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min(g, cap)));
}

}  // namespace f3d

extern "C" {

int f3d_krylov_workspace_bytes(int64_t n, int32_t kmax, size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  if (n < 0 || kmax < 1 || kmax > f3d::kMaxBasis) return F3D_ERR_SHAPE;
  const int parts = f3d::sm_count() * 2;
  *bytes = f3d::round_up(static_cast<size_t>(parts) * (kmax + 1) * sizeof(double), 256);
  return F3D_OK;
}

int f3d_krylov_multidot(const double *V, int64_t ldv, const double *w, const int32_t *k,
                        int32_t kmax, double *h, int64_t n, int accumulate, void *workspace,
                        size_t workspace_bytes, void *stream) {
  if (!V || !w || !k || !h) return F3D_ERR_NULL;
  if (n <= 0 || kmax < 1 || kmax > f3d::kMaxBasis || ldv < n) return F3D_ERR_SHAPE;
  size_t need = 0;
  f3d_krylov_workspace_bytes(n, kmax, &need);
  if (!workspace || workspace_bytes < need) return F3D_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int parts = std::max(1, std::min<int>(f3d::sm_count() * 2, static_cast<int>((n + 255) / 256)));
  double *part = static_cast<double *>(workspace);
  f3d::multidot_stage1<<<parts, f3d::kDotThreads, 0, st>>>(V, w, k, n, ldv, part, kmax);
  int rc = f3d::launch_status();
  if (rc) return rc;
  f3d::multidot_stage2<<<(kmax + 7) / 8, 256, 0, st>>>(part, parts, k, kmax, h, accumulate);
  return f3d::launch_status();
}

int f3d_krylov_multiaxpy(const double *V, int64_t ldv, const double *h, const int32_t *k,
                         double *w, int64_t n, void *stream) {
  if (!V || !w || !k || !h) return F3D_ERR_NULL;
  if (n <= 0 || ldv < n) return F3D_ERR_SHAPE;
  f3d::multiaxpy_kernel<<<f3d::grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      V, h, k, w, n, ldv);
  return f3d::launch_status();
}

int f3d_krylov_combine(const double *V, int64_t ldv, const double *c, int32_t k, double *y,
                       int64_t n, int accumulate, void *stream) {
  if (!V || !c || !y) return F3D_ERR_NULL;
  if (n <= 0 || ldv < n || k < 0 || k > f3d::kMaxBasis) return F3D_ERR_SHAPE;
  f3d::combine_kernel<<<f3d::grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      V, c, k, y, n, ldv, accumulate);
  return f3d::launch_status();
}

int f3d_krylov_norm(const double *w, int64_t n, const int32_t *k, double *hcol, double *beta,
                    void *workspace, size_t workspace_bytes, void *stream) {
  if (!w) return F3D_ERR_NULL;
  if (n <= 0) return F3D_ERR_SHAPE;
  if (!workspace || workspace_bytes < 256 * sizeof(double)) return F3D_ERR_WORKSPACE;
  if (hcol && !k) return F3D_ERR_NULL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int parts = std::max(1, std::min<int>(256, static_cast<int>((n + 1023) / 1024)));
  double *part = static_cast<double *>(workspace);
  f3d::sumsq_stage1<<<parts, f3d::kDotThreads, 0, st>>>(w, n, part);
  int rc = f3d::launch_status();
  if (rc) return rc;
  f3d::norm_stage2<<<1, 32, 0, st>>>(part, parts, k, hcol, beta);
  return f3d::launch_status();
}

int f3d_krylov_scale_into(const double *w, const double *beta, int32_t *k, double *V,
                          int64_t ldv, int64_t n, int bump, double *also, void *stream) {
  if (!w || !beta || !k || !V) return F3D_ERR_NULL;
  if (n <= 0 || ldv < n) return F3D_ERR_SHAPE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  f3d::scale_into_kernel<<<f3d::grid_for(n, 256), 256, 0, st>>>(w, beta, k, V, n, ldv, also);
  int rc = f3d::launch_status();
  if (rc || !bump) return rc;
  f3d::bump_kernel<<<1, 32, 0, st>>>(k);
  return f3d::launch_status();
}

int f3d_krylov_store(const double *src, const int32_t *k, int32_t offset, double *dst,
                     int64_t ld, int64_t n, void *stream) {
  if (!src || !k || !dst) return F3D_ERR_NULL;
  if (n <= 0 || ld < n) return F3D_ERR_SHAPE;
  f3d::store_row_kernel<<<f3d::grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      src, k, offset, dst, n, ld);
  return f3d::launch_status();
}

int f3d_gemv_batched(const double *M, const int64_t *m_off, const int64_t *n, const int64_t *x_off,
                     const int64_t *y_off, int32_t count, int64_t max_n, int vec, const double *x, double *y,
                     void *stream) {
  if (count < 0 || max_n < 0) return F3D_ERR_SHAPE;
  if (count == 0 || max_n == 0) return F3D_OK;
  if (!M || !m_off || !n || !x_off || !y_off || !x || !y) return F3D_ERR_NULL;
  if (vec && reinterpret_cast<uintptr_t>(M) % 16 != 0) return F3D_ERR_ALIGN;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t per = std::max<int64_t>(1, std::min<int64_t>((max_n + 31) / 32,
                                                             (static_cast<int64_t>(f3d::sm_count()) * 4 + count - 1) / count));
  const dim3 grid(static_cast<unsigned>(per), static_cast<unsigned>(count));
  if (vec)
    f3d::gemv_batched_kernel<2><<<grid, 256, 0, st>>>(M, m_off, n, x_off, y_off, x, y);
  else
    f3d::gemv_batched_kernel<1><<<grid, 256, 0, st>>>(M, m_off, n, x_off, y_off, x, y);
  return f3d::launch_status();
}

int f3d_gemv(int precision, const void *M, int64_t ld, const double *x, double *y, int64_t rows,
             int64_t cols, void *stream) {
  if (!M || !x || !y) return F3D_ERR_NULL;
  if (rows < 0 || cols < 0 || ld < cols) return F3D_ERR_SHAPE;
  if (rows == 0) return F3D_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(
      1, std::min<int64_t>((rows + 31) / 32, static_cast<int64_t>(f3d::sm_count()) * 4)));
  // 16-byte vector loads when every row starts 16-byte aligned and the x
  // chunks (4096 elements) split into whole vectors.
  const uintptr_t base = reinterpret_cast<uintptr_t>(M);
  if (precision == F3D_FP64) {
    const bool vec = (base % 16 == 0) && (ld % 2 == 0) && (cols % 2 == 0);
    if (vec)
      f3d::gemv_kernel<double, 2><<<grid, 256, 0, st>>>(static_cast<const double *>(M), x, y, rows, cols, ld);
    else
      f3d::gemv_kernel<double, 1><<<grid, 256, 0, st>>>(static_cast<const double *>(M), x, y, rows, cols, ld);
  } else if (precision == F3D_FP32C) {
    const bool vec = (base % 16 == 0) && (ld % 4 == 0) && (cols % 4 == 0);
    if (vec)
      f3d::gemv_kernel<float, 4><<<grid, 256, 0, st>>>(static_cast<const float *>(M), x, y, rows, cols, ld);
    else
      f3d::gemv_kernel<float, 1><<<grid, 256, 0, st>>>(static_cast<const float *>(M), x, y, rows, cols, ld);
  } else {
    return F3D_ERR_ARG;
  }
  return f3d::launch_status();
}

int f3d_quantize_rows_f16(const double *M, int64_t ld, int64_t rows, int64_t cols,
                          int32_t diag_block, void *M16, int64_t ld16, float *row_scale,
                          double *diag, void *stream) {
  if (!M || !M16 || !row_scale) return F3D_ERR_NULL;
  if (rows < 0 || cols < 0 || ld < cols || ld16 < cols || diag_block < 0) return F3D_ERR_SHAPE;
  if (diag_block > 0 && (!diag || rows != cols || rows % diag_block != 0)) return F3D_ERR_ARG;
  if (rows == 0) return F3D_OK;
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(
      1, std::min<int64_t>((rows + 7) / 8, static_cast<int64_t>(f3d::sm_count()) * 8)));
  f3d::quantize_rows_f16_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      M, ld, rows, cols, diag_block, static_cast<__half *>(M16), ld16, row_scale, diag);
  return f3d::launch_status();
}

int f3d_gemv_f16(const void *M16, int64_t ld16, const float *row_scale, const double *diag,
                 int32_t diag_block, const double *x, double *y, int64_t rows, int64_t cols,
                 void *stream) {
  if (!M16 || !row_scale || !x || !y) return F3D_ERR_NULL;
  if (rows < 0 || cols < 0 || ld16 < cols || diag_block < 0) return F3D_ERR_SHAPE;
  if (diag_block > 0 && !diag) return F3D_ERR_NULL;
  if (rows == 0) return F3D_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(
      1, std::min<int64_t>((rows + 31) / 32, static_cast<int64_t>(f3d::sm_count()) * 4)));
  const uintptr_t base = reinterpret_cast<uintptr_t>(M16);
  const bool vec = (base % 16 == 0) && (ld16 % 8 == 0) && (cols % 8 == 0);
  const __half *M = static_cast<const __half *>(M16);
  if (vec && cols <= f3d::kGemvF16FullX) {
    static bool attr_set[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return F3D_ERR_CUDA;
    const size_t smem = static_cast<size_t>(cols) * sizeof(float);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
      if (cudaFuncSetAttribute(f3d::gemv_f16_fullx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(f3d::kGemvF16FullX * sizeof(float))) != cudaSuccess)
        return F3D_ERR_CUDA;
      if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    f3d::gemv_f16_fullx_kernel<<<static_cast<unsigned>(f3d::sm_count()), 1024, smem, st>>>(
        M, ld16, row_scale, diag, diag_block, x, y, rows, cols);
  } else if (vec)
    f3d::gemv_f16_kernel<8><<<grid, 256, 0, st>>>(M, ld16, row_scale, diag, diag_block, x, y, rows, cols);
  else
    f3d::gemv_f16_kernel<1><<<grid, 256, 0, st>>>(M, ld16, row_scale, diag, diag_block, x, y, rows, cols);
  return f3d::launch_status();
}

int f3d_cast_to_float(const double *a, float *b, int64_t n, void *stream) {
  if (!a || !b) return F3D_ERR_NULL;
  if (n < 0) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  f3d::cast_to_float_kernel<<<f3d::grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      a, b, n);
  return f3d::launch_status();
}

}  // extern "C"
