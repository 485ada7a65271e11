// Batched LU factorisation with partial pivoting, and the matching solve,
// for many small dense FP64 systems of uneven size in ONE persistent launch
// each: the per-fiber (4N x 4N) and per-body ((3Nb+6)^2) blocks of the
// block-diagonal preconditioner.
//
// Replaces, per block, scipy.linalg.lu_factor / lu_solve as called by
// build_block_diagonal_lu_preconditioner_fiber (tstep/tstep_utils.py:1405-1419),
// build_block_diagonal_preconditioner_body (tstep_utils.py:1341-1386) and
// P_inv (tstep/tstep.py:950-994).  Pivot convention as LAPACK getrf: at step
// i, row i was swapped with row piv[i] (0-based here), the pivot being the
// first entry of largest magnitude in the column.
//
// Factor: one CTA per matrix, CTAs take matrices from a queue (atomic counter,
// host-supplied order, largest first) until it is empty.  Blocked
// right-looking algorithm with an NB-column panel held in shared memory:
//   1. panel (n-k0) x NB loaded to shared memory (column-major), unblocked
//      LU with pivot search by block argmax reduction;
//   2. panel written back, its row swaps applied to the other columns;
//   3. U12 = L11^-1 A12 (one thread per column, NB unrolled);
//   4. A22 -= L21 U12 in column chunks of 64 staged in shared memory,
//      4x2 register tiles.
// The trailing matrix stays in global memory; it is L2-resident while the CTA
// works on it.
// Solve: one warp per system (persistent over systems), right-hand side in
// shared memory, row-oriented substitution with shuffle reductions.
#include <algorithm>

#include "f3d_common.cuh"

namespace f3d {

constexpr int kLuThreads = 256;
constexpr int kChunk = 64;  // columns of U12 staged per GEMM chunk

struct LuArgs {
  double *A;
  const int64_t *moff;   // matrix offsets (elements)
  const int64_t *voff;   // vector/pivot offsets (elements)
  const int32_t *sizes;
  const int32_t *order;  // processing order or nullptr
  int32_t *piv;
  int32_t *info;
  unsigned *queue;       // [2] work counter, finished-CTA counter (zero on entry and exit)
  int count;
};

template <int NB>
__device__ void lu_factor_one(double *__restrict__ A, int n, int32_t *__restrict__ piv,
                              int32_t *info, double *smem) {
  double *P = smem;                                // panel, column-major, m rows
  double *U = smem + static_cast<size_t>(n) * NB;  // U12 chunk: NB x kChunk (row-major)
  __shared__ int s_piv[NB];
  __shared__ double s_val[kLuThreads / 32];
  __shared__ int s_idx[kLuThreads / 32];
  __shared__ int s_info;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_info = 0;

  for (int k0 = 0; k0 < n; k0 += NB) {
    const int nb = min(NB, n - k0);
    const int m = n - k0;
    for (int idx = tid; idx < m * nb; idx += kLuThreads) {
      const int r = idx / nb, c = idx - r * nb;
      P[c * m + r] = A[static_cast<int64_t>(k0 + r) * n + k0 + c];
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
      // argmax |P[j:m, j]|, first index on ties
      double best = -1.0;
      int bi = m;
      for (int r = j + tid; r < m; r += kLuThreads) {
        const double v = fabs(P[j * m + r]);
        if (v > best) { best = v; bi = r; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
      }
      if (lane == 0) { s_val[warp] = best; s_idx[warp] = bi; }
      __syncthreads();
      if (tid == 0) {
        double bv = s_val[0];
        int bix = s_idx[0];
        for (int w = 1; w < kLuThreads / 32; ++w) {
          if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < bix)) { bv = s_val[w]; bix = s_idx[w]; }
        }
        if (bix >= m) bix = j;
        s_piv[j] = bix;
        if (P[j * m + bix] == 0.0 && s_info == 0) s_info = k0 + j + 1;
      }
      __syncthreads();
      const int p = s_piv[j];
      if (p != j) {
        for (int c = tid; c < nb; c += kLuThreads) {
          const double t = P[c * m + j];
          P[c * m + j] = P[c * m + p];
          P[c * m + p] = t;
        }
      }
      __syncthreads();
      const double pv = P[j * m + j];
      if (pv != 0.0) {
        for (int r = j + 1 + tid; r < m; r += kLuThreads) P[j * m + r] /= pv;
      }
      __syncthreads();
      const int mr = m - j - 1, nc = nb - j - 1;
      for (int idx = tid; idx < mr * nc; idx += kLuThreads) {
        const int c = j + 1 + idx / mr, r = j + 1 + idx % mr;
        P[c * m + r] -= P[j * m + r] * P[c * m + j];
      }
      __syncthreads();
    }
    for (int idx = tid; idx < m * nb; idx += kLuThreads) {
      const int r = idx / nb, c = idx - r * nb;
      A[static_cast<int64_t>(k0 + r) * n + k0 + c] = P[c * m + r];
    }
    if (tid < nb) piv[k0 + tid] = k0 + s_piv[tid];
    // Row swaps on the columns outside the panel.  Thread t owns the same
    // columns for every j, so the swaps stay in order without barriers.
    const int nout = n - nb;
    for (int j = 0; j < nb; ++j) {
      const int p = s_piv[j];
      if (p == j) continue;
      for (int c = tid; c < nout; c += kLuThreads) {
        const int col = c < k0 ? c : c + nb;
        double *a = A + static_cast<int64_t>(k0 + j) * n + col;
        double *b = A + static_cast<int64_t>(k0 + p) * n + col;
        const double t = *a;
        *a = *b;
        *b = t;
      }
    }
    __syncthreads();
    const int n2 = n - k0 - nb;
    if (n2 > 0) {
      // U12 = L11^-1 A12 (unit lower L11 = P[0:nb, 0:nb])
      for (int col = k0 + nb + tid; col < n; col += kLuThreads) {
        double u[NB];
#pragma unroll
        for (int r = 0; r < NB; ++r) u[r] = (r < nb) ? A[static_cast<int64_t>(k0 + r) * n + col] : 0.0;
#pragma unroll
        for (int r = 1; r < NB; ++r) {
#pragma unroll
          for (int q = 0; q < NB; ++q)
            if (q < r && r < nb) u[r] -= P[q * m + r] * u[q];
        }
#pragma unroll
        for (int r = 0; r < NB; ++r)
          if (r < nb) A[static_cast<int64_t>(k0 + r) * n + col] = u[r];
      }
      __syncthreads();
      // A22 -= L21 U12, chunked over columns
      const int m2 = m - nb;
      for (int c0 = 0; c0 < n2; c0 += kChunk) {
        const int cw = min(kChunk, n2 - c0);
        for (int idx = tid; idx < nb * kChunk; idx += kLuThreads) {
          const int l = idx / kChunk, c = idx - l * kChunk;
          U[l * kChunk + c] = (c < cw) ? A[static_cast<int64_t>(k0 + l) * n + k0 + nb + c0 + c] : 0.0;
        }
        __syncthreads();
        // thread tile: 4 rows x 2 columns; 32 column pairs x 8 row groups
        const int cp = tid & 31;        // column pair
        const int rg = tid >> 5;        // row group (warp)
        const int cA = 2 * cp, cB = 2 * cp + 1;
        for (int r0 = 4 * rg; r0 < m2; r0 += 4 * (kLuThreads / 32)) {
          double acc[4][2];
#pragma unroll
          for (int a = 0; a < 4; ++a) { acc[a][0] = 0.0; acc[a][1] = 0.0; }
#pragma unroll 4
          for (int l = 0; l < nb; ++l) {
            const double uA = U[l * kChunk + cA], uB = U[l * kChunk + cB];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
              const int r = r0 + a;
              const double lv = (r < m2) ? P[l * m + nb + r] : 0.0;
              acc[a][0] = fma(lv, uA, acc[a][0]);
              acc[a][1] = fma(lv, uB, acc[a][1]);
            }
          }
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int r = r0 + a;
            if (r < m2) {
              double *row = A + static_cast<int64_t>(k0 + nb + r) * n + k0 + nb + c0;
              if (cA < cw) row[cA] -= acc[a][0];
              if (cB < cw) row[cB] -= acc[a][1];
            }
          }
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  if (tid == 0) *info = s_info;
}

template <int NB>
__global__ void __launch_bounds__(kLuThreads) batched_lu_factor_kernel(const LuArgs a) {
  extern __shared__ __align__(16) double lu_smem[];
  __shared__ int s_item;
  while (true) {
    if (threadIdx.x == 0) s_item = static_cast<int>(atomicAdd(&a.queue[0], 1u));
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= a.count) break;
    const int b = a.order ? a.order[item] : item;
    const int n = a.sizes[b];
    if (n > 0) lu_factor_one<NB>(a.A + a.moff[b], n, a.piv + a.voff[b], a.info + b, lu_smem);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.queue[1], 1u) == gridDim.x - 1) {
      a.queue[0] = 0u;
      a.queue[1] = 0u;
    }
  }
}

struct LuSolveArgs {
  const double *LU;
  const int64_t *moff, *voff;
  const int32_t *sizes;
  const int32_t *order;
  const int32_t *piv;
  double *x;  // right-hand sides in, solutions out (packed by voff)
  unsigned *queue;
  int count;
  int max_n;
};

constexpr int kSolveWarps = 8;

__global__ void __launch_bounds__(kSolveWarps * 32) batched_lu_solve_kernel(const LuSolveArgs a) {
  extern __shared__ __align__(16) double sv_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *y = sv_smem + static_cast<size_t>(warp) * a.max_n;
  while (true) {
    int item = 0;
    if (lane == 0) item = static_cast<int>(atomicAdd(&a.queue[0], 1u));
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= a.count) break;
    const int b = a.order ? a.order[item] : item;
    const int n = a.sizes[b];
    const double *L = a.LU + a.moff[b];
    const int32_t *pv = a.piv + a.voff[b];
    double *x = a.x + a.voff[b];
    for (int i = lane; i < n; i += 32) y[i] = x[i];
    __syncwarp();
    if (lane == 0) {
      for (int i = 0; i < n; ++i) {
        const int p = pv[i];
        if (p != i) { const double t = y[i]; y[i] = y[p]; y[p] = t; }
      }
    }
    __syncwarp();
    for (int i = 1; i < n; ++i) {  // forward, unit lower
      const double *row = L + static_cast<int64_t>(i) * n;
      double s = 0.0;
      for (int j = lane; j < i; j += 32) s = fma(row[j], y[j], s);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) y[i] -= s;
      __syncwarp();
    }
    for (int i = n - 1; i >= 0; --i) {  // backward, upper with diagonal
      const double *row = L + static_cast<int64_t>(i) * n;
      double s = 0.0;
      for (int j = i + 1 + lane; j < n; j += 32) s = fma(row[j], y[j], s);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) y[i] = (y[i] - s) / row[i];
      __syncwarp();
    }
    for (int i = lane; i < n; i += 32) x[i] = y[i];
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.queue[1], 1u) == gridDim.x - 1) {
      a.queue[0] = 0u;
      a.queue[1] = 0u;
    }
  }
}

static int pick_nb(int max_n) {
  if (max_n <= 640) return 32;
  if (max_n <= 1280) return 16;
  if (max_n <= 2560) return 8;
  return 0;
}

static size_t factor_smem(int nb, int max_n) {
  return (static_cast<size_t>(max_n) * nb + static_cast<size_t>(nb) * kChunk) * sizeof(double);
}

// Raises a kernel's dynamic shared-memory limit to the opt-in maximum once
// per device (a host-side attribute, so later launches and stream captures
// need no further runtime calls).
template <typename K>
static int allow_max_smem(K kernel, bool (&done)[64]) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return F3D_ERR_CUDA;
  if (done[dev]) return F3D_OK;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return F3D_ERR_CUDA;
  // the opt-in limit covers static plus dynamic shared memory
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return F3D_ERR_CUDA;
  const int dyn = optin - static_cast<int>(fa.sharedSizeBytes);
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess)
    return F3D_ERR_CUDA;
  done[dev] = true;
  return F3D_OK;
}

template <int NB>
static int launch_factor(const LuArgs &a, int max_n, cudaStream_t st) {
  const size_t smem = factor_smem(NB, max_n);
  auto k = batched_lu_factor_kernel<NB>;
  static bool done[64] = {false};
  if (allow_max_smem(k, done)) return F3D_ERR_CUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kLuThreads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int grid = std::max(1, std::min(a.count, per_sm * sm_count()));
  k<<<grid, kLuThreads, smem, st>>>(a);
  return launch_status();
}

}  // namespace f3d

extern "C" {

int f3d_batched_lu_workspace_bytes(size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  *bytes = 256;  // two queue counters
  return F3D_OK;
}

int f3d_batched_lu_factor_panel(double *A, const int64_t *matrix_offsets,
                                const int64_t *vector_offsets, const int32_t *sizes,
                                const int32_t *order, int32_t count, int32_t max_n, int32_t panel,
                                int32_t *piv, int32_t *info, void *workspace,
                                size_t workspace_bytes, void *stream) {
  if (count < 0 || max_n < 0) return F3D_ERR_SHAPE;
  if (count == 0) return F3D_OK;
  if (!A || !matrix_offsets || !vector_offsets || !sizes || !piv || !info) return F3D_ERR_NULL;
  if (!workspace || workspace_bytes < 256) return F3D_ERR_WORKSPACE;
  if (!f3d::aligned(A, 8)) return F3D_ERR_ALIGN;
  if (panel != 0 && panel != 8 && panel != 16 && panel != 32) return F3D_ERR_ARG;
  const int nb = panel ? panel : f3d::pick_nb(max_n);
  if (nb == 0 || f3d::factor_smem(nb, max_n) > 220 * 1024) return F3D_ERR_TOO_LARGE;
  f3d::LuArgs a{A, matrix_offsets, vector_offsets, sizes, order, piv, info,
                static_cast<unsigned *>(workspace), count};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (nb == 32) return f3d::launch_factor<32>(a, max_n, st);
  if (nb == 16) return f3d::launch_factor<16>(a, max_n, st);
  return f3d::launch_factor<8>(a, max_n, st);
}

int f3d_batched_lu_factor(double *A, const int64_t *matrix_offsets, const int64_t *vector_offsets,
                          const int32_t *sizes, const int32_t *order, int32_t count, int32_t max_n,
                          int32_t *piv, int32_t *info, void *workspace, size_t workspace_bytes,
                          void *stream) {
  return f3d_batched_lu_factor_panel(A, matrix_offsets, vector_offsets, sizes, order, count, max_n, 0,
                                     piv, info, workspace, workspace_bytes, stream);
}

int f3d_batched_lu_solve(const double *LU, const int64_t *matrix_offsets,
                         const int64_t *vector_offsets, const int32_t *sizes, const int32_t *order,
                         int32_t count, int32_t max_n, const int32_t *piv, double *x,
                         void *workspace, size_t workspace_bytes, void *stream) {
  if (count < 0 || max_n < 0) return F3D_ERR_SHAPE;
  if (count == 0) return F3D_OK;
  if (!LU || !matrix_offsets || !vector_offsets || !sizes || !piv || !x) return F3D_ERR_NULL;
  if (!workspace || workspace_bytes < 256) return F3D_ERR_WORKSPACE;
  const size_t smem = static_cast<size_t>(f3d::kSolveWarps) * max_n * sizeof(double);
  if (smem > 200 * 1024) return F3D_ERR_TOO_LARGE;
  auto k = f3d::batched_lu_solve_kernel;
  static bool done[64] = {false};
  if (f3d::allow_max_smem(k, done)) return F3D_ERR_CUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, f3d::kSolveWarps * 32, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int want = (count + f3d::kSolveWarps - 1) / f3d::kSolveWarps;
  const int grid = std::max(1, std::min(want, per_sm * f3d::sm_count()));
  // queue counters live after the factor's two words
  f3d::LuSolveArgs a{LU, matrix_offsets, vector_offsets, sizes, order, piv, x,
                     static_cast<unsigned *>(workspace) + 2, count, max_n};
  k<<<grid, f3d::kSolveWarps * 32, smem, static_cast<cudaStream_t>(stream)>>>(a);
  return f3d::launch_status();
}

}  // extern "C"
