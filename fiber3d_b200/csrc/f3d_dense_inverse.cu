// Explicit inverse of a dense FP64 matrix: the periphery operator's inverse
// that the shell preconditioner applies (fiber3d factors the dense shell
// matrix once with scipy.linalg.lu_factor, tstep/tstep.py:327-348, and
// applies lu_solve per GMRES iteration, tstep.py:950-994; here the inverse is
// formed once and applied as a GEMV), and the rigid-body blocks
// (tstep/tstep_utils.py:1341-1386).
//
// Blocked in-place Gauss-Jordan elimination ("sweep" of one 128-row block per
// step).  With b the step's block of rows/columns and r the rest, a step
// replaces
//   A_bb <- Q = A_bb^-1,   A_rb <- -A_rb Q,   A_br <- Q A_br,
//   A_rr <- A_rr - A_rb Q A_br;
// after the last step the array holds A^-1 (2 n^3 flops, as LU + inversion).
// In terms of the panel W = [-A_rb Q; Q] (the new column block) and R = A_b.
// (the old block row): every column J outside b becomes
//   A_.J <- [rows outside b] A_.J + W R_.J
// one FP64 GEMM of rank 128.  Pivoting is local: Q comes from the batched
// Gauss-Jordan inverse with partial pivoting inside the 128 x 128 block
// (f3d_batched_inverse), there is no row exchange across blocks.  Block
// elimination without global pivoting is stable for the operators this
// library inverts (second-kind boundary integral operators, whose diagonal
// blocks carry the 1/w-scaled identity): on spheres of 1000 and 2000 nodes
// the result agrees with an LU-with-partial-pivoting inverse to 3e-14 and
// entries grow by at most 1.06 during elimination.  A zero pivot inside a
// block is reported (F3D_ERR_SINGULAR).
//
// Per step: the pivot block is copied out and inverted (one CTA), the old
// block row is copied to R, gj_panel_kernel forms W in place in the panel
// columns (one CTA per 128-row tile, 8 x 8 FP64 FMA accumulators per
// thread), and gj_update_kernel updates every other 128 x 128 tile on the
// FP64 tensor cores: one persistent CTA per SM (8 warps of 64 x 32 outputs,
// mma.sync m16n8k16) walks its tiles with one continuous stream of operand
// chunks (32 k, cp.async, a three-stage ring, one barrier per chunk) across
// tile boundaries; a tile's old values are prefetched into L2 when its first
// chunk is requested and added in its epilogue.
#include <algorithm>
#include <vector>

#include "f3d_common.cuh"

namespace f3d {
namespace {

constexpr int kGjB = 128;             // rows/columns of a step and of a tile
constexpr int kGjKC = 16;             // k per staged chunk
constexpr int kGjChunks = kGjB / kGjKC;
constexpr int kGjThreads = 256;       // 16 x 16 threads, 8 x 8 outputs each
constexpr int kGjAStride = kGjKC + 2; // padded row of the m-major operand chunk (144 B)
constexpr int kGjABuf = kGjB * kGjAStride;
constexpr int kGjBBuf = kGjKC * kGjB;
constexpr size_t kGjSmemPanel = (2 * kGjABuf + 2 * kGjBBuf) * sizeof(double);
// update: 256 threads, 8 warps of 64 x 32 outputs on the FP64 tensor cores
// (mma.sync m16n8k16), operands in a three-stage ring of 32-k chunks.
// Shared row strides (doubles) chosen so that every fragment read is two
// conflict-free wavefronts: W chunk [128][36] (row-major A fragments: 4g + t
// distinct mod 16 over a half-warp), R chunk [32][132] (k-major B
// fragments: 4t + g).
constexpr int kGuThreads = 256;
constexpr int kGuKC = 32, kGuChunks = kGjB / kGuKC, kGuStages = 3;
constexpr int kGuAS = 36, kGuBS = 132;
constexpr int kGuABuf = kGjB * kGuAS, kGuBBuf = kGuKC * kGuBS;
constexpr size_t kGjSmemUpdate =
    static_cast<size_t>(kGuStages) * (static_cast<size_t>(kGuABuf) + kGuBBuf) * sizeof(double);

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

struct GjArgs {
  double *A;        // np x np (leading dimension ld), np a multiple of 128
  const double *R;  // 128 x ld: the step's block row before the step
  const double *Q;  // 128 x 128: inverse of the step's pivot block
  int64_t ld;
  int s;            // step: pivot block index
  int *err;         // the device error word (read by the host after the last step)
};

// Thread (tx, ty) owns rows 2ty + 32q + e and columns 2tx + 32q + e
// (q < 4, e < 2) of its tile: pairs of adjacent columns for 16-byte accesses,
// the pairs of a warp contiguous (conflict-free shared-memory reads).

// Chunk c of a tile's operands into buffer `buf`: A(row0 + m, k0 + 16c + kk)
// (the step's panel columns) and B(16c + kk, n) = bsrc[(16c + kk) * bld + n].
__device__ __forceinline__ void gj_load_chunk(double *As, double *Bs, const double *A, int64_t ld, int64_t row0,
                                              int64_t k0, const double *bsrc, int64_t bld, int c, int buf, int tid) {
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int seg = tid + u * kGjThreads;  // 128 rows x 8 segments of 16 B
    const int m = seg >> 3, q = seg & 7;
    cp_async16(As + buf * kGjABuf + m * kGjAStride + 2 * q, A + (row0 + m) * ld + k0 + c * kGjKC + 2 * q);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int seg = tid + u * kGjThreads;  // 16 rows x 64 segments of 16 B
    const int kk = seg >> 6, q = seg & 63;
    cp_async16(Bs + buf * kGjBBuf + kk * kGjB + 2 * q, bsrc + static_cast<int64_t>(c * kGjKC + kk) * bld + 2 * q);
  }
  cp_async_commit();
}

// acc += A-chunk x B-chunk (16 k) from shared memory.
__device__ __forceinline__ void gj_mma_chunk(double (&acc)[8][8], const double *as, const double *bs, int tx,
                                             int ty) {
#pragma unroll
  for (int kk = 0; kk < kGjKC; ++kk) {
    double av[8], bv[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = 2 * ty + 32 * q;
      av[2 * q] = as[r * kGjAStride + kk];
      av[2 * q + 1] = as[(r + 1) * kGjAStride + kk];
      const double2 b2 = *reinterpret_cast<const double2 *>(bs + kk * kGjB + 2 * tx + 32 * q);
      bv[2 * q] = b2.x;
      bv[2 * q + 1] = b2.y;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
  }
}

// The panel: W_I = -A(I, b) Q for row tiles I != s, W_s = Q, written in
// place into the panel columns (one CTA per row tile).
__global__ void __launch_bounds__(kGjThreads, 1) gj_panel_kernel(const GjArgs a) {
  extern __shared__ __align__(16) unsigned char gj_smem[];
  double *As = reinterpret_cast<double *>(gj_smem);  // [2][128][kGjAStride]: A[row][k]
  double *Bs = As + 2 * kGjABuf;                      // [2][16][128]: Q[k][col]
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int I = blockIdx.x;
  const int64_t row0 = static_cast<int64_t>(I) * kGjB, k0 = static_cast<int64_t>(a.s) * kGjB;
  if (I == a.s) {
    for (int i = tid; i < kGjB * kGjB / 2; i += kGjThreads) {
      const int r = i / (kGjB / 2), c2 = i % (kGjB / 2);
      reinterpret_cast<double2 *>(a.A + (row0 + r) * a.ld + k0)[c2] =
          reinterpret_cast<const double2 *>(a.Q + r * kGjB)[c2];
    }
    return;
  }
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  gj_load_chunk(As, Bs, a.A, a.ld, row0, k0, a.Q, kGjB, 0, 0, tid);
  for (int c = 0; c < kGjChunks; ++c) {
    cp_async_wait<0>();
    __syncthreads();
    if (c + 1 < kGjChunks) gj_load_chunk(As, Bs, a.A, a.ld, row0, k0, a.Q, kGjB, c + 1, (c + 1) & 1, tid);
    gj_mma_chunk(acc, As + (c & 1) * kGjABuf, Bs + (c & 1) * kGjBBuf, tx, ty);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = 2 * ty + 32 * (i >> 1) + (i & 1);
    double *o = a.A + (row0 + r) * a.ld + k0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      *reinterpret_cast<double2 *>(o + 2 * tx + 32 * q) = make_double2(-acc[i][2 * q], -acc[i][2 * q + 1]);
  }
}

// The update of every tile outside the panel columns, persistent: CTA x
// takes tiles x, x + gridDim.x, ... (row-major over (I, J), J skipping the
// panel), its chunks one continuous stream through a three-stage ring
// across tile boundaries (one barrier per chunk: wait for chunk g, barrier,
// issue chunk g + 2 into the stage chunk g - 1 used, compute chunk g).
// Warp w computes rows 64 (w / 4) .. + 63 and columns 32 (w % 4) .. + 31 of
// the tile as 4 x 4 tensor-core tiles of 16 x 8.  A tile's old values are
// prefetched into L2 (bulk prefetch, no shared memory) when its first chunk
// is requested, and read from there in its epilogue.
__global__ void __launch_bounds__(kGuThreads, 1) gj_update_kernel(const GjArgs a, int tiles) {
  extern __shared__ __align__(16) unsigned char gj_smem[];
  double *As = reinterpret_cast<double *>(gj_smem);  // [3][128][kGuAS]: W[row][k]
  double *Bs = As + kGuStages * kGuABuf;              // [3][32][kGuBS]: R[k][col]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = 64 * (warp >> 2), wc = 32 * (warp & 3);
  const int ncol = tiles - 1;
  const int64_t ntile = static_cast<int64_t>(ncol) * tiles;
  const int64_t first = blockIdx.x;
  if (first >= ntile) return;
  const int mine = static_cast<int>((ntile - first + gridDim.x - 1) / gridDim.x);
  const int total = mine * kGuChunks;
  const int64_t k0 = static_cast<int64_t>(a.s) * kGjB;
  auto tile_rc = [&](int it, int64_t &row0, int64_t &col0) {
    const int64_t tt = first + static_cast<int64_t>(it) * gridDim.x;
    const int I = static_cast<int>(tt / ncol), jx = static_cast<int>(tt % ncol);
    row0 = static_cast<int64_t>(I) * kGjB;
    col0 = static_cast<int64_t>(jx < a.s ? jx : jx + 1) * kGjB;
  };
  // chunk gc's copies in four parts of 2 + 2 per thread (part p: W
  // segments u = 2p, 2p + 1 and R segments likewise), so that a chunk's
  // requests are spread over the compute of the chunk two before it instead
  // of queueing at the load/store unit all at once; the last part commits
  auto load_part = [&](int gc, int part) {
    if (gc < total) {
      int64_t row0, col0;
      tile_rc(gc / kGuChunks, row0, col0);
      const int c = gc % kGuChunks, stage = gc % kGuStages;
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int seg = tid + (2 * part + v) * kGuThreads;  // W: 128 rows x 16 segments of 16 B
        const int m = seg >> 4, q = seg & 15;
        cp_async16(As + stage * kGuABuf + m * kGuAS + 2 * q, a.A + (row0 + m) * a.ld + k0 + c * kGuKC + 2 * q);
      }
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int seg = tid + (2 * part + v) * kGuThreads;  // R: 32 rows x 64 segments of 16 B
        const int kk = seg >> 6, q = seg & 63;
        cp_async16(Bs + stage * kGuBBuf + kk * kGuBS + 2 * q,
                   a.R + static_cast<int64_t>(c * kGuKC + kk) * a.ld + col0 + 2 * q);
      }
      // the tile's old values (none for the pivot block's rows, which become
      // Q R) on their way into L2
      if (part == 0 && c == 0 && row0 != k0 && tid < kGjB) {
        const double *src = a.A + (row0 + tid) * a.ld + col0;
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(static_cast<unsigned>(kGjB * sizeof(double)))
                     : "memory");
      }
    }
    if (part == 3) cp_async_commit();  // an empty group past the end keeps the count uniform
  };
  auto load = [&](int gc) {
#pragma unroll
    for (int part = 0; part < 4; ++part) load_part(gc, part);
  };

  load(0);
  load(1);
  double acc[4][4][4];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[mi][ni][i] = 0.0;
  for (int gc = 0; gc < total; ++gc) {
    cp_async_wait<1>();
    __syncthreads();
    const int stage = gc % kGuStages;
#pragma unroll
    for (int ks = 0; ks < kGuKC / 16; ++ks) {
      const double *as = As + stage * kGuABuf + (wr + g) * kGuAS + 16 * ks + t;
      const double *bs = Bs + stage * kGuBBuf + (16 * ks + t) * kGuBS + wc + g;
      double bf[4][4];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[ni][j] = bs[4 * j * kGuBS + 8 * ni];
      // A fragments double-buffered: those of row block mi + 1 are read while
      // the tensor-core steps of row block mi issue
      double af[2][8];
#pragma unroll
      for (int i = 0; i < 8; ++i) af[0][i] = as[8 * (i & 1) * kGuAS + 4 * (i >> 1)];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        if (mi + 1 < 4) {
#pragma unroll
          for (int i = 0; i < 8; ++i)
            af[(mi + 1) & 1][i] = as[(16 * (mi + 1) + 8 * (i & 1)) * kGuAS + 4 * (i >> 1)];
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_f64_16816(acc[mi][ni], af[mi & 1], bf[ni]);
        // chunk gc + 2 into the stage chunk gc - 1 used (free since the barrier)
        if ((mi & 1) == 1) load_part(gc + 2, 2 * ks + (mi >> 1));
      }
    }
    if (gc % kGuChunks != kGuChunks - 1) continue;
    // epilogue of tile it: old values (from L2) + W R
    int64_t row0, col0;
    tile_rc(gc / kGuChunks, row0, col0);
    const bool needC = row0 != k0;
    double2 old[4][2][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const int r = wr + 16 * mi + g + 8 * h, c = wc + 8 * ni + 2 * t;
          old[mi][h][ni] = needC ? __ldcg(reinterpret_cast<const double2 *>(a.A + (row0 + r) * a.ld + col0 + c))
                                 : make_double2(0.0, 0.0);
        }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = wr + 16 * mi + g + 8 * h;
        double *o = a.A + (row0 + r) * a.ld + col0;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const int c = wc + 8 * ni + 2 * t;
          *reinterpret_cast<double2 *>(o + c) = make_double2(old[mi][h][ni].x + acc[mi][ni][2 * h],
                                                             old[mi][h][ni].y + acc[mi][ni][2 * h + 1]);
          acc[mi][ni][2 * h] = 0.0;
          acc[mi][ni][2 * h + 1] = 0.0;
        }
      }
  }
}

// The padding of an n x n matrix to np x np: identity (its inverse is the
// identity again, and it never mixes with the n x n part); and the
// bookkeeping arrays of the pivot-block inversions.
__global__ void gj_prepare_kernel(double *A, int64_t n, int64_t np, int64_t ld, int64_t *off, int32_t *size,
                                  int32_t *info, int steps) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t pad = np - n;
  // rows n..np-1 (all np columns), then columns n..np-1 of rows 0..n-1
  const int64_t total = pad * np + n * pad;
  for (int64_t t = t0; t < total; t += stride) {
    int64_t i, j;
    if (t < pad * np) {
      i = n + t / np;
      j = t % np;
    } else {
      i = (t - pad * np) / pad;
      j = n + (t - pad * np) % pad;
    }
    A[i * ld + j] = (i == j) ? 1.0 : 0.0;
  }
  if (t0 == 0) {
    off[0] = 0;
    size[0] = kGjB;
  }
  for (int64_t t = t0; t < steps; t += stride) info[t] = 0;
}

struct GjWorkspace {
  size_t q, r, info, off, size, bytes;
};

GjWorkspace gj_layout(int64_t np, int64_t ld) {
  GjWorkspace w{};
  size_t o = 0;
  auto take = [&](size_t nb) {
    const size_t at = o;
    o += round_up(nb, 256);
    return at;
  };
  w.q = take(static_cast<size_t>(kGjB) * kGjB * sizeof(double));
  w.r = take(static_cast<size_t>(kGjB) * static_cast<size_t>(ld) * sizeof(double));
  w.info = take(static_cast<size_t>(np / kGjB) * sizeof(int32_t));
  w.off = take(sizeof(int64_t));
  w.size = take(sizeof(int32_t));
  w.bytes = o;
  return w;
}

}  // namespace
}  // namespace f3d

extern "C" {

int f3d_dense_inverse_workspace_bytes(int64_t n, int64_t ld, size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  if (n < 0 || ld < 0) return F3D_ERR_SHAPE;
  const int64_t np = static_cast<int64_t>(f3d::round_up(static_cast<size_t>(n), f3d::kGjB));
  *bytes = f3d::gj_layout(np, std::max<int64_t>(ld, np)).bytes;
  return F3D_OK;
}

int f3d_dense_inverse(double *A, int64_t n, int64_t ld, void *workspace, size_t workspace_bytes, void *stream) {
  using namespace f3d;
  if (n < 0) return F3D_ERR_SHAPE;
  if (n == 0) return F3D_OK;
  if (!A || !workspace) return F3D_ERR_NULL;
  const int64_t np = static_cast<int64_t>(round_up(static_cast<size_t>(n), kGjB));
  const int64_t tiles = np / kGjB;
  if (ld < np || (ld & 1)) return F3D_ERR_SHAPE;
  if (tiles > 65535) return F3D_ERR_TOO_LARGE;
  if (!aligned(A, 16) || !aligned(workspace, 256)) return F3D_ERR_ALIGN;
  const GjWorkspace L = gj_layout(np, ld);
  if (workspace_bytes < L.bytes) return F3D_ERR_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char *w = static_cast<unsigned char *>(workspace);
  double *Q = reinterpret_cast<double *>(w + L.q), *R = reinterpret_cast<double *>(w + L.r);
  int32_t *info = reinterpret_cast<int32_t *>(w + L.info);
  int64_t *off = reinterpret_cast<int64_t *>(w + L.off);
  int32_t *size = reinterpret_cast<int32_t *>(w + L.size);

  if (cudaFuncSetAttribute(gj_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kGjSmemPanel)) != cudaSuccess ||
      cudaFuncSetAttribute(gj_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kGjSmemUpdate)) != cudaSuccess)
    return F3D_ERR_CUDA;
  const int64_t update_tiles = (tiles - 1) * tiles;
  const unsigned update_grid = static_cast<unsigned>(std::min<int64_t>(update_tiles, sm_count()));
  const int prep_blocks = static_cast<int>(std::min<int64_t>(4 * sm_count(), std::max<int64_t>(1, (np - n) * 2 * np / 256 + 1)));
  gj_prepare_kernel<<<prep_blocks, 256, 0, st>>>(A, n, np, ld, off, size, info, static_cast<int>(tiles));
  if (launch_status()) return F3D_ERR_CUDA;

  GjArgs a{};
  a.A = A;
  a.R = R;
  a.Q = Q;
  a.ld = ld;
  a.err = device_error_word();
  if (!a.err) return F3D_ERR_CUDA;
  const size_t row_bytes = static_cast<size_t>(ld) * sizeof(double);
  for (int s = 0; s < tiles; ++s) {
    const int64_t k0 = static_cast<int64_t>(s) * kGjB;
    if (cudaMemcpy2DAsync(Q, kGjB * sizeof(double), A + k0 * ld + k0, row_bytes, kGjB * sizeof(double), kGjB,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return F3D_ERR_CUDA;
    int rc = f3d_batched_inverse(Q, off, size, 1, kGjB, nullptr, info + s, st);
    if (rc) return rc;
    if (cudaMemcpyAsync(R, A + k0 * ld, kGjB * row_bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return F3D_ERR_CUDA;
    a.s = s;
    gj_panel_kernel<<<static_cast<unsigned>(tiles), kGjThreads, kGjSmemPanel, st>>>(a);
    if (launch_status()) return F3D_ERR_CUDA;
    if (tiles > 1) {
      gj_update_kernel<<<update_grid, kGuThreads, kGjSmemUpdate, st>>>(a, static_cast<int>(tiles));
      if (launch_status()) return F3D_ERR_CUDA;
    }
  }
  std::vector<int32_t> h(static_cast<size_t>(tiles));
  int err = 0;
  if (cudaMemcpyAsync(h.data(), info, h.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&err, a.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return F3D_ERR_CUDA;
  if (err != 0) {
    if (cudaMemsetAsync(a.err, 0, sizeof(int), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return F3D_ERR_CUDA;
    return err;
  }
  for (int32_t v : h)
    if (v != 0) return F3D_ERR_SINGULAR;
  return F3D_OK;
}

}  // extern "C"
