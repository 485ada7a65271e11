// Fast multipole evaluation of the Stokes single- and double-layer sums for
// large point counts: the GPU counterpart of the STKFMM calls fiber3d makes
// when options.useFMM is set (python/kernels/kernels.py:1298-1485, the
// PVel kernel, set up at tstep/tstep.py:116-137).  STKFMM itself is an
// external kernel-independent FMM (KIFMM); this file is a KIFMM of its own
// on a uniform octree, designed for one GPU:
//
//   * Equivalent densities live on cube surfaces of p points per edge
//     (n = 6 (p - 1)^2 + 2 points): upward equivalent surface at 1.05 box
//     half-widths, upward check at 2.95, downward check at 1.05 and
//     downward equivalent at 2.95.  A density has 4 components per point,
//     a Stokeslet (3) and a potential source r / r^3 (1): the far field of a
//     double layer with a trace carries a net flux that Stokeslets alone
//     cannot represent.  The far-field kernel K4 = [I/r + r r^T/r^3 | r/r^3]
//     has no constants; the densities absorb them.
//   * Densities are stored unit-scaled, (f, q / h) for a box of half-width
//     h, so that every translation operator is the same at every level: the
//     Stokeslet part of K4 is homogeneous of degree -1 and the source part
//     of degree -2, which leaves factors 1/2 (child to parent) and 2
//     (parent to child) on the source component.
//   * The only stored matrices are the two pseudo-inverses, check potential
//     to equivalent density (4n x 3n each, computed by the caller).  Every
//     translation (M2M, M2L, L2L) is generated on the fly from the geometry
//     inside a gathered FP64 GEMM: a CTA tile of check-point rows times
//     box columns, the K dimension running over the terms of the operator
//     (8 children, up to 189 interaction-list boxes and the parent; at level
//     2, where every level-1 box neighbours every other, the 316 far
//     offsets) and each term's 4n equivalent-density components; the kernel
//     values are formed into shared memory for each K slice and reused by
//     all 64 columns, the products on the FP64 tensor cores (mma.sync
//     m16n8k16).
//   * Near field (the 27 neighbour leaves, both kernels, coincident points
//     excluded) and the local expansion's evaluation at the targets (L2P)
//     run in one kernel per target leaf.
//   * Tree: Morton keys at depth 8, a bitonic sort of (key, index) pairs
//     (deterministic), dense per-level slot tables built by a scan, the
//     depth chosen as the smallest with at most max_pts sources per
//     non-empty leaf on average (2 <= depth <= 8).
#include <algorithm>
#include <cmath>
#include <vector>

#include "f3d_common.cuh"
#include "f3d_pair_math.cuh"

struct f3d_fmm;

namespace f3d {
namespace fmm {

constexpr int kMaxDepth = 8;
constexpr double kRin = 1.05, kRout = 2.95;
constexpr double kCoincident2 = 1e-300;  // pairs closer than 1e-150 are excluded
constexpr int kScanTile = 4096;          // 1024 threads x 4
constexpr int64_t kMaxScan = int64_t(kScanTile) * kScanTile;

// ------------------------------------------------------------ Morton keys --
__host__ __device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 8 bits -> 24
  v &= 0xFFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__host__ __device__ __forceinline__ uint32_t compact3(uint32_t v) {  // inverse of spread3
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030C30C3u;
  v = (v | (v >> 4)) & 0x0300F00Fu;
  v = (v | (v >> 8)) & 0x030000FFu;
  v = (v | (v >> 16)) & 0x000000FFu;
  return v;
}

__host__ __device__ __forceinline__ uint32_t morton(uint32_t ix, uint32_t iy, uint32_t iz) {
  return (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
}

__host__ __device__ __forceinline__ void unmorton(uint32_t key, int &ix, int &iy, int &iz) {
  ix = static_cast<int>(compact3(key >> 2));
  iy = static_cast<int>(compact3(key >> 1));
  iz = static_cast<int>(compact3(key));
}

// (key at depth 8) << 32 | index; past-the-end slots of the padded array
// hold the largest value
__global__ void keys_kernel(const double *__restrict__ x, int64_t n, int64_t n2, double lo0, double lo1,
                            double lo2, double inv_cell, uint64_t *kv) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n2) return;
  if (i >= n) {
    kv[i] = ~uint64_t(0);
    return;
  }
  auto cell = [inv_cell](double v, double lo) {
    const double c = floor((v - lo) * inv_cell);
    return static_cast<uint32_t>(c < 0.0 ? 0.0 : (c > 255.0 ? 255.0 : c));
  };
  const uint32_t key = morton(cell(x[3 * i], lo0), cell(x[3 * i + 1], lo1), cell(x[3 * i + 2], lo2));
  kv[i] = (static_cast<uint64_t>(key) << 32) | static_cast<uint32_t>(i);
}

// ------------------------------------------------------------ bitonic sort --
// Ascending sort of a power-of-two array (at least 2048 elements): chunks of
// 2048 are sorted in shared memory, then each merge stage runs its strides of
// 2048 and more as one global pass each and the rest in shared memory.
__device__ __forceinline__ void cmp_swap(uint64_t &a, uint64_t &b, bool asc) {
  if ((a > b) == asc) {
    const uint64_t t = a;
    a = b;
    b = t;
  }
}

__global__ void __launch_bounds__(1024) bitonic_chunks_kernel(uint64_t *a, int64_t kmin) {
  __shared__ uint64_t s[2048];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * 2048;
  const int t = threadIdx.x;
  s[t] = a[base + t];
  s[t + 1024] = a[base + t + 1024];
  __syncthreads();
  // kmin == 2: full sort of the chunk; kmin > 2048: the in-chunk strides of
  // merge stage kmin
  const int64_t k_lo = kmin, k_hi = kmin > 2048 ? kmin : 2048;
  for (int64_t k = k_lo; k <= k_hi; k <<= 1) {
    for (int64_t j = (k > 2048 ? 1024 : k >> 1); j > 0; j >>= 1) {
      const int i = static_cast<int>((t / j) * 2 * j + (t % j));
      const bool asc = ((base + i) & k) == 0;
      cmp_swap(s[i], s[i + j], asc);
      __syncthreads();
    }
  }
  a[base + t] = s[t];
  a[base + t + 1024] = s[t + 1024];
}

__global__ void bitonic_global_kernel(uint64_t *a, int64_t half, int64_t j, int64_t k) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= half) return;
  const int64_t i = (t / j) * 2 * j + (t % j);
  const bool asc = (i & k) == 0;
  uint64_t x = a[i], y = a[i + j];
  cmp_swap(x, y, asc);
  a[i] = x;
  a[i + j] = y;
}

static int sort_u64(uint64_t *a, int64_t n2, cudaStream_t st) {
  const unsigned chunks = static_cast<unsigned>(n2 / 2048);
  bitonic_chunks_kernel<<<chunks, 1024, 0, st>>>(a, 2);
  for (int64_t k = 4096; k <= n2; k <<= 1) {
    for (int64_t j = k >> 1; j >= 2048; j >>= 1) {
      const int64_t half = n2 / 2;
      bitonic_global_kernel<<<static_cast<unsigned>((half + 255) / 256), 256, 0, st>>>(a, half, j, k);
    }
    bitonic_chunks_kernel<<<chunks, 1024, 0, st>>>(a, k);
  }
  return launch_status();
}

// ------------------------------------------------------------ exclusive scan --
__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += u;
  }
  return v;
}

// block-wide exclusive scan of one value per thread (1024 threads); returns
// the block total through *total
__device__ __forceinline__ int block_excl_scan(int v, int *total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int inc = warp_incl_scan(v);
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int w = ws[lane];
    ws[lane] = warp_incl_scan(w) - w;
  }
  __syncthreads();
  const int res = ws[warp] + inc - v;
  if (threadIdx.x == 1023) *total = res + v;
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(1024) scan_tiles_kernel(int *a, int64_t n, int *tile_sums) {
  __shared__ int total;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + 4 * threadIdx.x;
  int v[4], s = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    v[q] = base + q < n ? a[base + q] : 0;
    s += v[q];
  }
  int pre = block_excl_scan(s, &total);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (base + q < n) a[base + q] = pre;
    pre += v[q];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(int *sums, int ntiles, int *grand_total) {
  __shared__ int total;
  int v[4], s = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = 4 * threadIdx.x + q;
    v[q] = i < ntiles ? sums[i] : 0;
    s += v[q];
  }
  int pre = block_excl_scan(s, &total);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = 4 * threadIdx.x + q;
    if (i < ntiles) sums[i] = pre;
    pre += v[q];
  }
  if (threadIdx.x == 0) *grand_total = total;
}

__global__ void scan_add_kernel(int *a, int64_t n, const int *tile_sums) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) a[i] += tile_sums[i / kScanTile];
}

// in-place exclusive scan of a[0, n), n <= 2^24; the total to *d_total
static int scan_exclusive(int *a, int64_t n, int *tile_sums, int *d_total, cudaStream_t st) {
  if (n > kMaxScan) return F3D_ERR_TOO_LARGE;
  const int ntiles = static_cast<int>((n + kScanTile - 1) / kScanTile);
  scan_tiles_kernel<<<ntiles, 1024, 0, st>>>(a, n, tile_sums);
  scan_sums_kernel<<<1, 1024, 0, st>>>(tile_sums, ntiles, d_total);
  scan_add_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(a, n, tile_sums);
  return launch_status();
}

// ------------------------------------------------------------ tree kernels --
// number of distinct keys at depths 2..8 of a sorted key array (counts[d])
__global__ void count_levels_kernel(const uint64_t *__restrict__ kv, int64_t n, unsigned *counts) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool in = i < n;
  const uint32_t k = in ? static_cast<uint32_t>(kv[i] >> 32) : 0u;
  const uint32_t kp = (in && i > 0) ? static_cast<uint32_t>(kv[i - 1] >> 32) : 0u;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 2; d <= kMaxDepth; ++d) {
    const int sh = 3 * (kMaxDepth - d);
    const bool first = in && (i == 0 || (k >> sh) != (kp >> sh));
    const unsigned b = __ballot_sync(0xffffffffu, first);
    if (lane == 0 && b) atomicAdd(&counts[d], static_cast<unsigned>(__popc(b)));
  }
}

// flags[key at depth d] = 1 for every point of a sorted array
__global__ void flag_points_kernel(const uint64_t *__restrict__ kv, int64_t n, int shift, int *flags) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) flags[static_cast<uint32_t>(kv[i] >> 32) >> shift] = 1;
}

// flags[parent] = 1 for every box of the level below
__global__ void flag_parents_kernel(const int *__restrict__ keys, int nbox, int *flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nbox) flags[keys[i] >> 3] = 1;
}

// after the exclusive scan of flags (copy kept in flagged): table[key] =
// slot or -1, keys[slot] = key
__global__ void finish_table_kernel(const int *__restrict__ flagged, int *table, int64_t nkeys, int *keys) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= nkeys) return;
  if (flagged[k]) {
    keys[table[k]] = static_cast<int>(k);
  } else {
    table[k] = -1;
  }
}

// point range [start, end) of each leaf of a sorted array
__global__ void leaf_ranges_kernel(const uint64_t *__restrict__ kv, int64_t n, int shift,
                                   const int *__restrict__ table, int64_t *start, int64_t *end) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t k = static_cast<uint32_t>(kv[i] >> 32) >> shift;
  const int slot = table[k];
  if (i == 0 || (static_cast<uint32_t>(kv[i - 1] >> 32) >> shift) != k) start[slot] = i;
  if (i == n - 1 || (static_cast<uint32_t>(kv[i + 1] >> 32) >> shift) != k) end[slot] = i + 1;
}

// (octant << 32 | slot) of every box of a level, for grouping by octant
__global__ void octant_keys_kernel(const int *__restrict__ keys, int nbox, int64_t n2, uint64_t *kv,
                                   unsigned *oct_count) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n2) return;
  if (i >= nbox) {
    kv[i] = ~uint64_t(0);
    return;
  }
  const unsigned oct = static_cast<unsigned>(keys[i]) & 7u;
  kv[i] = (static_cast<uint64_t>(oct) << 32) | static_cast<uint32_t>(i);
  atomicAdd(&oct_count[oct], 1u);
}

// number of non-empty source boxes in the interaction lists of a level's
// target boxes (the M2L work: each is one 3n x 4n block product)
__global__ void count_m2l_kernel(const int *__restrict__ trg_keys, int ntrg, const int *__restrict__ src_table,
                                 int level, unsigned long long *count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned c = 0;
  if (i < ntrg) {
    int bx, by, bz;
    unmorton(static_cast<uint32_t>(trg_keys[i]), bx, by, bz);
    const int px = bx >> 1, py = by >> 1, pz = bz >> 1, m = 1 << level;
    for (int x = 2 * px - 2; x < 2 * px + 4; ++x)
      for (int y = 2 * py - 2; y < 2 * py + 4; ++y)
        for (int z = 2 * pz - 2; z < 2 * pz + 4; ++z) {
          if (x < 0 || y < 0 || z < 0 || x >= m || y >= m || z >= m) continue;
          if (max(abs(x - bx), max(abs(y - by), abs(z - bz))) < 2) continue;
          c += src_table[morton(x, y, z)] >= 0;
        }
  }
  for (int d = 16; d > 0; d >>= 1) c += __shfl_down_sync(0xffffffffu, c, d);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

__global__ void low_words_kernel(const uint64_t *__restrict__ kv, int64_t n, int *out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = static_cast<int>(static_cast<uint32_t>(kv[i]));
}

// out[i] = in[index of sorted element i] (c values per point)
__global__ void gather_kernel(const double *__restrict__ in, const uint64_t *__restrict__ kv, int64_t n, int c,
                              double *out) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= n * c) return;
  const int64_t i = e / c;
  const uint32_t src = static_cast<uint32_t>(kv[i]);
  out[e] = in[static_cast<int64_t>(src) * c + (e - i * c)];
}

// out[index of sorted element i] = scale * in[i] (3 values per point)
__global__ void scatter_kernel(const double *__restrict__ in, const uint64_t *__restrict__ kv, int64_t n,
                               double scale, double *out) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= 3 * n) return;
  const int64_t i = e / 3;
  const uint32_t dst = static_cast<uint32_t>(kv[i]);
  out[3 * static_cast<int64_t>(dst) + (e - 3 * i)] = scale * in[e];
}

// per-block min and max of three point sets (6 values per block)
__global__ void bbox_kernel(const double *__restrict__ a, int64_t na, const double *__restrict__ b, int64_t nb,
                            const double *__restrict__ c, int64_t nc, double *partial) {
  __shared__ double s[6][256];
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  const int64_t total = na + nb + nc;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double *p = i < na ? a + 3 * i : (i < na + nb ? b + 3 * (i - na) : c + 3 * (i - na - nb));
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mn[d] = fmin(mn[d], p[d]);
      mx[d] = fmax(mx[d], p[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    s[d][threadIdx.x] = mn[d];
    s[3 + d][threadIdx.x] = mx[d];
  }
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + w]);
        s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + w]);
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < 6) partial[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

// ------------------------------------------------------------ P2M check --
struct Geometry {
  double lo[3];
  double width;  // side of the cube
};

__device__ __forceinline__ void box_center(const Geometry &g, int key, int level, double c[3], double &h) {
  int ix, iy, iz;
  unmorton(static_cast<uint32_t>(key), ix, iy, iz);
  const double cell = g.width / static_cast<double>(1 << level);
  h = 0.5 * cell;
  c[0] = g.lo[0] + (ix + 0.5) * cell;
  c[1] = g.lo[1] + (iy + 0.5) * cell;
  c[2] = g.lo[2] + (iz + 0.5) * cell;
}

struct SourceSet {
  const double *xsl, *fsl;  // single layer: positions, forces (n x 3), sorted
  const double *xdl, *ddl;  // double layer: positions (n x 3), tensors D (n x 9), sorted
  const int64_t *sl_start, *sl_end, *dl_start, *dl_end;  // per source leaf
};

// Stokeslet (single layer) and stresslet (double layer) velocities of the
// sources of one leaf at its n upward check points, with the kernels'
// constants: 1/(8 pi) and -3/(8 pi) r_i (r^T D r) / r^5.
__global__ void __launch_bounds__(128) p2m_check_kernel(const Geometry g, int level, const int *__restrict__ keys,
                                                        SourceSet src, const double *__restrict__ surf, int n,
                                                        double *Y) {
  __shared__ double sp[128][3], sv[128][9];
  const int leaf = blockIdx.x;
  double c[3], h;
  box_center(g, keys[leaf], level, c, h);
  const int k = blockIdx.y * 128 + threadIdx.x;
  const bool kv = k < n;
  double x[3] = {0.0, 0.0, 0.0};
  if (kv) {
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = c[d] + kRout * h * surf[3 * k + d];
  }
  double us[3] = {0.0, 0.0, 0.0}, ud[3] = {0.0, 0.0, 0.0};
  for (int type = 0; type < 2; ++type) {
    const int64_t j0 = type == 0 ? src.sl_start[leaf] : src.dl_start[leaf];
    const int64_t j1 = type == 0 ? src.sl_end[leaf] : src.dl_end[leaf];
    const double *px = type == 0 ? src.xsl : src.xdl;
    const double *pv = type == 0 ? src.fsl : src.ddl;
    const int nv = type == 0 ? 3 : 9;
    for (int64_t jb = j0; jb < j1; jb += 128) {
      const int cnt = static_cast<int>(min(static_cast<int64_t>(128), j1 - jb));
      __syncthreads();
      if (threadIdx.x < cnt) {
        const int64_t j = jb + threadIdx.x;
#pragma unroll
        for (int d = 0; d < 3; ++d) sp[threadIdx.x][d] = px[3 * j + d];
        for (int q = 0; q < nv; ++q) sv[threadIdx.x][q] = pv[nv * j + q];
      }
      __syncthreads();
      if (!kv) continue;
      for (int s = 0; s < cnt; ++s) {
        const double r0 = x[0] - sp[s][0], r1 = x[1] - sp[s][1], r2 = x[2] - sp[s][2];
        const double d2 = fma(r0, r0, fma(r1, r1, r2 * r2));
        if (type == 0) {
          const double ri = rsqrt_refined(d2);
          const double g3 = ri * ri * ri * fma(r0, sv[s][0], fma(r1, sv[s][1], r2 * sv[s][2]));
          us[0] = fma(g3, r0, fma(ri, sv[s][0], us[0]));
          us[1] = fma(g3, r1, fma(ri, sv[s][1], us[1]));
          us[2] = fma(g3, r2, fma(ri, sv[s][2], us[2]));
        } else {
          const double *D = sv[s];
          const double q = r0 * fma(D[0], r0, fma(D[1], r1, D[2] * r2)) +
                           r1 * fma(D[3], r0, fma(D[4], r1, D[5] * r2)) +
                           r2 * fma(D[6], r0, fma(D[7], r1, D[8] * r2));
          const double f = times_rsqrt5(q, d2);
          ud[0] = fma(f, r0, ud[0]);
          ud[1] = fma(f, r1, ud[1]);
          ud[2] = fma(f, r2, ud[2]);
        }
      }
    }
  }
  if (kv) {
    const double cs = 1.0 / (8.0 * kPi), cd = -3.0 / (8.0 * kPi);
    double *y = Y + static_cast<int64_t>(leaf) * 3 * n + 3 * k;
#pragma unroll
    for (int d = 0; d < 3; ++d) y[d] = cs * us[d] + cd * ud[d];
  }
}

// ------------------------------------------------------------ gathered GEMM --
// Y[slot(col)][row] (+)= scale * sum_t sum_k A_t[row][k] X_t[src(col, t)][k]
//
// A is either a stored matrix (the pseudo-inverses) or generated from K4
// between check points (crad * surface) and a term's equivalent points
// (off_t + erad_t * surface), with the source component scaled by qscale_t.
// Terms: M2M, the 8 children of the column's box; M2L, the column's
// interaction list (189 boxes of the 6 x 6 x 6 children of its parent's
// neighbours that are not its own neighbours; which 189 depends on the
// box's octant in its parent) and optionally the parent's local expansion.
// The columns of M2L are grouped by octant; a CTA's 64 columns share one.
// Terms are split over grid.z; each split writes its own partial and a
// second kernel adds the partials in split order (deterministic).
constexpr int GBM = 96, GBN = 64, GBK = 32, GTHREADS = 128;
// shared row strides (doubles), 4 mod 16: the tensor-core fragment reads of
// a half-warp (A: k = t + 4q, row g; B: k = t + 4j, column g) hit 16
// different bank pairs
constexpr int GAS = GBM + 4, GXS = GBN + 4;
constexpr int kM2LTerms = 189;
constexpr int kFarTerms = 316;  // level 2: every box at distance >= 2, (7^3 - 3^3) offsets

enum GenMode { GEN_STORED = 0, GEN_M2M = 1, GEN_M2L = 2 };

struct GemmOp {
  double *Y;
  int ldy, rows, accumulate;
  double scale;
  double *partial;  // nsplit > 1: [nsplit][nslots][ldy]
  int nslots, nsplit;
  int ncols;
  const int *cols;  // column -> box slot (null: identity)
  int oct_col_start[9], oct_tile_start[9];  // column groups by octant (M2L); else one group
  const int *box_keys;
  int level;
  int mode;
  const double *A;
  int lda, K;
  const double *surf;
  int n;
  double crad;
  int nterms, parent;
  unsigned char m2l_idx[8][kM2LTerms];  // a*36 + b*6 + d of each interaction box, per octant
  int all_offsets;                      // level 2: the terms are the 316 far offsets, no octant groups
  unsigned short far_idx[kFarTerms];    // a*49 + b*7 + d of each offset (a, b, d - 3)
  const int *table;   // sources of this level (M2L) or of the level below (M2M)
  const int *table2;  // targets of the level above (the parent term)
  const double *X, *X2;
  int ldx;
};

struct TermGeom {
  double off[3];
  double erad, qscale;
};

__device__ __forceinline__ TermGeom term_geom(const GemmOp &op, int oct, int t) {
  TermGeom g;
  const int cx = (oct >> 2) & 1, cy = (oct >> 1) & 1, cz = oct & 1;
  if (op.mode == GEN_M2M) {
    g.off[0] = (t & 4) ? 0.5 : -0.5;
    g.off[1] = (t & 2) ? 0.5 : -0.5;
    g.off[2] = (t & 1) ? 0.5 : -0.5;
    g.erad = 0.5 * kRin;
    g.qscale = 0.5;
  } else if (op.parent && t == op.nterms - 1) {
    // the parent's downward equivalent surface in this box's units
    g.off[0] = cx ? -1.0 : 1.0;
    g.off[1] = cy ? -1.0 : 1.0;
    g.off[2] = cz ? -1.0 : 1.0;
    g.erad = 2.0 * kRout;
    g.qscale = 2.0;
  } else if (op.all_offsets) {
    const int idx = op.far_idx[t];
    g.off[0] = 2.0 * (idx / 49 - 3);
    g.off[1] = 2.0 * ((idx / 7) % 7 - 3);
    g.off[2] = 2.0 * (idx % 7 - 3);
    g.erad = kRin;
    g.qscale = 1.0;
  } else {
    const int idx = op.m2l_idx[oct][t];
    g.off[0] = 2.0 * (idx / 36 - 2 - cx);
    g.off[1] = 2.0 * ((idx / 6) % 6 - 2 - cy);
    g.off[2] = 2.0 * (idx % 6 - 2 - cz);
    g.erad = kRin;
    g.qscale = 1.0;
  }
  return g;
}

__device__ __forceinline__ int source_slot(const GemmOp &op, int oct, int slot, int t) {
  if (op.mode == GEN_STORED) return slot;
  const int key = op.box_keys[slot];
  if (op.mode == GEN_M2M) return op.table[(key << 3) | t];
  if (op.parent && t == op.nterms - 1) return op.table2[key >> 3];
  int ix, iy, iz;
  unmorton(static_cast<uint32_t>(key), ix, iy, iz);
  if (op.all_offsets) {
    const int idx = op.far_idx[t];
    ix += idx / 49 - 3;
    iy += (idx / 7) % 7 - 3;
    iz += idx % 7 - 3;
  } else {
    const int idx = op.m2l_idx[oct][t];
    const int cx = (oct >> 2) & 1, cy = (oct >> 1) & 1, cz = oct & 1;
    ix += idx / 36 - 2 - cx;
    iy += (idx / 6) % 6 - 2 - cy;
    iz += idx % 6 - 2 - cz;
  }
  const int m = 1 << op.level;
  if (ix < 0 || iy < 0 || iz < 0 || ix >= m || iy >= m || iz >= m) return -1;
  return op.table[morton(ix, iy, iz)];
}

__global__ void __launch_bounds__(GTHREADS) fmm_gemm_kernel(const __grid_constant__ GemmOp op) {
  __shared__ __align__(16) double As[GBK][GAS];
  __shared__ __align__(16) double Xs[GBK][GXS];
  __shared__ int s_src[GBN];
  __shared__ int s_any;
  const int tid = threadIdx.x;
  const int row0 = blockIdx.x * GBM;
  // the column tile's octant group
  const int tile = blockIdx.y;
  int oct = 0;
  while (oct < 7 && tile >= op.oct_tile_start[oct + 1]) ++oct;
  const int col0 = op.oct_col_start[oct] + (tile - op.oct_tile_start[oct]) * GBN;
  const int col_end = op.oct_col_start[oct + 1];
  const int tps = (op.nterms + op.nsplit - 1) / op.nsplit;
  const int t_lo = blockIdx.z * tps, t_hi = min(op.nterms, t_lo + tps);
  // FP64 tensor cores (mma.sync m16n8k16): warp w computes rows
  // 48 (w / 2) .. + 47 and columns 32 (w % 2) .. + 31 of the tile as 3 x 4
  // tiles of 16 x 8; lane = 4 lg + t4 holds rows lg, lg + 8 and columns
  // 2 t4, 2 t4 + 1 of each
  const int lane = tid & 31, warp = tid >> 5;
  const int lg = lane >> 2, t4 = lane & 3;
  const int wr = 48 * (warp >> 1), wc = 32 * (warp & 1);
  double acc[3][4][4];
#pragma unroll
  for (int mi = 0; mi < 3; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[mi][ni][i] = 0.0;

  for (int t = t_lo; t < t_hi; ++t) {
    if (tid == 0) s_any = 0;
    __syncthreads();
    if (tid < GBN) {
      const int col = col0 + tid;
      int s = -1;
      if (col < col_end) s = source_slot(op, oct, op.cols ? op.cols[col] : col, t);
      s_src[tid] = s;
      if (s >= 0) s_any = 1;
    }
    __syncthreads();
    if (!s_any) continue;
    const bool par = op.mode == GEN_M2L && op.parent && t == op.nterms - 1;
    const double *X = par ? op.X2 : op.X;
    TermGeom g{};
    if (op.mode != GEN_STORED) g = term_geom(op, oct, t);
    for (int k0 = 0; k0 < op.K; k0 += GBK) {
      if (op.mode == GEN_STORED) {
        for (int e = tid; e < GBM * GBK; e += GTHREADS) {
          const int r = e / GBK, kk = e % GBK;
          const int row = row0 + r, k = k0 + kk;
          As[kk][r] = (row < op.rows && k < op.K) ? op.A[static_cast<int64_t>(row) * op.lda + k] : 0.0;
        }
      } else {
        // 32 check points x 8 equivalent points: one 3 x 4 block of K4 each
        // (a warp takes 32 consecutive check points of one equivalent point)
        for (int pp = tid; pp < (GBM / 3) * (GBK / 4); pp += GTHREADS) {
          const int ci = pp % (GBM / 3), ei = pp / (GBM / 3);
          const int cp = row0 / 3 + ci, ep = k0 / 4 + ei;
          double v[3][4];
          if (cp < op.n && ep < op.n) {
            const double r0 = op.crad * op.surf[3 * cp] - (g.off[0] + g.erad * op.surf[3 * ep]);
            const double r1 = op.crad * op.surf[3 * cp + 1] - (g.off[1] + g.erad * op.surf[3 * ep + 1]);
            const double r2 = op.crad * op.surf[3 * cp + 2] - (g.off[2] + g.erad * op.surf[3 * ep + 2]);
            const double ri = rsqrt_refined(fma(r0, r0, fma(r1, r1, r2 * r2)));
            const double ri3 = ri * ri * ri;
            const double r[3] = {r0, r1, r2};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
#pragma unroll
              for (int j = 0; j < 3; ++j) v[i][j] = fma(r[i] * r[j], ri3, i == j ? ri : 0.0);
              v[i][3] = r[i] * ri3 * g.qscale;
            }
          } else {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
              for (int j = 0; j < 4; ++j) v[i][j] = 0.0;
          }
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) As[4 * ei + j][3 * ci + i] = v[i][j];
        }
      }
      // a warp gathers 4 boxes x 8 consecutive k (64-byte runs of each box's
      // densities); its stores then fill the 16 bank pairs twice over
      // (4 kk + c over the stride 4 mod 16), the minimum for 256 bytes
      for (int e = tid; e < GBN * GBK; e += GTHREADS) {
        const int blk = e >> 5;
        const int c = 4 * (blk % (GBN / 4)) + (e & 3);
        const int kk = 8 * (blk / (GBN / 4)) + ((e >> 2) & 7);
        const int s = s_src[c], k = k0 + kk;
        Xs[kk][c] = (s >= 0 && k < op.K) ? X[static_cast<int64_t>(s) * op.ldx + k] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int ks = 0; ks < GBK; ks += 16) {
        double bf[4][4];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
          for (int j = 0; j < 4; ++j) bf[ni][j] = Xs[ks + t4 + 4 * j][wc + 8 * ni + lg];
#pragma unroll
        for (int mi = 0; mi < 3; ++mi) {
          double af[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) af[q] = As[ks + t4 + 4 * (q >> 1)][wr + 16 * mi + lg + 8 * (q & 1)];
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) mma_f64_16816(acc[mi][ni], af, bf[ni]);
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int ni = 0; ni < 4; ++ni)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int col = col0 + wc + 8 * ni + 2 * t4 + e;
      if (col >= col_end) continue;
      const int slot = op.cols ? op.cols[col] : col;
      double *y = op.nsplit > 1 ? op.partial + (static_cast<int64_t>(blockIdx.z) * op.nslots + slot) * op.ldy
                                : op.Y + static_cast<int64_t>(slot) * op.ldy;
#pragma unroll
      for (int mi = 0; mi < 3; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = row0 + wr + 16 * mi + lg + 8 * h;
          if (row >= op.rows) continue;
          const double v = acc[mi][ni][2 * h + e];
          if (op.nsplit > 1)
            y[row] = v;
          else
            y[row] = op.accumulate ? fma(op.scale, v, y[row]) : op.scale * v;
        }
    }
}

// Y[slot][row] (+)= scale * sum over splits of the partials, in split order
__global__ void split_sum_kernel(const double *__restrict__ partial, int nsplit, int64_t nslots, int ldy, int rows,
                                 double scale, int accumulate, double *Y) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= nslots * rows) return;
  const int64_t slot = e / rows;
  const int row = static_cast<int>(e - slot * rows);
  double v = 0.0;
  for (int z = 0; z < nsplit; ++z) v += partial[(z * nslots + slot) * ldy + row];
  double *y = Y + slot * ldy + row;
  *y = accumulate ? fma(scale, v, *y) : scale * v;
}


// ------------------------------------------------------------ near field + L2P --
struct NearArgs {
  Geometry g;
  int level;
  const int *trg_keys;                  // target leaf slot -> key
  const int64_t *trg_start, *trg_end;   // target leaf ranges (sorted targets)
  const double *xt;                     // sorted targets
  const int *src_table;                 // dense source-leaf table
  SourceSet src;
  const double *psi;                    // downward equivalent densities (4n per target leaf)
  const double *surf;
  int n;
  double *out;                          // sorted targets x 3
};

// Two targets per thread (t and t + 128 of a 256-target block of the leaf):
// each staged source serves both.
__global__ void __launch_bounds__(128) near_l2p_kernel(const NearArgs a) {
  __shared__ double sp[128][3], sv[128][9];
  const int leaf = blockIdx.x;
  const int key = a.trg_keys[leaf];
  double c[3], h;
  box_center(a.g, key, a.level, c, h);
  int bx, by, bz;
  unmorton(static_cast<uint32_t>(key), bx, by, bz);
  const int m = 1 << a.level;
  const int64_t t0 = a.trg_start[leaf], t1 = a.trg_end[leaf];
  for (int64_t tb = t0; tb < t1; tb += 256) {
    double x[2][3];
    bool iv[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int64_t i = tb + threadIdx.x + 128 * q;
      iv[q] = i < t1;
#pragma unroll
      for (int d = 0; d < 3; ++d) x[q][d] = iv[q] ? a.xt[3 * i + d] : c[d];
    }
    double us[2][3] = {}, ud[2][3] = {}, uf[2][3] = {};
    for (int nb = 0; nb < 27; ++nb) {
      const int nx = bx + nb / 9 - 1, ny = by + (nb / 3) % 3 - 1, nz = bz + nb % 3 - 1;
      if (nx < 0 || ny < 0 || nz < 0 || nx >= m || ny >= m || nz >= m) continue;
      const int slot = a.src_table[morton(nx, ny, nz)];
      if (slot < 0) continue;
      // single layer
      for (int64_t jb = a.src.sl_start[slot], j1 = a.src.sl_end[slot]; jb < j1; jb += 128) {
        const int cnt = static_cast<int>(min(static_cast<int64_t>(128), j1 - jb));
        __syncthreads();
        if (threadIdx.x < cnt) {
          const int64_t j = jb + threadIdx.x;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            sp[threadIdx.x][d] = a.src.xsl[3 * j + d];
            sv[threadIdx.x][d] = a.src.fsl[3 * j + d];
          }
        }
        __syncthreads();
        for (int s = 0; s < cnt; ++s) {
          const double p0 = sp[s][0], p1 = sp[s][1], p2 = sp[s][2];
          const double f0 = sv[s][0], f1 = sv[s][1], f2 = sv[s][2];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const double r0 = x[q][0] - p0, r1 = x[q][1] - p1, r2 = x[q][2] - p2;
            const double d2 = fma(r0, r0, fma(r1, r1, r2 * r2));
            double ri = rsqrt_refined(d2);
            ri = d2 > kCoincident2 ? ri : 0.0;
            const double g3 = ri * ri * ri * fma(r0, f0, fma(r1, f1, r2 * f2));
            us[q][0] = fma(g3, r0, fma(ri, f0, us[q][0]));
            us[q][1] = fma(g3, r1, fma(ri, f1, us[q][1]));
            us[q][2] = fma(g3, r2, fma(ri, f2, us[q][2]));
          }
        }
      }
      // double layer
      for (int64_t jb = a.src.dl_start[slot], j1 = a.src.dl_end[slot]; jb < j1; jb += 128) {
        const int cnt = static_cast<int>(min(static_cast<int64_t>(128), j1 - jb));
        __syncthreads();
        if (threadIdx.x < cnt) {
          const int64_t j = jb + threadIdx.x;
#pragma unroll
          for (int d = 0; d < 3; ++d) sp[threadIdx.x][d] = a.src.xdl[3 * j + d];
#pragma unroll
          for (int e = 0; e < 9; ++e) sv[threadIdx.x][e] = a.src.ddl[9 * j + e];
        }
        __syncthreads();
        for (int s = 0; s < cnt; ++s) {
          const double p0 = sp[s][0], p1 = sp[s][1], p2 = sp[s][2];
          const double *D = sv[s];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const double r0 = x[q][0] - p0, r1 = x[q][1] - p1, r2 = x[q][2] - p2;
            const double d2 = fma(r0, r0, fma(r1, r1, r2 * r2));
            const double qq = r0 * fma(D[0], r0, fma(D[1], r1, D[2] * r2)) +
                              r1 * fma(D[3], r0, fma(D[4], r1, D[5] * r2)) +
                              r2 * fma(D[6], r0, fma(D[7], r1, D[8] * r2));
            double f = times_rsqrt5(qq, d2);
            f = d2 > kCoincident2 ? f : 0.0;
            ud[q][0] = fma(f, r0, ud[q][0]);
            ud[q][1] = fma(f, r1, ud[q][1]);
            ud[q][2] = fma(f, r2, ud[q][2]);
          }
        }
      }
    }
    // the local expansion: K4 from the leaf's downward equivalent surface,
    // source component q scaled back by h
    const double *psi = a.psi + static_cast<int64_t>(leaf) * 4 * a.n;
    for (int kb = 0; kb < a.n; kb += 128) {
      const int cnt = min(128, a.n - kb);
      __syncthreads();
      if (threadIdx.x < cnt) {
        const int k = kb + threadIdx.x;
#pragma unroll
        for (int d = 0; d < 3; ++d) sp[threadIdx.x][d] = c[d] + kRout * h * a.surf[3 * k + d];
#pragma unroll
        for (int e = 0; e < 3; ++e) sv[threadIdx.x][e] = psi[4 * k + e];
        sv[threadIdx.x][3] = h * psi[4 * k + 3];
      }
      __syncthreads();
      for (int s = 0; s < cnt; ++s) {
        const double p0 = sp[s][0], p1 = sp[s][1], p2 = sp[s][2];
        const double f0 = sv[s][0], f1 = sv[s][1], f2 = sv[s][2], fq = sv[s][3];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const double r0 = x[q][0] - p0, r1 = x[q][1] - p1, r2 = x[q][2] - p2;
          const double ri = rsqrt_refined(fma(r0, r0, fma(r1, r1, r2 * r2)));
          const double g3 = ri * ri * ri * (fma(r0, f0, fma(r1, f1, r2 * f2)) + fq);
          uf[q][0] = fma(g3, r0, fma(ri, f0, uf[q][0]));
          uf[q][1] = fma(g3, r1, fma(ri, f1, uf[q][1]));
          uf[q][2] = fma(g3, r2, fma(ri, f2, uf[q][2]));
        }
      }
    }
    const double cs = 1.0 / (8.0 * kPi), cd = -3.0 / (8.0 * kPi);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (!iv[q]) continue;
      const int64_t i = tb + threadIdx.x + 128 * q;
#pragma unroll
      for (int d = 0; d < 3; ++d) a.out[3 * i + d] = fma(cs, us[q][d], fma(cd, ud[q][d], uf[q][d]));
    }
  }
}

// D = 2 n (x) d per double-layer source (fiber3d's convention for STKFMM,
// kernels.py:1410)
__global__ void dl_tensor_kernel(const double *__restrict__ nrm, const double *__restrict__ dens, int64_t n,
                                 double *D) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= 9 * n) return;
  const int64_t i = e / 9;
  const int jk = static_cast<int>(e - 9 * i);
  D[e] = 2.0 * nrm[3 * i + jk / 3] * dens[3 * i + jk % 3];
}

}  // namespace fmm
}  // namespace f3d

// ============================================================ host side ====
using namespace f3d;
using namespace f3d::fmm;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};

int reserve(DevBuf &b, size_t bytes) {
  if (b.cap >= bytes && b.p) return F3D_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  if (bytes == 0) return F3D_OK;
  if (cudaMalloc(&b.p, bytes) != cudaSuccess) return F3D_ERR_CUDA;
  b.cap = bytes;
  return F3D_OK;
}

template <typename T>
T *as(DevBuf &b) {
  return static_cast<T *>(b.p);
}

int64_t pow2_at_least(int64_t n, int64_t lo) {
  int64_t p = lo;
  while (p < n) p <<= 1;
  return p;
}

unsigned blocks(int64_t n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

struct Level {
  int nsrc = 0, ntrg = 0;
  DevBuf src_table, trg_table, src_keys, trg_keys, trg_cols, phi, psi;
  int oct_start[9] = {0};
};

}  // namespace

struct f3d_fmm {
  int p = 0, n = 0, max_pts = 0;
  DevBuf surf, uc2ue, dc2de;
  bool box_set = false;
  Geometry geo{};
  int64_t nsl = 0, ndl = 0, ntrg = 0;
  int depth = 0;
  DevBuf kv_sl, kv_dl, kv_trg;          // sorted (key << 32 | index), padded
  DevBuf x_sl, x_dl, x_trg;             // sorted coordinates
  DevBuf f_sl, d_dl, dl_tmp;            // sorted densities (3 and 9 per point)
  DevBuf sl_start, sl_end, dl_start, dl_end, trg_start, trg_end;
  DevBuf flags, tile_sums, scalars, okv, ybuf, out_sorted, bbox, split_partial;
  int64_t m2l_pairs = 0;  // non-empty interaction-list entries over all levels
  int launches = 0;       // kernels the last evaluate launched
  Level lev[kMaxDepth + 1];
};

namespace {

int sync_read(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess) return F3D_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return F3D_ERR_CUDA;
  return F3D_OK;
}

// sorted (key << 32 | index) of n points into kv (padded to a power of two)
int sort_points(f3d_fmm *h, const double *x, int64_t n, DevBuf &kv, cudaStream_t st) {
  if (n == 0) return F3D_OK;
  const int64_t n2 = pow2_at_least(n, 2048);
  int rc = reserve(kv, static_cast<size_t>(n2) * sizeof(uint64_t));
  if (rc) return rc;
  keys_kernel<<<blocks(n2), 256, 0, st>>>(x, n, n2, h->geo.lo[0], h->geo.lo[1], h->geo.lo[2],
                                          256.0 / h->geo.width, as<uint64_t>(kv));
  if ((rc = launch_status())) return rc;
  return sort_u64(as<uint64_t>(kv), n2, st);
}

// dense table of `nkeys` entries from the flags already set in flags: the
// table (slot or -1) and the slot -> key list; returns the slot count
int finish_table(f3d_fmm *h, int64_t nkeys, DevBuf &table, DevBuf &keys, int *count, cudaStream_t st) {
  int rc = reserve(table, static_cast<size_t>(nkeys) * sizeof(int));
  if (rc) return rc;
  // the scan runs on the table buffer; flags keeps the 0/1 marks
  if (cudaMemcpyAsync(table.p, h->flags.p, static_cast<size_t>(nkeys) * sizeof(int), cudaMemcpyDeviceToDevice,
                      st) != cudaSuccess)
    return F3D_ERR_CUDA;
  if ((rc = scan_exclusive(as<int>(table), nkeys, as<int>(h->tile_sums), as<int>(h->scalars), st))) return rc;
  if ((rc = sync_read(count, h->scalars.p, sizeof(int), st))) return rc;
  if ((rc = reserve(keys, static_cast<size_t>(std::max(*count, 1)) * sizeof(int)))) return rc;
  finish_table_kernel<<<blocks(nkeys), 256, 0, st>>>(as<int>(h->flags), as<int>(table), nkeys, as<int>(keys));
  return launch_status();
}

int build_tree(f3d_fmm *h, cudaStream_t st) {
  int rc;
  // depth: the smallest with at most max_pts sources per non-empty leaf
  if ((rc = reserve(h->scalars, 64 * sizeof(int)))) return rc;
  if (cudaMemsetAsync(h->scalars.p, 0, 64 * sizeof(int), st) != cudaSuccess) return F3D_ERR_CUDA;
  unsigned *cnt = as<unsigned>(h->scalars) + 16;
  if (h->nsl) count_levels_kernel<<<blocks(h->nsl), 256, 0, st>>>(as<uint64_t>(h->kv_sl), h->nsl, cnt);
  if (h->ndl) count_levels_kernel<<<blocks(h->ndl), 256, 0, st>>>(as<uint64_t>(h->kv_dl), h->ndl, cnt);
  if ((rc = launch_status())) return rc;
  unsigned counts[16];
  if ((rc = sync_read(counts, cnt, sizeof(counts), st))) return rc;
  const int64_t nsrc = h->nsl + h->ndl;
  h->depth = kMaxDepth;
  for (int d = 2; d <= kMaxDepth; ++d) {
    if (counts[d] > 0 && nsrc <= static_cast<int64_t>(h->max_pts) * counts[d]) {
      h->depth = d;
      break;
    }
  }
  const int L = h->depth;
  const int shift = 3 * (kMaxDepth - L);
  if ((rc = reserve(h->tile_sums, kScanTile * sizeof(int)))) return rc;
  // leaves: sources and targets
  for (int side = 0; side < 2; ++side) {
    const int64_t nk = int64_t(1) << (3 * L);
    if ((rc = reserve(h->flags, static_cast<size_t>(nk) * sizeof(int)))) return rc;
    if (cudaMemsetAsync(h->flags.p, 0, static_cast<size_t>(nk) * sizeof(int), st) != cudaSuccess) return F3D_ERR_CUDA;
    if (side == 0) {
      if (h->nsl) flag_points_kernel<<<blocks(h->nsl), 256, 0, st>>>(as<uint64_t>(h->kv_sl), h->nsl, shift, as<int>(h->flags));
      if (h->ndl) flag_points_kernel<<<blocks(h->ndl), 256, 0, st>>>(as<uint64_t>(h->kv_dl), h->ndl, shift, as<int>(h->flags));
    } else {
      flag_points_kernel<<<blocks(h->ntrg), 256, 0, st>>>(as<uint64_t>(h->kv_trg), h->ntrg, shift, as<int>(h->flags));
    }
    if ((rc = launch_status())) return rc;
    Level &lv = h->lev[L];
    int count = 0;
    if ((rc = finish_table(h, nk, side == 0 ? lv.src_table : lv.trg_table, side == 0 ? lv.src_keys : lv.trg_keys,
                           &count, st)))
      return rc;
    (side == 0 ? lv.nsrc : lv.ntrg) = count;
  }
  // leaf point ranges
  Level &leaf = h->lev[L];
  const size_t rs = static_cast<size_t>(std::max(leaf.nsrc, 1)) * sizeof(int64_t);
  const size_t rt = static_cast<size_t>(std::max(leaf.ntrg, 1)) * sizeof(int64_t);
  if ((rc = reserve(h->sl_start, rs)) || (rc = reserve(h->sl_end, rs)) || (rc = reserve(h->dl_start, rs)) ||
      (rc = reserve(h->dl_end, rs)) || (rc = reserve(h->trg_start, rt)) || (rc = reserve(h->trg_end, rt)))
    return rc;
  for (DevBuf *b : {&h->sl_start, &h->sl_end, &h->dl_start, &h->dl_end})
    if (cudaMemsetAsync(b->p, 0, rs, st) != cudaSuccess) return F3D_ERR_CUDA;
  for (DevBuf *b : {&h->trg_start, &h->trg_end})
    if (cudaMemsetAsync(b->p, 0, rt, st) != cudaSuccess) return F3D_ERR_CUDA;
  if (h->nsl)
    leaf_ranges_kernel<<<blocks(h->nsl), 256, 0, st>>>(as<uint64_t>(h->kv_sl), h->nsl, shift, as<int>(leaf.src_table),
                                                       as<int64_t>(h->sl_start), as<int64_t>(h->sl_end));
  if (h->ndl)
    leaf_ranges_kernel<<<blocks(h->ndl), 256, 0, st>>>(as<uint64_t>(h->kv_dl), h->ndl, shift, as<int>(leaf.src_table),
                                                       as<int64_t>(h->dl_start), as<int64_t>(h->dl_end));
  leaf_ranges_kernel<<<blocks(h->ntrg), 256, 0, st>>>(as<uint64_t>(h->kv_trg), h->ntrg, shift, as<int>(leaf.trg_table),
                                                      as<int64_t>(h->trg_start), as<int64_t>(h->trg_end));
  if ((rc = launch_status())) return rc;
  // upper levels: parents of the boxes below
  for (int l = L - 1; l >= 2; --l) {
    const int64_t nk = int64_t(1) << (3 * l);
    for (int side = 0; side < 2; ++side) {
      if (cudaMemsetAsync(h->flags.p, 0, static_cast<size_t>(nk) * sizeof(int), st) != cudaSuccess)
        return F3D_ERR_CUDA;
      Level &below = h->lev[l + 1];
      const int nb = side == 0 ? below.nsrc : below.ntrg;
      if (nb > 0)
        flag_parents_kernel<<<blocks(nb), 256, 0, st>>>(as<int>(side == 0 ? below.src_keys : below.trg_keys), nb,
                                                        as<int>(h->flags));
      if ((rc = launch_status())) return rc;
      Level &lv = h->lev[l];
      int count = 0;
      if ((rc = finish_table(h, nk, side == 0 ? lv.src_table : lv.trg_table, side == 0 ? lv.src_keys : lv.trg_keys,
                             &count, st)))
        return rc;
      (side == 0 ? lv.nsrc : lv.ntrg) = count;
    }
  }
  // target boxes of each level grouped by octant (the columns of M2L / L2L)
  for (int l = 2; l <= L; ++l) {
    Level &lv = h->lev[l];
    if (lv.ntrg == 0) continue;
    const int64_t n2 = pow2_at_least(lv.ntrg, 2048);
    if ((rc = reserve(h->okv, static_cast<size_t>(n2) * sizeof(uint64_t)))) return rc;
    if ((rc = reserve(lv.trg_cols, static_cast<size_t>(lv.ntrg) * sizeof(int)))) return rc;
    unsigned *oc = as<unsigned>(h->scalars) + 32;
    if (cudaMemsetAsync(oc, 0, 8 * sizeof(unsigned), st) != cudaSuccess) return F3D_ERR_CUDA;
    octant_keys_kernel<<<blocks(n2), 256, 0, st>>>(as<int>(lv.trg_keys), lv.ntrg, n2, as<uint64_t>(h->okv), oc);
    if ((rc = launch_status())) return rc;
    if ((rc = sort_u64(as<uint64_t>(h->okv), n2, st))) return rc;
    low_words_kernel<<<blocks(lv.ntrg), 256, 0, st>>>(as<uint64_t>(h->okv), lv.ntrg, as<int>(lv.trg_cols));
    if ((rc = launch_status())) return rc;
    unsigned ocount[8];
    if ((rc = sync_read(ocount, oc, sizeof(ocount), st))) return rc;
    lv.oct_start[0] = 0;
    for (int c = 0; c < 8; ++c) lv.oct_start[c + 1] = lv.oct_start[c] + static_cast<int>(ocount[c]);
  }
  // the far-field work of this tree, for reports
  unsigned long long *pc = reinterpret_cast<unsigned long long *>(as<unsigned>(h->scalars) + 48);
  if (cudaMemsetAsync(pc, 0, sizeof(unsigned long long), st) != cudaSuccess) return F3D_ERR_CUDA;
  for (int l = 2; l <= L; ++l) {
    Level &lv = h->lev[l];
    if (lv.ntrg > 0)
      count_m2l_kernel<<<blocks(lv.ntrg), 256, 0, st>>>(as<int>(lv.trg_keys), lv.ntrg, as<int>(lv.src_table), l, pc);
  }
  if ((rc = launch_status())) return rc;
  unsigned long long pairs = 0;
  if ((rc = sync_read(&pairs, pc, sizeof(pairs), st))) return rc;
  h->m2l_pairs = static_cast<int64_t>(pairs);
  return F3D_OK;
}

// equivalent-density and check-potential storage for the current tree
int reserve_expansions(f3d_fmm *h) {
  int rc;
  const size_t n4 = 4 * static_cast<size_t>(h->n), n3 = 3 * static_cast<size_t>(h->n);
  size_t ymax = 1;
  for (int l = 2; l <= h->depth; ++l) {
    Level &lv = h->lev[l];
    if ((rc = reserve(lv.phi, std::max<size_t>(lv.nsrc, 1) * n4 * sizeof(double)))) return rc;
    if ((rc = reserve(lv.psi, std::max<size_t>(lv.ntrg, 1) * n4 * sizeof(double)))) return rc;
    ymax = std::max(ymax, static_cast<size_t>(std::max(lv.nsrc, lv.ntrg)));
  }
  return reserve(h->ybuf, ymax * n3 * sizeof(double));
}

// Launches a gathered GEMM over all its column groups.  Columns without
// groups (not M2L) form one group.  The terms are split over grid.z so that
// the launch fills the GPU at least twice over (capped at 32 splits and at
// 256 MiB of partial sums); the splits' partials are then added in order.
int launch_gemm(GemmOp op, const int *group_start, DevBuf &partial, cudaStream_t st, int *launches) {
  if (op.ncols <= 0) return F3D_OK;
  int tiles = 0;
  op.oct_tile_start[0] = 0;
  for (int c = 0; c < 8; ++c) {
    const int c0 = group_start ? group_start[c] : (c == 0 ? 0 : op.ncols);
    const int c1 = group_start ? group_start[c + 1] : op.ncols;
    op.oct_col_start[c] = c0;
    tiles += (c1 - c0 + GBN - 1) / GBN;
    op.oct_tile_start[c + 1] = tiles;
  }
  op.oct_col_start[8] = group_start ? group_start[8] : op.ncols;
  if (tiles > 65535) return F3D_ERR_TOO_LARGE;  // more boxes in a level than one launch covers
  const int rtiles = (op.rows + GBM - 1) / GBM;
  const int64_t want = 4 * static_cast<int64_t>(sm_count());
  int nsplit = static_cast<int>(std::min<int64_t>({(want + int64_t(rtiles) * tiles - 1) / (int64_t(rtiles) * tiles),
                                                   int64_t(op.nterms), int64_t(32)}));
  const size_t per_split = static_cast<size_t>(op.nslots) * op.ldy * sizeof(double);
  nsplit = std::max(1, std::min<int>(nsplit, static_cast<int>((size_t(256) << 20) / std::max<size_t>(per_split, 1))));
  op.nsplit = nsplit;
  if (nsplit > 1) {
    int rc = reserve(partial, nsplit * per_split);
    if (rc) return rc;
    op.partial = as<double>(partial);
  }
  const dim3 grid(static_cast<unsigned>(rtiles), static_cast<unsigned>(tiles), static_cast<unsigned>(nsplit));
  fmm_gemm_kernel<<<grid, GTHREADS, 0, st>>>(op);
  ++*launches;
  if (nsplit > 1) {
    const int64_t ne = static_cast<int64_t>(op.nslots) * op.rows;
    split_sum_kernel<<<blocks(ne), 256, 0, st>>>(op.partial, nsplit, op.nslots, op.ldy, op.rows, op.scale,
                                                 op.accumulate, op.Y);
    ++*launches;
  }
  return launch_status();
}

GemmOp stored_op(const double *A, int rows, int K, const double *X, int ldx, double *Y, int ldy, int ncols,
                 double scale) {
  GemmOp op{};
  op.mode = GEN_STORED;
  op.A = A;
  op.lda = K;
  op.K = K;
  op.rows = rows;
  op.X = X;
  op.ldx = ldx;
  op.Y = Y;
  op.ldy = ldy;
  op.ncols = ncols;
  op.nslots = ncols;
  op.scale = scale;
  op.nterms = 1;
  return op;
}

}  // namespace

extern "C" {

int f3d_fmm_create(int order, int max_pts, const double *surface, const double *uc2ue, const double *dc2de,
                   f3d_fmm **out) {
  if (!out || !surface || !uc2ue || !dc2de) return F3D_ERR_NULL;
  *out = nullptr;
  if (order < 4 || order > 16 || (order & 1) || max_pts < 1) return F3D_ERR_ARG;
  f3d_fmm *h = new f3d_fmm();
  h->p = order;
  h->n = 6 * (order - 1) * (order - 1) + 2;
  h->max_pts = max_pts;
  const size_t n = static_cast<size_t>(h->n);
  int rc;
  if ((rc = reserve(h->surf, 3 * n * sizeof(double))) || (rc = reserve(h->uc2ue, 12 * n * n * sizeof(double))) ||
      (rc = reserve(h->dc2de, 12 * n * n * sizeof(double)))) {
    delete h;
    return rc;
  }
  if (cudaMemcpy(h->surf.p, surface, 3 * n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->uc2ue.p, uc2ue, 12 * n * n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->dc2de.p, dc2de, 12 * n * n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete h;
    return F3D_ERR_CUDA;
  }
  *out = h;
  return F3D_OK;
}

int f3d_fmm_destroy(f3d_fmm *h) {
  if (!h) return F3D_OK;
  auto release = [](DevBuf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
  };
  for (DevBuf *b : {&h->surf, &h->uc2ue, &h->dc2de, &h->kv_sl, &h->kv_dl, &h->kv_trg, &h->x_sl, &h->x_dl, &h->x_trg,
                    &h->f_sl, &h->d_dl, &h->dl_tmp, &h->sl_start, &h->sl_end, &h->dl_start, &h->dl_end,
                    &h->trg_start, &h->trg_end, &h->flags, &h->tile_sums, &h->scalars, &h->okv, &h->ybuf,
                    &h->out_sorted, &h->bbox, &h->split_partial})
    release(*b);
  for (Level &lv : h->lev)
    for (DevBuf *b : {&lv.src_table, &lv.trg_table, &lv.src_keys, &lv.trg_keys, &lv.trg_cols, &lv.phi, &lv.psi})
      release(*b);
  delete h;
  return F3D_OK;
}

int f3d_fmm_set_box(f3d_fmm *h, const double *lo, double width) {
  if (!h || !lo) return F3D_ERR_NULL;
  if (!(width > 0.0) || !std::isfinite(width)) return F3D_ERR_ARG;
  for (int d = 0; d < 3; ++d) {
    if (!std::isfinite(lo[d])) return F3D_ERR_ARG;
    h->geo.lo[d] = lo[d];
  }
  h->geo.width = width;
  h->box_set = true;
  return F3D_OK;
}

int f3d_fmm_set_points(f3d_fmm *h, int64_t nsl, const double *src_sl, int64_t ndl, const double *src_dl,
                       int64_t ntrg, const double *trg, void *stream) {
  if (!h) return F3D_ERR_NULL;
  if (nsl < 0 || ndl < 0 || ntrg < 0) return F3D_ERR_SHAPE;
  if (nsl > INT32_MAX || ndl > INT32_MAX || ntrg > INT32_MAX) return F3D_ERR_TOO_LARGE;
  if ((nsl && !src_sl) || (ndl && !src_dl) || (ntrg && !trg)) return F3D_ERR_NULL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  h->nsl = nsl;
  h->ndl = ndl;
  h->ntrg = ntrg;
  h->depth = 0;
  int rc;
  if (ntrg == 0 || nsl + ndl == 0) return F3D_OK;
  if (!h->box_set) {
    // bounding cube of every point, 10 % margin on each side (kernels.py:1339-1348)
    const int nb = 64;
    if ((rc = reserve(h->bbox, 6 * nb * sizeof(double)))) return rc;
    bbox_kernel<<<nb, 256, 0, st>>>(src_sl, nsl, src_dl, ndl, trg, ntrg, as<double>(h->bbox));
    if ((rc = launch_status())) return rc;
    std::vector<double> part(6 * nb);
    if ((rc = sync_read(part.data(), h->bbox.p, part.size() * sizeof(double), st))) return rc;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = 0; b < nb; ++b)
      for (int d = 0; d < 3; ++d) {
        mn[d] = std::min(mn[d], part[6 * b + d]);
        mx[d] = std::max(mx[d], part[6 * b + 3 + d]);
      }
    double w = 0.0;
    for (int d = 0; d < 3; ++d) {
      if (!std::isfinite(mn[d]) || !std::isfinite(mx[d])) return F3D_ERR_NONFINITE;
      w = std::max(w, mx[d] - mn[d]);
    }
    if (w == 0.0) w = 1.0;
    for (int d = 0; d < 3; ++d) h->geo.lo[d] = mn[d] - 0.1 * w;
    h->geo.width = 1.2 * w;
  }
  if ((rc = sort_points(h, src_sl, nsl, h->kv_sl, st)) || (rc = sort_points(h, src_dl, ndl, h->kv_dl, st)) ||
      (rc = sort_points(h, trg, ntrg, h->kv_trg, st)))
    return rc;
  // sorted coordinates
  if ((rc = reserve(h->x_sl, std::max<size_t>(nsl, 1) * 3 * sizeof(double))) ||
      (rc = reserve(h->x_dl, std::max<size_t>(ndl, 1) * 3 * sizeof(double))) ||
      (rc = reserve(h->x_trg, std::max<size_t>(ntrg, 1) * 3 * sizeof(double))))
    return rc;
  if (nsl) gather_kernel<<<blocks(3 * nsl), 256, 0, st>>>(src_sl, as<uint64_t>(h->kv_sl), nsl, 3, as<double>(h->x_sl));
  if (ndl) gather_kernel<<<blocks(3 * ndl), 256, 0, st>>>(src_dl, as<uint64_t>(h->kv_dl), ndl, 3, as<double>(h->x_dl));
  gather_kernel<<<blocks(3 * ntrg), 256, 0, st>>>(trg, as<uint64_t>(h->kv_trg), ntrg, 3, as<double>(h->x_trg));
  if ((rc = launch_status())) return rc;
  if ((rc = build_tree(h, st))) return rc;
  return reserve_expansions(h);
}

int f3d_fmm_evaluate(f3d_fmm *h, const double *sl_density, const double *dl_normal, const double *dl_density,
                     const double *dl_tensor, double *out, double eta, void *stream) {
  if (!h) return F3D_ERR_NULL;
  if (!(eta > 0.0)) return F3D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nsl = h->nsl, ndl = h->ndl, ntrg = h->ntrg;
  if (ntrg == 0) return F3D_OK;
  if (!out) return F3D_ERR_NULL;
  if (nsl && !sl_density) return F3D_ERR_NULL;
  if (ndl && !dl_tensor && (!dl_normal || !dl_density)) return F3D_ERR_NULL;
  if (nsl + ndl == 0) {
    return cudaMemsetAsync(out, 0, static_cast<size_t>(ntrg) * 3 * sizeof(double), st) == cudaSuccess ? F3D_OK
                                                                                                     : F3D_ERR_CUDA;
  }
  if (h->depth < 2) return F3D_ERR_ARG;  // set_points has not run for these points
  int rc;
  const int n = h->n, n3 = 3 * n, n4 = 4 * n, L = h->depth;
  // densities in sorted order
  if ((rc = reserve(h->f_sl, std::max<size_t>(nsl, 1) * 3 * sizeof(double))) ||
      (rc = reserve(h->d_dl, std::max<size_t>(ndl, 1) * 9 * sizeof(double))) ||
      (rc = reserve(h->out_sorted, static_cast<size_t>(ntrg) * 3 * sizeof(double))))
    return rc;
  h->launches = 0;
  if (nsl) {
    gather_kernel<<<blocks(3 * nsl), 256, 0, st>>>(sl_density, as<uint64_t>(h->kv_sl), nsl, 3, as<double>(h->f_sl));
    ++h->launches;
  }
  if (ndl) {
    const double *D = dl_tensor;
    if (!D) {
      if ((rc = reserve(h->dl_tmp, static_cast<size_t>(ndl) * 9 * sizeof(double)))) return rc;
      dl_tensor_kernel<<<blocks(9 * ndl), 256, 0, st>>>(dl_normal, dl_density, ndl, as<double>(h->dl_tmp));
      ++h->launches;
      D = as<double>(h->dl_tmp);
    }
    gather_kernel<<<blocks(9 * ndl), 256, 0, st>>>(D, as<uint64_t>(h->kv_dl), ndl, 9, as<double>(h->d_dl));
    ++h->launches;
  }
  if ((rc = launch_status())) return rc;
  SourceSet src{};
  src.xsl = as<double>(h->x_sl);
  src.fsl = as<double>(h->f_sl);
  src.xdl = as<double>(h->x_dl);
  src.ddl = as<double>(h->d_dl);
  src.sl_start = as<int64_t>(h->sl_start);
  src.sl_end = as<int64_t>(h->sl_end);
  src.dl_start = as<int64_t>(h->dl_start);
  src.dl_end = as<int64_t>(h->dl_end);
  const double *surf = as<double>(h->surf);
  double *Y = as<double>(h->ybuf);
  // upward pass: leaf check potentials, then equivalent densities
  Level &leaf = h->lev[L];
  DevBuf &part = h->split_partial;
  {
    const dim3 grid(static_cast<unsigned>(leaf.nsrc), static_cast<unsigned>((n + 127) / 128));
    p2m_check_kernel<<<grid, 128, 0, st>>>(h->geo, L, as<int>(leaf.src_keys), src, surf, n, Y);
    ++h->launches;
    const double hL = h->geo.width / static_cast<double>(2 << L);
    if ((rc = launch_status()) ||
        (rc = launch_gemm(stored_op(as<double>(h->uc2ue), n4, n3, Y, n3, as<double>(leaf.phi), n4, leaf.nsrc, hL),
                          nullptr, part, st, &h->launches)))
      return rc;
  }
  for (int l = L - 1; l >= 2; --l) {
    Level &lv = h->lev[l], &below = h->lev[l + 1];
    if (lv.nsrc == 0) continue;
    GemmOp op{};
    op.mode = GEN_M2M;
    op.rows = n3;
    op.K = n4;
    op.surf = surf;
    op.n = n;
    op.crad = kRout;
    op.nterms = 8;
    op.table = as<int>(below.src_table);
    op.box_keys = as<int>(lv.src_keys);
    op.level = l;
    op.X = as<double>(below.phi);
    op.ldx = n4;
    op.Y = Y;
    op.ldy = n3;
    op.ncols = lv.nsrc;
    op.nslots = lv.nsrc;
    op.scale = 1.0;
    if ((rc = launch_gemm(op, nullptr, part, st, &h->launches)) ||
        (rc = launch_gemm(stored_op(as<double>(h->uc2ue), n4, n3, Y, n3, as<double>(lv.phi), n4, lv.nsrc, 1.0),
                          nullptr, part, st, &h->launches)))
      return rc;
  }
  // downward pass: the interaction lists and the parent's local expansion
  // in one launch per level, then the equivalent densities
  for (int l = 2; l <= L; ++l) {
    Level &lv = h->lev[l];
    if (lv.ntrg == 0) continue;
    GemmOp op{};
    op.mode = GEN_M2L;
    op.rows = n3;
    op.K = n4;
    op.surf = surf;
    op.n = n;
    op.crad = kRin;
    op.table = as<int>(lv.src_table);
    op.box_keys = as<int>(lv.trg_keys);
    op.level = l;
    op.X = as<double>(lv.phi);
    op.ldx = n4;
    op.Y = Y;
    op.ldy = n3;
    op.cols = as<int>(lv.trg_cols);
    op.ncols = lv.ntrg;
    op.nslots = lv.ntrg;
    op.scale = 1.0;
    op.accumulate = 0;
    for (int c = 0; c < 8; ++c) {
      const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;
      int t = 0;
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b)
          for (int d = 0; d < 6; ++d) {
            const int ox = a - 2 - cx, oy = b - 2 - cy, oz = d - 2 - cz;
            if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) < 2) continue;
            op.m2l_idx[c][t++] = static_cast<unsigned char>(36 * a + 6 * b + d);
          }
      if (t != kM2LTerms) return F3D_ERR_ARG;
    }
    op.nterms = kM2LTerms;
    const int *groups = lv.oct_start;
    if (l == 2) {
      // every level-1 box neighbours every other: the interaction list of a
      // level-2 box is every box at distance >= 2, whatever its octant
      int t = 0;
      for (int a = 0; a < 7; ++a)
        for (int b = 0; b < 7; ++b)
          for (int d = 0; d < 7; ++d)
            if (std::max(std::abs(a - 3), std::max(std::abs(b - 3), std::abs(d - 3))) >= 2)
              op.far_idx[t++] = static_cast<unsigned short>(49 * a + 7 * b + d);
      if (t != kFarTerms) return F3D_ERR_ARG;
      op.all_offsets = 1;
      op.nterms = kFarTerms;
      groups = nullptr;
    }
    if (l > 2) {
      op.parent = 1;
      op.nterms = kM2LTerms + 1;
      op.table2 = as<int>(h->lev[l - 1].trg_table);
      op.X2 = as<double>(h->lev[l - 1].psi);
    }
    if ((rc = launch_gemm(op, groups, part, st, &h->launches)) ||
        (rc = launch_gemm(stored_op(as<double>(h->dc2de), n4, n3, Y, n3, as<double>(lv.psi), n4, lv.ntrg, 1.0),
                          nullptr, part, st, &h->launches)))
      return rc;
  }
  // near field and the local expansions at the targets
  NearArgs na{};
  na.g = h->geo;
  na.level = L;
  na.trg_keys = as<int>(leaf.trg_keys);
  na.trg_start = as<int64_t>(h->trg_start);
  na.trg_end = as<int64_t>(h->trg_end);
  na.xt = as<double>(h->x_trg);
  na.src_table = as<int>(leaf.src_table);
  na.src = src;
  na.psi = as<double>(leaf.psi);
  na.surf = surf;
  na.n = n;
  na.out = as<double>(h->out_sorted);
  near_l2p_kernel<<<static_cast<unsigned>(leaf.ntrg), 128, 0, st>>>(na);
  h->launches += 2;  // with the scatter below
  scatter_kernel<<<blocks(3 * ntrg), 256, 0, st>>>(as<double>(h->out_sorted), as<uint64_t>(h->kv_trg), ntrg,
                                                   1.0 / eta, out);
  return launch_status();
}

int f3d_fmm_last_launches(const f3d_fmm *h, int *launches) {
  if (!h || !launches) return F3D_ERR_NULL;
  *launches = h->launches;
  return F3D_OK;
}

int f3d_fmm_tree_info(const f3d_fmm *h, int *depth, int64_t *src_leaves, int64_t *trg_leaves, double *box,
                      int64_t *m2l_pairs) {
  if (!h || !depth) return F3D_ERR_NULL;
  *depth = h->depth;
  if (m2l_pairs) *m2l_pairs = h->depth ? h->m2l_pairs : 0;
  if (src_leaves) *src_leaves = h->depth ? h->lev[h->depth].nsrc : 0;
  if (trg_leaves) *trg_leaves = h->depth ? h->lev[h->depth].ntrg : 0;
  if (box) {
    for (int d = 0; d < 3; ++d) box[d] = h->geo.lo[d];
    box[3] = h->geo.width;
  }
  return F3D_OK;
}

}  // extern "C"
