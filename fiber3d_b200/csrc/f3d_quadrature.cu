// RBF quadrature weights of a smooth closed surface: fiber3d's
// Smooth_Closed_Surface_Quadrature_RBF with the exact surface gradient
// (python/quadratures/Smooth_Closed_Surface_Quadrature_RBF.py:3-470; the
// method of Reeger, Fornberg & Watts, Proc. R. Soc. A 472 (2016)), the
// periphery's and bodies' set-up step (tstep/tstep.py:297-300,
// body/body.py:104-107).
//
// The reference loops over triangles in Python (about 5 ms each).  Here the
// whole computation is eight kernels on one stream:
//   1. quad_prep: per triangle, sorted vertices, unit normal and midpoint;
//      its three edges go into a device hash table (key = i * n + j).
//   2. quad_edges: per triangle edge, the partner triangle from the table and
//      the edge normal, the average of the two triangles' normals (:118-127).
//   3. quad_knn: per triangle, the 80 nodes nearest its midpoint (:114-115),
//      an exact radix select over the float-rounded squared distances held
//      in shared memory, ties resolved on the double distances, then index.
//      The nodes go in tiles of 24576, the best 80 carried from tile to tile.
//   4. quad_triangle: per triangle, the projection onto the triangle's plane
//      (:162-236), the exact integrals of r^7 (:262-309) and of the degree-7
//      monomials (:473-622, here by Gauss-Legendre on Green's-theorem line
//      integrals) and the 116 x 116 saddle-point solve (:334-336),
//      Gauss-Jordan elimination with partial pivoting held in registers
//      (16 x 16 threads, an 8 x 8 tile each), the right-hand side carried
//      along as column 116; then the area-element distortion (:431-447).
//   5. quad_count / quad_scan / quad_fill / quad_sum: the per-node sum of the
//      triangle weights in triangle order (:460-468), deterministic.
#include <algorithm>

#include "f3d_common.cuh"

namespace f3d {

// Node coordinates are addressed as 3 * node in 32-bit int arithmetic, so a
// surface has at most INT32_MAX / 3 nodes.
constexpr int64_t kQuadMaxNodes = 0x7fffffffLL / 3;

constexpr int kQuadNbr = 80;                 // nearest neighbours (n in the paper)
constexpr int kQuadOrder = 7;                // polynomial degree (m)
constexpr int kQuadPoly = 36;                // (m + 1)(m + 2) / 2
constexpr int kQuadDim = kQuadNbr + kQuadPoly;  // 116
constexpr int kQuadRhsCol = kQuadDim;        // column 116 holds the right-hand side
constexpr int kKnnThreads = 256;
constexpr int kKnnBins = 2048;
constexpr int kKnnCand = 256;
constexpr int kKnnTile = 24576;             // nodes per k-NN pass (squared distances in shared memory)
constexpr double kEpsMult = 1e-4;
constexpr double kDblEps = 2.220446049250313e-16;

// 6-point Gauss-Legendre on [-1, 1] (exact to degree 11).
__constant__ double kGlX[6] = {-0.9324695142031520278123016, -0.6612093864662645136613996,
                               -0.2386191860831969086305017, 0.2386191860831969086305017,
                               0.6612093864662645136613996,  0.9324695142031520278123016};
__constant__ double kGlW[6] = {0.1713244923791703450402961, 0.3607615730481386075698335,
                               0.4679139345726910473898703, 0.4679139345726910473898703,
                               0.3607615730481386075698335, 0.1713244923791703450402961};

struct QuadWs {
  int32_t *tri;     // ntri x 3, sorted vertex indices
  double *tnorm;    // ntri x 3
  double *mid;      // ntri x 3
  double *enorm;    // ntri x 9: edges (i0,i1), (i0,i2), (i1,i2)
  long long *hkey;  // hash keys (-1 empty)
  int32_t *hid;     // 2 per key: stacked edge ids (-1 empty)
  int32_t *nni;     // ntri x 80
  double *wt;       // ntri x 80
  int32_t *count;   // n + 1 (exclusive offsets after the scan)
  int32_t *cursor;  // n
  int32_t *entry;   // ntri x 80
  int hbits;
};

__device__ __forceinline__ unsigned hash_slot(long long key, int hbits) {
  return static_cast<unsigned>((static_cast<unsigned long long>(key) * 0x9E3779B97F4A7C15ull) >> (64 - hbits));
}

__device__ __forceinline__ double dot3_rn(const double *a, const double *b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}

__device__ __forceinline__ void cross_rn(const double *a, const double *b, double *c) {
  c[0] = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(a[2], b[1]));
  c[1] = __dsub_rn(__dmul_rn(a[2], b[0]), __dmul_rn(a[0], b[2]));
  c[2] = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(a[1], b[0]));
}

// ---------------------------------------------------------------- 1. prep --
__global__ void quad_prep_kernel(const double *__restrict__ X, int n, const int32_t *__restrict__ tri_in,
                                 int ntri, QuadWs w, int *err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  int i0 = tri_in[3 * t], i1 = tri_in[3 * t + 1], i2 = tri_in[3 * t + 2];
  if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= n || i1 >= n || i2 >= n) {
    record_error(err, F3D_ERR_ARG);
    i0 = 0, i1 = 0, i2 = 0;
  }
  if (i0 > i1) { const int s = i0; i0 = i1; i1 = s; }
  if (i1 > i2) { const int s = i1; i1 = i2; i2 = s; }
  if (i0 > i1) { const int s = i0; i0 = i1; i1 = s; }
  if (i0 == i1 || i1 == i2) record_error(err, F3D_ERR_ARG);
  w.tri[3 * t] = i0, w.tri[3 * t + 1] = i1, w.tri[3 * t + 2] = i2;
  double v1[3], v2[3], nrm[3];
  for (int c = 0; c < 3; ++c) {
    v1[c] = __dsub_rn(X[3 * i1 + c], X[3 * i0 + c]);
    v2[c] = __dsub_rn(X[3 * i2 + c], X[3 * i0 + c]);
  }
  // (V1 x V2) in the reference's component order (:111)
  nrm[0] = __dsub_rn(__dmul_rn(v1[1], v2[2]), __dmul_rn(v2[1], v1[2]));
  nrm[1] = __dsub_rn(__dmul_rn(v2[0], v1[2]), __dmul_rn(v1[0], v2[2]));
  nrm[2] = __dsub_rn(__dmul_rn(v1[0], v2[1]), __dmul_rn(v2[0], v1[1]));
  const double nn = __dsqrt_rn(dot3_rn(nrm, nrm));
  for (int c = 0; c < 3; ++c) {
    w.tnorm[3 * t + c] = __ddiv_rn(nrm[c], nn);
    w.mid[3 * t + c] = __ddiv_rn(__dadd_rn(__dadd_rn(X[3 * i0 + c], X[3 * i1 + c]), X[3 * i2 + c]), 3.0);
  }
  const int ea[3] = {i0, i0, i1}, eb[3] = {i1, i2, i2};
  const unsigned hmask = (1u << w.hbits) - 1u;
  for (int s = 0; s < 3; ++s) {
    const long long key = static_cast<long long>(ea[s]) * n + eb[s];
    const int id = s * ntri + t;
    unsigned slot = hash_slot(key, w.hbits);
    bool placed = false;
    for (unsigned probe = 0; probe <= hmask; ++probe) {
      const long long prev = static_cast<long long>(atomicCAS(reinterpret_cast<unsigned long long *>(w.hkey + slot),
                                                              ~0ull, static_cast<unsigned long long>(key)));
      if (prev == -1 || prev == key) {
        if (atomicCAS(w.hid + 2 * slot, -1, id) != -1 && atomicCAS(w.hid + 2 * slot + 1, -1, id) != -1)
          record_error(err, F3D_ERR_ARG);  // an edge shared by more than two triangles
        placed = true;
        break;
      }
      slot = (slot + 1) & hmask;
    }
    if (!placed) record_error(err, F3D_ERR_ARG);
  }
}

// --------------------------------------------------------------- 2. edges --
__global__ void quad_edges_kernel(int n, int ntri, QuadWs w, int *err) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= 3 * ntri) return;
  const int t = g / 3, s = g % 3;
  const int i0 = w.tri[3 * t], i1 = w.tri[3 * t + 1], i2 = w.tri[3 * t + 2];
  const int a = s == 2 ? i1 : i0, b = s == 0 ? i1 : i2;
  const long long key = static_cast<long long>(a) * n + b;
  const int id = s * ntri + t;
  const unsigned hmask = (1u << w.hbits) - 1u;
  unsigned slot = hash_slot(key, w.hbits);
  int other = -1;
  for (unsigned probe = 0; probe <= hmask; ++probe) {
    const long long k = w.hkey[slot];
    if (k == key) {
      const int p = w.hid[2 * slot], q = w.hid[2 * slot + 1];
      other = p == id ? q : (q == id ? p : -1);
      break;
    }
    if (k == -1) break;
    slot = (slot + 1) & hmask;
  }
  double e[3] = {0.0, 0.0, 0.0};
  if (other < 0) {
    record_error(err, F3D_ERR_ARG);  // an edge of only one triangle: the surface is not closed
  } else {
    // the first copy in the stacked edge order comes first in the average
    const int first = id < other ? id : other, second = id < other ? other : id;
    const double *na = w.tnorm + 3 * (first % ntri);
    const double *nb = w.tnorm + 3 * (second % ntri);
    const double d = dot3_rn(na, nb);
    const double sg = d > 0.0 ? 1.0 : (d < 0.0 ? -1.0 : 0.0);
    for (int c = 0; c < 3; ++c) e[c] = __ddiv_rn(__dadd_rn(na[c], __dmul_rn(sg, nb[c])), 2.0);
    const double en = __dsqrt_rn(dot3_rn(e, e));
    for (int c = 0; c < 3; ++c) e[c] = __ddiv_rn(e[c], en);
  }
  for (int c = 0; c < 3; ++c) w.enorm[9 * t + 3 * s + c] = e[c];
}

// ----------------------------------------------------------------- 3. kNN --
__device__ __forceinline__ unsigned fkey(double d) { return __float_as_uint(__double2float_rn(d)); }

// The nodes are taken in tiles of `tile`: each tile's squared distances,
// together with the best 80 of the earlier tiles, go through the select, so
// a surface of any size fits the shared memory; a surface of at most `tile`
// nodes is one pass.
__global__ void __launch_bounds__(kKnnThreads) quad_knn_kernel(const double *__restrict__ X, int n,
                                                               const double *__restrict__ mid, int ntri, int tile,
                                                               int32_t *__restrict__ nni, int *err) {
  extern __shared__ __align__(16) unsigned char knn_smem[];
  double *dist = reinterpret_cast<double *>(knn_smem);     // tile + 80
  double *cd = dist + tile + kQuadNbr;                     // kKnnCand candidate distances
  int *cj = reinterpret_cast<int *>(cd + kKnnCand);        // kKnnCand candidate indices
  int *pj = cj + kKnnCand;                                 // 80: indices of the earlier tiles' best
  int *hist = pj + kQuadNbr;                               // kKnnBins
  __shared__ int s_part[kKnnThreads / 32];
  __shared__ int s_bin, s_below, s_ncand;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int t = blockIdx.x; t < ntri; t += gridDim.x) {
    const double q0 = mid[3 * t], q1 = mid[3 * t + 1], q2 = mid[3 * t + 2];
    int nprev = 0;
    for (int base = 0; base < n; base += tile) {
      const int tl = min(tile, n - base);
      for (int j = tid; j < tl; j += kKnnThreads) {
        const int g = base + j;
        const double dx = __dsub_rn(q0, X[3 * g]), dy = __dsub_rn(q1, X[3 * g + 1]), dz = __dsub_rn(q2, X[3 * g + 2]);
        dist[j] = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      }
      for (int p = tid; p < nprev; p += kKnnThreads) {
        dist[tl + p] = cd[p];
        pj[p] = cj[p];
      }
      const int m = tl + nprev;  // >= 80: the first tile has min(n, tile) >= 80 nodes
      __syncthreads();
      unsigned prefix = 0;
      int kk = kQuadNbr;  // rank (1-based) still to find among keys matching the prefix
      for (int pass = 0; pass < 3; ++pass) {
        const int shift = pass == 0 ? 21 : (pass == 1 ? 10 : 0), width = pass == 2 ? 10 : 11;
        for (int b = tid; b < kKnnBins; b += kKnnThreads) hist[b] = 0;
        __syncthreads();
        for (int pb = 0; pb < m; pb += kKnnThreads) {
          const int j = pb + tid;
          int bin = -1 - lane;  // distinct per lane when not counted
          if (j < m) {
            const unsigned key = fkey(dist[j]);
            if (pass == 0 || (key >> (shift + width)) == prefix)
              bin = static_cast<int>((key >> shift) & ((1u << width) - 1u));
          }
          const unsigned peers = __match_any_sync(0xffffffffu, bin);
          if (bin >= 0 && lane == __ffs(peers) - 1) atomicAdd(hist + bin, __popc(peers));
        }
        __syncthreads();
        // the bin where the running count reaches kk
        int local = 0;
        for (int b = 0; b < kKnnBins / kKnnThreads; ++b) local += hist[tid * (kKnnBins / kKnnThreads) + b];
        int incl = local;
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        if (lane == 31) s_part[warp] = incl;
        __syncthreads();
        int before = 0;
        for (int w2 = 0; w2 < warp; ++w2) before += s_part[w2];
        const int excl = before + incl - local;
        if (excl < kk && excl + local >= kk) {
          int c = excl;
          for (int b = 0; b < kKnnBins / kKnnThreads; ++b) {
            const int bin = tid * (kKnnBins / kKnnThreads) + b;
            if (c + hist[bin] >= kk) {
              s_bin = bin;
              s_below = c;
              break;
            }
            c += hist[bin];
          }
        }
        __syncthreads();
        prefix = (prefix << width) | static_cast<unsigned>(s_bin);
        kk -= s_below;
        __syncthreads();
      }
      // prefix is now the float key of the 80th smallest distance: every
      // node at or below it is a candidate (rounding to float is monotone)
      if (tid == 0) s_ncand = 0;
      __syncthreads();
      for (int j = tid; j < m; j += kKnnThreads) {
        if (fkey(dist[j]) <= prefix) {
          const int slot = atomicAdd(&s_ncand, 1);
          if (slot < kKnnCand) {
            cd[slot] = dist[j];
            cj[slot] = j < tl ? base + j : pj[j - tl];
          }
        }
      }
      __syncthreads();
      const int nc = s_ncand;
      if (nc > kKnnCand && tid == 0) record_error(err, F3D_ERR_TOO_LARGE);
      for (int c = nc + tid; c < kKnnCand; c += kKnnThreads) {
        cd[c] = __longlong_as_double(0x7ff0000000000000ll);
        cj[c] = 0x7fffffff;
      }
      __syncthreads();
      // bitonic sort of the candidates by (distance, index)
      for (int size = 2; size <= kKnnCand; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          const int i = tid, p = i ^ stride;
          if (p > i) {
            const bool up = (i & size) == 0;
            const double di = cd[i], dp = cd[p];
            const int ji = cj[i], jp = cj[p];
            const bool gt = di > dp || (di == dp && ji > jp);
            if (gt == up) {
              cd[i] = dp, cd[p] = di;
              cj[i] = jp, cj[p] = ji;
            }
          }
          __syncthreads();
        }
      }
      nprev = kQuadNbr;
    }
    if (tid < kQuadNbr) nni[static_cast<int64_t>(t) * kQuadNbr + tid] = cj[tid] < n ? cj[tid] : 0;
    __syncthreads();
  }
}

// ------------------------------------------------------------ 4. triangle --
// Integral of r^7 over the right triangle with legs alpha and beta (:302).
__device__ __forceinline__ double rbf_right_triangle(double a, double b) {
  const double a2 = a * a, b2 = b * b;
  return a * (b * sqrt(a2 + b2) * (279.0 * a2 * a2 * a2 + 326.0 * a2 * a2 * b2 + 200.0 * a2 * b2 * b2 + 48.0 * b2 * b2 * b2) +
              105.0 * (a2 * a2) * (a2 * a2) * asinh(b / a)) /
         3456.0;
}

__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

constexpr int kTriThreads = 256;

struct TriShared {
  double c[kQuadNbr][2];         // projected, shifted centres
  double pm[kQuadNbr][kQuadPoly];  // monomials of the centres
  double rhs[kQuadDim];
  double dist[kQuadNbr];
  double l[128];
  double u[128];
  double ys[128];
  double x[kQuadDim];
  double piv[kQuadDim];
  double recip[kQuadDim];
  int order[kQuadDim];
  int where[128];
  double xp[3], rot[9], shift[2], v[3][2], height;
  int prow;
};

// The pivot row's entries in register columns KB..7 go to S.u (u_j = 0 for
// j <= k in column block KB).
template <int KB>
__device__ __forceinline__ void stage_row(const double (&row)[8], TriShared &S, int tx, int k) {
  const int j = tx + 16 * KB;
  S.u[j] = j > k ? row[KB] : 0.0;
#pragma unroll
  for (int b = KB + 1; b < 8; ++b) S.u[tx + 16 * b] = row[b];
}

// Pivot of column k (register column C of the threads with tx == k % 16,
// one half-warp): the largest |a_ik| over the rows not yet pivoted (`used`:
// bit a for row ty + 16 a), the first in the current row order on ties
// (LAPACK's choice); its lane stores the pivot and its reciprocal, lane 0
// exchanges the rows.
template <int C>
__device__ __forceinline__ void pivot_column(const double (&M)[8][8], TriShared &S, unsigned used, int k, int ty,
                                             int tx, int *err) {
  const unsigned half = (tx & 1) ? 0xffff0000u : 0x0000ffffu;
  double best = -1.0, mine = 0.0;
  int ia = -1;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int i = ty + 16 * a;
    if (i < kQuadDim && !((used >> a) & 1u)) {
      const double av = fabs(M[a][C]);
      if (av > best || (av == best && S.where[i] < S.where[ty + 16 * ia])) best = av, ia = a, mine = M[a][C];
    }
  }
  int bpos = ia >= 0 ? S.where[ty + 16 * ia] : 0x7fffffff;
  const int my_pos = bpos;
  const double my_recip = 1.0 / mine;  // formed while the reduction runs
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(half, best, o, 16);
    const int op = __shfl_xor_sync(half, bpos, o, 16);
    if (ob > best || (ob == best && op < bpos)) best = ob, bpos = op;
  }
  if (my_pos == bpos && bpos != 0x7fffffff) {
    S.piv[k] = mine;
    S.recip[k] = my_recip;
  }
  __syncwarp(half);
  if (ty == 0) {
    if (!(best > 0.0)) {
      record_error(err, F3D_ERR_SINGULAR);
      bpos = k;
      S.piv[k] = 1.0;
      S.recip[k] = 1.0;
    }
    const int rk = S.order[k], rp = S.order[bpos];
    S.order[k] = rp, S.order[bpos] = rk;
    S.where[rp] = k, S.where[rk] = bpos;
    S.prow = rp;
  }
}

// Gauss-Jordan steps k = 16 KB .. 16 KB + ncol - 1 (the pivot of step k
// already chosen): every row but the pivot row loses l_i = a_ik / a_pk times
// the pivot row, so that after the last step row order[k] holds u_kk in
// column k and y_k in column 116, and x_k = y_k / u_kk (no back
// substitution).  Columns up to k are left as they are.  The pivot column is
// register column KB of the threads with tx == k % 16: a static index, so it
// never leaves registers; column blocks before KB are skipped.  After its own
// update, the half-warp that owns column k + 1 chooses that column's pivot
// while the other warps finish theirs.
template <int KB>
__device__ __forceinline__ void gj_columns(double (&M)[8][8], TriShared &S, unsigned &used, int ncol, int ty, int tx,
                                           int *err) {
  for (int kk = 0; kk < ncol; ++kk) {
    const int k = 16 * KB + kk;
    const int prow = S.prow;
    if (ty == (prow & 15)) used |= 1u << (prow >> 4);
    if (tx == kk) {
      const double r = S.recip[k];
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        const int i = ty + 16 * a;
        S.l[i] = (i < kQuadDim && i != prow) ? M[a][KB] * r : 0.0;
      }
    }
    if (ty == (prow & 15)) {
      switch (prow >> 4) {
        case 0: stage_row<KB>(M[0], S, tx, k); break;
        case 1: stage_row<KB>(M[1], S, tx, k); break;
        case 2: stage_row<KB>(M[2], S, tx, k); break;
        case 3: stage_row<KB>(M[3], S, tx, k); break;
        case 4: stage_row<KB>(M[4], S, tx, k); break;
        case 5: stage_row<KB>(M[5], S, tx, k); break;
        case 6: stage_row<KB>(M[6], S, tx, k); break;
        default: stage_row<KB>(M[7], S, tx, k); break;
      }
    }
    __syncthreads();
    double ur[8 - KB];
#pragma unroll
    for (int b = KB; b < 8; ++b) ur[b - KB] = S.u[tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double lr = -S.l[ty + 16 * a];
#pragma unroll
      for (int b = KB; b < 8; ++b) M[a][b] = fma(lr, ur[b - KB], M[a][b]);
    }
    if (k + 1 < kQuadDim) {
      if (kk + 1 < 16) {
        if (tx == kk + 1) pivot_column<KB>(M, S, used, k + 1, ty, tx, err);
      } else if constexpr (KB < 7) {
        if (tx == 0) pivot_column<KB + 1>(M, S, used, k + 1, ty, tx, err);
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kTriThreads, 1) quad_triangle_kernel(const double *__restrict__ X,
                                                                       const double *__restrict__ grad, int ntri,
                                                                       QuadWs w, int *err) {
  __shared__ TriShared S;
  const int tid = threadIdx.x;
  const int ty = tid & 15, tx = tid >> 4;  // rows ty + 16a, columns tx + 16b
  for (int t = blockIdx.x; t < ntri; t += gridDim.x) {
    const int *tv = w.tri + 3 * t;
    const double *nrm = w.tnorm + 3 * t;
    const int32_t *nb = w.nni + static_cast<int64_t>(t) * kQuadNbr;
    if (tid == 0) {
      // projection point (:162-201)
      double A[3], B[3], C[3], AB[3], BC[3], CA[3];
      for (int c = 0; c < 3; ++c) {
        A[c] = X[3 * tv[0] + c], B[c] = X[3 * tv[1] + c], C[c] = X[3 * tv[2] + c];
        AB[c] = __dsub_rn(B[c], A[c]), BC[c] = __dsub_rn(C[c], B[c]), CA[c] = __dsub_rn(A[c], C[c]);
      }
      const double *nAB = w.enorm + 9 * t, *nCA = nAB + 3, *nBC = nAB + 6;
      double nOAB[3], nOBC[3], nOCA[3], vOA[3];
      cross_rn(nAB, AB, nOAB);
      cross_rn(nBC, BC, nOBC);
      cross_rn(nCA, CA, nOCA);
      cross_rn(nOAB, nOCA, vOA);
      const double tA = __ddiv_rn(dot3_rn(nOBC, AB), dot3_rn(nOBC, vOA));
      for (int c = 0; c < 3; ++c) S.xp[c] = __dadd_rn(A[c], __dmul_rn(tA, vOA[c]));
      // rotation taking the normal to +z (:210-220)
      const double rxy = __dsqrt_rn(__dadd_rn(__dmul_rn(nrm[0], nrm[0]), __dmul_rn(nrm[1], nrm[1])));
      if (rxy < kDblEps) {
        for (int i = 0; i < 9; ++i) S.rot[i] = (i % 4 == 0) ? 1.0 : 0.0;
      } else {
        const double nn = __dsqrt_rn(dot3_rn(nrm, nrm));
        const double r1[9] = {__ddiv_rn(nrm[2], nn), 0.0, -__ddiv_rn(rxy, nn), 0.0, 1.0, 0.0,
                              __ddiv_rn(rxy, nn), 0.0, __ddiv_rn(nrm[2], nn)};
        const double r2[9] = {__ddiv_rn(nrm[0], rxy), __ddiv_rn(nrm[1], rxy), 0.0, -__ddiv_rn(nrm[1], rxy),
                              __ddiv_rn(nrm[0], rxy), 0.0, 0.0, 0.0, 1.0};
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            S.rot[3 * i + j] = __dadd_rn(__dadd_rn(__dmul_rn(r1[3 * i], r2[j]), __dmul_rn(r1[3 * i + 1], r2[3 + j])),
                                         __dmul_rn(r1[3 * i + 2], r2[6 + j]));
      }
      double d[3];
      for (int c = 0; c < 3; ++c) d[c] = __dsub_rn(w.mid[3 * t + c], S.xp[c]);
      S.shift[0] = dot3_rn(S.rot, d);
      S.shift[1] = dot3_rn(S.rot + 3, d);
      const double *V[3] = {A, B, C};
      for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) d[c] = __dsub_rn(V[r][c], S.xp[c]);
        S.v[r][0] = __dsub_rn(dot3_rn(S.rot, d), S.shift[0]);
        S.v[r][1] = __dsub_rn(dot3_rn(S.rot + 3, d), S.shift[1]);
      }
    }
    __syncthreads();
    if (tid < kQuadNbr) {
      // project neighbour tid into the plane (:225-236)
      const int j = nb[tid];
      double Q[3], d[3], p[3];
      for (int c = 0; c < 3; ++c) Q[c] = X[3 * j + c];
      const double A0 = X[3 * tv[0]], A1 = X[3 * tv[0] + 1], A2 = X[3 * tv[0] + 2];
      const double num = __dadd_rn(__dadd_rn(__dmul_rn(nrm[0], __dsub_rn(A0, Q[0])), __dmul_rn(nrm[1], __dsub_rn(A1, Q[1]))),
                                   __dmul_rn(nrm[2], __dsub_rn(A2, Q[2])));
      for (int c = 0; c < 3; ++c) d[c] = __dsub_rn(Q[c], S.xp[c]);
      const double mult = __ddiv_rn(num, dot3_rn(nrm, d));
      for (int c = 0; c < 3; ++c) p[c] = __dsub_rn(__dadd_rn(Q[c], __dmul_rn(mult, d[c])), S.xp[c]);
      const double u0 = dot3_rn(S.rot, p), u1 = dot3_rn(S.rot + 3, p), u2 = dot3_rn(S.rot + 6, p);
      if (tid == 0) S.height = u2;
      const double cx = __dsub_rn(u0, S.shift[0]), cy = __dsub_rn(u1, S.shift[1]);
      S.c[tid][0] = cx, S.c[tid][1] = cy;
      // monomials by the reference's recursion (:324-329)
      double *pm = S.pm[tid];
      pm[0] = 1.0;
      for (int dg = 1; dg <= kQuadOrder; ++dg)
        for (int k = 0; k <= dg; ++k)
          pm[dg * (dg + 1) / 2 + k] = (k >= (dg + 1) / 2) ? __dmul_rn(cy, pm[(dg - 1) * dg / 2 + k - 1])
                                                          : __dmul_rn(cx, pm[(dg - 1) * dg / 2 + k]);
      // area-element distortion (:431-442)
      const double *g = grad + 3 * j;
      const double gn = __dsqrt_rn(dot3_rn(g, g));
      const double nv = __dsqrt_rn(dot3_rn(d, d));
      double vh[3], ns[3];
      for (int c = 0; c < 3; ++c) vh[c] = __ddiv_rn(d[c], nv), ns[c] = __ddiv_rn(g[c], gn);
      const double pn = __dsqrt_rn(dot3_rn(nrm, nrm));
      double pu[3];
      for (int c = 0; c < 3; ++c) pu[c] = __ddiv_rn(nrm[c], pn);
      S.ys[tid] = __ddiv_rn(dot3_rn(pu, vh), dot3_rn(ns, vh));  // ratio of the normal projections
      S.l[tid] = nv;
    }
    __syncthreads();
    if (tid < kQuadNbr) {
      const double cx = __dadd_rn(S.c[tid][0], S.shift[0]), cy = __dadd_rn(S.c[tid][1], S.shift[1]);
      const double R = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(S.height, S.height)));
      const double rr = __ddiv_rn(S.l[tid], R);
      S.dist[tid] = fabs(__dmul_rn(S.ys[tid], __dmul_rn(rr, rr)));
      // exact integral of r^7 centred at this node over the triangle (:262-309)
      const double c0 = S.c[tid][0], c1 = S.c[tid][1];
      const double(*V)[2] = S.v;
      const double sabc = sgn(__dadd_rn(__dmul_rn(__dsub_rn(V[0][1], V[1][1]), __dsub_rn(V[2][0], V[0][0])),
                                        __dmul_rn(__dsub_rn(V[1][0], V[0][0]), __dsub_rn(V[2][1], V[0][1]))));
      double irbf = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double *p1 = V[s], *p2 = V[(s + 1) % 3];
        const double ex = __dsub_rn(p2[0], p1[0]), ey = __dsub_rn(p2[1], p1[1]);
        const double m = __ddiv_rn(__dadd_rn(__dmul_rn(__dsub_rn(c0, p1[0]), ex), __dmul_rn(__dsub_rn(c1, p1[1]), ey)),
                                   __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)));
        const double fx = __dadd_rn(__dmul_rn(m, ex), p1[0]), fy = __dadd_rn(__dmul_rn(m, ey), p1[1]);
        const double sg1 = sabc * sgn(__dadd_rn(__dmul_rn(__dsub_rn(c1, p1[1]), __dsub_rn(fx, c0)),
                                                __dmul_rn(__dsub_rn(p1[0], c0), __dsub_rn(fy, c1))));
        const double sg2 = sabc * sgn(__dadd_rn(__dmul_rn(__dsub_rn(c1, fy), __dsub_rn(p2[0], c0)),
                                                __dmul_rn(__dsub_rn(fx, c0), __dsub_rn(p2[1], c1))));
        const double ax = __dsub_rn(c0, fx), ay = __dsub_rn(c1, fy);
        const double alpha = __dsqrt_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)));
        const double b1x = __dsub_rn(fx, p1[0]), b1y = __dsub_rn(fy, p1[1]);
        const double b2x = __dsub_rn(fx, p2[0]), b2y = __dsub_rn(fy, p2[1]);
        const double beta1 = __dsqrt_rn(__dadd_rn(__dmul_rn(b1x, b1x), __dmul_rn(b1y, b1y)));
        const double beta2 = __dsqrt_rn(__dadd_rn(__dmul_rn(b2x, b2x), __dmul_rn(b2y, b2y)));
        const double tiny = kEpsMult * kDblEps;
        if (alpha > tiny && beta1 > tiny) irbf += sg1 * rbf_right_triangle(alpha, beta1);
        if (alpha > tiny && beta2 > tiny) irbf += sg2 * rbf_right_triangle(alpha, beta2);
      }
      S.rhs[tid] = irbf;
    } else if (tid < kQuadDim) {
      // polynomial moment m = tid - 80 of the triangle (Green's theorem,
      // Gauss-Legendre along each side)
      const int m = tid - kQuadNbr;
      int dg = 0;
      while ((dg + 1) * (dg + 2) / 2 <= m) ++dg;
      const int k = m - dg * (dg + 1) / 2, a = dg - k;
      const double(*V)[2] = S.v;
      const double sabc = sgn(__dadd_rn(__dmul_rn(__dsub_rn(V[0][1], V[1][1]), __dsub_rn(V[2][0], V[0][0])),
                                        __dmul_rn(__dsub_rn(V[1][0], V[0][0]), __dsub_rn(V[2][1], V[0][1]))));
      double acc = 0.0;
      for (int s = 0; s < 3; ++s) {
        const double *p1 = V[s], *p2 = V[(s + 1) % 3];
        const double ex = p2[0] - p1[0], ey = p2[1] - p1[1];
        double line = 0.0;
        for (int q = 0; q < 6; ++q) {
          const double tq = 0.5 * (kGlX[q] + 1.0);
          const double xq = p1[0] + tq * ex, yq = p1[1] + tq * ey;
          double v = 0.5 * kGlW[q];
          for (int e = 0; e <= a; ++e) v *= xq;
          for (int e = 0; e < k; ++e) v *= yq;
          line += v;
        }
        acc += ey * line / (a + 1);
      }
      S.rhs[tid] = sabc * acc;
    }
    if (tid < kQuadDim) {
      S.order[tid] = tid;
    }
    if (tid < 128) S.where[tid] = tid;
    __syncthreads();

    // augmented matrix [Phi P rhs; P^T 0 rhs] in registers, padded to 128 x 128
    double M[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int i = ty + 16 * a;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int j = tx + 16 * b;
        double v = 0.0;
        if (j == kQuadRhsCol) {
          v = i < kQuadDim ? S.rhs[i] : 0.0;
        } else if (i < kQuadNbr && j < kQuadNbr) {
          const double xi = S.c[i][0], yi = S.c[i][1], xj = S.c[j][0], yj = S.c[j][1];
          const double di = __dadd_rn(__dmul_rn(xi, xi), __dmul_rn(yi, yi));
          const double dj = __dadd_rn(__dmul_rn(xj, xj), __dmul_rn(yj, yj));
          const double ip = __dadd_rn(__dmul_rn(xi, xj), __dmul_rn(yi, yj));
          const double r2 = __dsub_rn(__dadd_rn(dj, di), __dmul_rn(2.0, ip));
          v = sqrt(pow(r2, 7.0));
        } else if (i < kQuadNbr && j < kQuadDim) {
          v = S.pm[i][j - kQuadNbr];
        } else if (i < kQuadDim && j < kQuadNbr) {
          v = S.pm[j][i - kQuadNbr];
        }
        M[a][b] = v;
      }
    }

    // Gauss-Jordan elimination with partial pivoting (rows stay in place;
    // order/where hold the row exchanges), the right-hand side carried along
    unsigned used = 0;
    if (tx == 0) pivot_column<0>(M, S, used, 0, ty, tx, err);
    __syncthreads();
    gj_columns<0>(M, S, used, 16, ty, tx, err);
    gj_columns<1>(M, S, used, 16, ty, tx, err);
    gj_columns<2>(M, S, used, 16, ty, tx, err);
    gj_columns<3>(M, S, used, 16, ty, tx, err);
    gj_columns<4>(M, S, used, 16, ty, tx, err);
    gj_columns<5>(M, S, used, 16, ty, tx, err);
    gj_columns<6>(M, S, used, 16, ty, tx, err);
    gj_columns<7>(M, S, used, kQuadDim - 112, ty, tx, err);
    if (tx == (kQuadRhsCol & 15)) {
#pragma unroll
      for (int a = 0; a < 8; ++a) S.ys[ty + 16 * a] = M[a][kQuadRhsCol >> 4];
    }
    __syncthreads();
    if (tid < kQuadNbr) S.x[tid] = S.ys[S.order[tid]] / S.piv[tid];
    if (tid < kQuadNbr) w.wt[static_cast<int64_t>(t) * kQuadNbr + tid] = __dmul_rn(S.x[tid], S.dist[tid]);
    __syncthreads();
  }
}

// ------------------------------------------------------------- 5. scatter --
__global__ void quad_count_kernel(int64_t m, QuadWs w) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g < m) atomicAdd(w.count + w.nni[g], 1);
}

// exclusive scan of count[0..n) into count[0..n], one CTA
__global__ void __launch_bounds__(1024) quad_scan_kernel(int n, QuadWs w) {
  __shared__ int part[32];
  __shared__ int carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int i = base + tid;
    const int v = i < n ? w.count[i] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) part[warp] = incl;
    __syncthreads();
    int before = carry;
    for (int w2 = 0; w2 < warp; ++w2) before += part[w2];
    if (i < n) w.count[i] = before + incl - v;
    __syncthreads();
    if (tid == 1023) carry = before + incl;
    __syncthreads();
  }
  if (tid == 0) w.count[n] = carry;
}

__global__ void quad_fill_kernel(int64_t m, QuadWs w) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= m) return;
  const int node = w.nni[g];
  const int pos = w.count[node] + atomicAdd(w.cursor + node, 1);
  w.entry[pos] = static_cast<int32_t>(g);
}

// per node: its entries sorted by (triangle, slot), summed in that order
__global__ void quad_sum_kernel(int n, QuadWs w, double *__restrict__ weights) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = w.count[i], e = w.count[i + 1];
  int32_t *en = w.entry;
  for (int p = b + 1; p < e; ++p) {
    const int32_t v = en[p];
    int q = p - 1;
    while (q >= b && en[q] > v) {
      en[q + 1] = en[q];
      --q;
    }
    en[q + 1] = v;
  }
  double s = 0.0;
  for (int p = b; p < e; ++p) s = __dadd_rn(s, w.wt[en[p]]);
  weights[i] = s;
}

static int hash_bits(int64_t ntri) {
  int b = 6;
  while ((1ll << b) < 4 * ntri) ++b;
  return b;
}

static size_t quad_layout(int64_t n, int64_t ntri, QuadWs *w, char *base) {
  const int hb = hash_bits(ntri);
  const int64_t H = 1ll << hb;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = round_up(off + bytes, 256);
    return base ? base + o : nullptr;
  };
  QuadWs q{};
  q.tri = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * 3 * ntri));
  q.tnorm = reinterpret_cast<double *>(take(sizeof(double) * 3 * ntri));
  q.mid = reinterpret_cast<double *>(take(sizeof(double) * 3 * ntri));
  q.enorm = reinterpret_cast<double *>(take(sizeof(double) * 9 * ntri));
  q.hkey = reinterpret_cast<long long *>(take(sizeof(long long) * H));
  q.hid = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * 2 * H));
  q.nni = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * kQuadNbr * ntri));
  q.wt = reinterpret_cast<double *>(take(sizeof(double) * kQuadNbr * ntri));
  q.count = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * (n + 1)));
  q.cursor = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * n));
  q.entry = reinterpret_cast<int32_t *>(take(sizeof(int32_t) * kQuadNbr * ntri));
  q.hbits = hb;
  if (w) *w = q;
  return off;
}

}  // namespace f3d

extern "C" {

int f3d_surface_quadrature_workspace_bytes(int64_t n, int64_t ntri, size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  if (n < 0 || ntri < 0) return F3D_ERR_SHAPE;
  if (n > f3d::kQuadMaxNodes) return F3D_ERR_TOO_LARGE;
  *bytes = f3d::quad_layout(n, ntri, nullptr, nullptr);
  return F3D_OK;
}

int f3d_surface_quadrature(const double *nodes, int64_t n, const int32_t *triangles, int64_t ntri,
                           const double *gradient, double *weights, int32_t *neighbors, void *workspace,
                           size_t workspace_bytes, void *stream) {
  if (n < f3d::kQuadNbr || ntri < 1 || ntri > (1ll << 24)) return F3D_ERR_SHAPE;
  if (n > f3d::kQuadMaxNodes) return F3D_ERR_TOO_LARGE;
  if (!nodes || !triangles || !gradient || !weights || !workspace) return F3D_ERR_NULL;
  if (!f3d::aligned(nodes, 8) || !f3d::aligned(gradient, 8) || !f3d::aligned(weights, 8) ||
      !f3d::aligned(workspace, 256) || !f3d::aligned(triangles, 4) || (neighbors && !f3d::aligned(neighbors, 4)))
    return F3D_ERR_ALIGN;
  f3d::QuadWs w{};
  const size_t need = f3d::quad_layout(n, ntri, &w, static_cast<char *>(workspace));
  if (workspace_bytes < need) return F3D_ERR_WORKSPACE;
  if (neighbors) w.nni = neighbors;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int *err = f3d::device_error_word();
  const int64_t H = 1ll << w.hbits;
  if (cudaMemsetAsync(w.hkey, 0xff, sizeof(long long) * H, st) != cudaSuccess ||
      cudaMemsetAsync(w.hid, 0xff, sizeof(int32_t) * 2 * H, st) != cudaSuccess ||
      cudaMemsetAsync(w.count, 0, sizeof(int32_t) * (n + 1), st) != cudaSuccess ||
      cudaMemsetAsync(w.cursor, 0, sizeof(int32_t) * n, st) != cudaSuccess)
    return F3D_ERR_CUDA;
  const int nt = static_cast<int>(ntri), nn = static_cast<int>(n);
  f3d::quad_prep_kernel<<<(nt + 127) / 128, 128, 0, st>>>(nodes, nn, triangles, nt, w, err);
  f3d::quad_edges_kernel<<<(3 * nt + 127) / 128, 128, 0, st>>>(nn, nt, w, err);
  const int tile = static_cast<int>(std::min<int64_t>(n, f3d::kKnnTile));
  const size_t knn_smem = sizeof(double) * (tile + f3d::kQuadNbr + f3d::kKnnCand) +
                          sizeof(int) * (f3d::kKnnCand + f3d::kQuadNbr + f3d::kKnnBins);
  // the opt-in limit counts the kernel's static shared memory too: ask for
  // what this call needs
  static size_t attr_bytes[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return F3D_ERR_CUDA;
  if (knn_smem > attr_bytes[dev]) {
    if (cudaFuncSetAttribute(f3d::quad_knn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(knn_smem)) != cudaSuccess)
      return F3D_ERR_CUDA;
    attr_bytes[dev] = knn_smem;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f3d::quad_knn_kernel, f3d::kKnnThreads, knn_smem) !=
          cudaSuccess ||
      per_sm < 1)
    return F3D_ERR_CUDA;
  const int64_t knn_grid = std::min<int64_t>(ntri, static_cast<int64_t>(per_sm) * f3d::sm_count());
  f3d::quad_knn_kernel<<<static_cast<unsigned>(knn_grid), f3d::kKnnThreads, knn_smem, st>>>(nodes, nn, w.mid, nt,
                                                                                            tile, w.nni, err);
  const int64_t tri_grid = std::min<int64_t>(ntri, f3d::sm_count());
  f3d::quad_triangle_kernel<<<static_cast<unsigned>(tri_grid), f3d::kTriThreads, 0, st>>>(nodes, gradient, nt, w, err);
  const int64_t m = f3d::kQuadNbr * ntri;
  f3d::quad_count_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, st>>>(m, w);
  f3d::quad_scan_kernel<<<1, 1024, 0, st>>>(nn, w);
  f3d::quad_fill_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, st>>>(m, w);
  f3d::quad_sum_kernel<<<(nn + 127) / 128, 128, 0, st>>>(nn, w, weights);
  return f3d::launch_status();
}

}  // extern "C"
