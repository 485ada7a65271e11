// Symmetric evaluation of the all-pairs self-sums over one point set: the
// Oseen sum of oseen_kernel_times_density_numba (python/kernels/kernels.py:
// 214-287) and the stresslet sum of stresslet_kernel_times_normal_times_
// density_numba (kernels.py:1123-1183), j == i skipped, and the same sums
// with the pairs of one group (fiber) skipped (tstep_utils.py:653-700,
// 812-851).  Further targets that are not sources (the off-surface points of
// a double-layer evaluation) may follow the n sources in the same array;
// they are summed one-sided in the same launch.
//
// A pair (i, j) contributes to target i through source j's density (and
// normal) and to target j through source i's; both terms share r = x_i - x_j,
// |r| and its powers, which is most of the arithmetic.  Each unordered pair
// is therefore evaluated once:
//   Oseen:     u_i += d_j/r + (r.d_j) r/r^3,   u_j += d_i/r + (r.d_i) r/r^3
//   stresslet: v_i += (r.d_j)(r.n_j) r/r^5,    v_j -= (r.d_i)(r.n_i) r/r^5
// (the prefactor is applied once per target, as everywhere): about 18 FP64
// instructions per ordered pair instead of 25-26.
//
// Decomposition: tiles of 128 points; one CTA of 64 threads per work item.
// Thread t holds targets t and t + 64 of its tile, with their partial sums,
// in registers.  Items, in this order:
//   * (I, J), I <= J < T, row by row (a tile's sum is complete once its row
//     is done, so the tile reductions below spread over the launch);
//   * (X, J), X >= T: a tile of further targets against source tile J.
// In an off-diagonal item (I < J) a warp meets tile J's sources 32 at a
// time, rotating: at step s lane l pairs its two targets with source
// (l + s) mod 32 of the group, whose position and running source-side sum
// it holds in registers and hands to lane l - 1 after the step (six
// shuffles per step, shared by the two targets); the density and normal
// come from shared memory.  After 32 steps lane l holds source l's sum over
// the warp's 64 targets; the CTA's two warps' sums are added in shared
// memory.  Diagonal items (I == J) and further-target items are summed
// from the target side only.  Each item writes its partial(s) to tile I's
// slot J (and tile J's slot I); every tile thus receives exactly T partials
// (T = number of source tiles), and the CTA that delivers the last one (a
// self-resetting counter per tile) sums them in slot order and writes the
// result, so the sum is the same run to run.
//
// Rules per pair (skip, regularisation of pairs closer than eps) are applied
// only where they can matter: in diagonal items, in items whose group-id
// ranges meet (SKIP_GROUP), and in items where a pair within eps is met
// (detected from the smallest r^2 of the plain pass, which is then redone).
// Tile slots past the end hold far-away points with zero density and normal
// (targets at +1e30, sources at -1e30), whose terms vanish without a select.
//
// The Oseen sum also has a two-density form (DUAL): two densities over the
// same pairs, the geometry once, each sum with the single form's exact
// arithmetic and order, so that each equals its single sum bit for bit.
//
// The same items serve a plain source -> target sum (the tile form: xt set,
// the targets in an array of their own): there are no symmetric items, every
// item is a tile of targets against a tile of sources, summed from the target
// side with two targets per thread, close pairs regularised; partials and
// counters are then kept for the target tiles only (tile0 = T).
#include <climits>
#include <type_traits>

#include "f3d_common.cuh"
#include "f3d_pair_math.cuh"

namespace f3d {

constexpr int kSymTile = 128;
constexpr int kSymThreads = 64;  // two targets per thread
constexpr int kSymWarps = kSymThreads / 32;
// Partial storage grows as T (T + T2) x 3 KB: 28 MB for the 12000-node sphere,
// 1 GB for 64000 fiber points onto 85600 targets; the caps keep it within 2 GiB.
constexpr int kSymMaxTiles = 1024;
constexpr size_t kSymMaxPartialBytes = size_t(2) << 30;

struct SymArgs {
  const double *x, *dens, *nrm;  // x: nt x 3 (the first n are the sources); dens, nrm: n x 3
  const double *dens2;           // n x 3 (DUAL only)
  const int32_t *grp;            // nt (SKIP_GROUP only)
  double *out, *out2;            // nt x 3 (out2: DUAL only)
  double *partial, *partial2;    // [T + T2][T][kSymTile][3] (partial2: DUAL only)
  unsigned *counters;            // [T + T2], zero on entry and on exit
  const double *xt;              // tile form: nt x 3 targets (x then holds the n sources only)
  int64_t n, nt;
  int ntiles, nextra;            // T source tiles, T2 tiles of further targets
  int tile0;                     // first tile with partials and a counter (tile form: T)
  int sub;                       // tile form: source sub-tiles per 128-point tile (1 or 2; else 1)
  int accumulate;
  double eps2, reg2, scale;
};

static int64_t sym_tiles(int64_t n) { return (n + kSymTile - 1) / kSymTile; }

size_t sym_partial_bytes(int64_t n, int64_t nt) {
  const int64_t T = sym_tiles(n), T2 = sym_tiles(nt - n);
  return static_cast<size_t>(T + T2) * static_cast<size_t>(T) * kSymTile * 3 * sizeof(double);
}

// Tile form: [T2][T sub][kSymTile][3] partials, T2 = target tiles, each
// 128-point source tile taken as `sub` sub-tiles (one partial each).
static int64_t tile_slots(int64_t ns, int sub) {
  const int64_t w = sub == 2 ? kSymTile / 2 : kSymTile;
  return (ns + w - 1) / w;
}

size_t tile_partial_bytes(int64_t ns, int64_t nt, int sub) {
  return static_cast<size_t>(sym_tiles(nt)) * static_cast<size_t>(tile_slots(ns, sub)) * kSymTile * 3 *
         sizeof(double);
}

bool tile_fits(int64_t ns, int64_t nt, int sub) {
  if (ns < 0 || nt < 0) return false;
  if (ns == 0 || nt == 0) return true;
  return sym_tiles(ns) <= kSymMaxTiles && sym_tiles(nt) <= kMaxCounters &&
         tile_partial_bytes(ns, nt, sub) <= kSymMaxPartialBytes;
}

bool sym_fits(int64_t n, int64_t nt) {
  if (n < 0 || nt < n) return false;
  if (n == 0) return true;
  const int64_t T = sym_tiles(n), T2 = sym_tiles(nt - n);
  return T <= kSymMaxTiles && T + T2 <= kMaxCounters && sym_partial_bytes(n, nt) <= kSymMaxPartialBytes;
}

__device__ __forceinline__ int64_t tile_slots_dev(int64_t ns, int w) { return (ns + w - 1) / w; }

template <int KIND, int MODE, bool DUAL>
__global__ void __launch_bounds__(kSymThreads) pair_sym_kernel(const SymArgs a) {
  static_assert(!DUAL || KIND == F3D_KERNEL_OSEEN, "the two-density form is Oseen only");
  constexpr bool kNrm = (KIND == F3D_KERNEL_STRESSLET);
  constexpr bool kGrp = (MODE == F3D_SELF_SKIP_GROUP);
  constexpr int ND = DUAL ? 2 : 1;  // densities
  // sources of tile J, one array per component (conflict-free when the
  // lanes of a warp read different sources)
  __shared__ __align__(16) double s_x[3][kSymTile];
  __shared__ __align__(16) double s_d[ND][3][kSymTile];
  __shared__ __align__(16) double s_n[kNrm ? 3 : 1][kSymTile];
  __shared__ int32_t s_grp[kGrp ? kSymTile : 1];
  __shared__ __align__(16) double s_accj[ND][kSymWarps][kSymTile][3];
  __shared__ int s_flags;
  __shared__ int s_range[kSymWarps][4];

  const int T = a.ntiles;
  const int64_t nsym = a.xt ? 0 : static_cast<int64_t>(T) * (T + 1) / 2;
  // partial slots per tile (one per source tile, or per source sub-tile in
  // the tile form) and the width of the item's source tile
  const int src_w = (a.xt && a.sub == 2) ? kSymTile / 2 : kSymTile;
  const int S = a.xt ? static_cast<int>(tile_slots_dev(a.n, src_w)) : T;
  const int64_t item = blockIdx.x;
  int I, J;
  if (item < nsym) {
    // row-major upper triangle: row r starts at item r (2T - r + 1) / 2
    auto start = [T](int r) { return static_cast<int64_t>(r) * (2 * T - r + 1) / 2; };
    const double b = 2.0 * T + 1.0;
    I = static_cast<int>((b - sqrt(b * b - 8.0 * static_cast<double>(item))) * 0.5);
    I = max(0, min(I, T - 1));
    while (I > 0 && start(I) > item) --I;
    while (I + 1 < T && start(I + 1) <= item) ++I;
    J = I + static_cast<int>(item - start(I));
  } else {
    const int64_t e = item - nsym;
    I = T + static_cast<int>(e / S);
    J = static_cast<int>(e % S);
  }
  const bool extra = I >= T;  // a tile of targets that are not sources
  const bool diag = !a.xt && (I == J);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // this thread's targets (k = 0: tile slot tid, k = 1: tid + 64), with their
  // own density and normal for the terms they send to the sources
  const int64_t tbase =
      extra ? (a.xt ? 0 : a.n) + static_cast<int64_t>(I - T) * kSymTile : static_cast<int64_t>(I) * kSymTile;
  const int64_t tend = extra ? a.nt : a.n;
  const double *const xtrg = (extra && a.xt) ? a.xt : a.x;
  double tx[2][3], td[ND][2][3], tn[2][3];
  int32_t tg[2];
  bool tv[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int64_t i = tbase + tid + k * kSymThreads;
    tv[k] = i < tend;
    tg[k] = INT32_MIN;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      tx[k][c] = tv[k] ? xtrg[3 * i + c] : 1e30;
      td[0][k][c] = (tv[k] && !extra) ? a.dens[3 * i + c] : 0.0;
      if (DUAL) td[ND - 1][k][c] = (tv[k] && !extra) ? a.dens2[3 * i + c] : 0.0;
      tn[k][c] = (kNrm && tv[k] && !extra) ? a.nrm[3 * i + c] : 0.0;
    }
    if (kGrp && tv[k]) tg[k] = a.grp[i];
  }
  // tile J's sources
  const int64_t j0 = static_cast<int64_t>(J) * src_w;
  const int cnt = static_cast<int>(min(static_cast<int64_t>(src_w), a.n - j0));
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int s = tid + k * kSymThreads;
    const bool sv = s < cnt;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s_x[c][s] = sv ? a.x[3 * (j0 + s) + c] : -1e30;
      s_d[0][c][s] = sv ? a.dens[3 * (j0 + s) + c] : 0.0;
      if (DUAL) s_d[ND - 1][c][s] = sv ? a.dens2[3 * (j0 + s) + c] : 0.0;
      if (kNrm) s_n[c][s] = sv ? a.nrm[3 * (j0 + s) + c] : 0.0;
    }
    if (kGrp) s_grp[s] = sv ? a.grp[j0 + s] : INT32_MIN;
  }

  // group-id ranges of the targets and the sources (SKIP_GROUP): pairs of
  // one group can occur only if they meet
  bool careful = diag;
  if (kGrp && !diag) {
    int tlo = INT32_MAX, thi = INT32_MIN, slo = INT32_MAX, shi = INT32_MIN;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (tv[k]) {
        tlo = min(tlo, tg[k]);
        thi = max(thi, tg[k]);
      }
      const int s = tid + k * kSymThreads;
      if (s < cnt) {
        const int32_t g = a.grp[j0 + s];
        slo = min(slo, g);
        shi = max(shi, g);
      }
    }
    tlo = __reduce_min_sync(0xffffffffu, tlo);
    thi = __reduce_max_sync(0xffffffffu, thi);
    slo = __reduce_min_sync(0xffffffffu, slo);
    shi = __reduce_max_sync(0xffffffffu, shi);
    if (lane == 0) {
      s_range[warp][0] = tlo;
      s_range[warp][1] = thi;
      s_range[warp][2] = slo;
      s_range[warp][3] = shi;
    }
  }
  __syncthreads();
  if (kGrp && !diag) {
    int TL = s_range[0][0], TH = s_range[0][1], SL = s_range[0][2], SH = s_range[0][3];
#pragma unroll
    for (int w = 1; w < kSymWarps; ++w) {
      TL = min(TL, s_range[w][0]);
      TH = max(TH, s_range[w][1]);
      SL = min(SL, s_range[w][2]);
      SH = max(SH, s_range[w][3]);
    }
    careful = (TL <= SH && SL <= TH);
  }

  const long long eps2_bits = __double_as_longlong(a.eps2);
  const int eps2_hi = __double2hiint(a.eps2);
  const double reg2 = a.reg2;
  double acc[ND][2][3];
  int hmin = INT32_MAX;

  // with the rules: regularise a close pair that is not skipped; without:
  // note the smallest r^2 (high word) for the close-pair check
  auto rules = [&](auto rules_tag, double &r2, bool skip) {
    constexpr bool R = decltype(rules_tag)::value;
    if (R) {
      if (!skip && __double_as_longlong(r2) < eps2_bits) r2 += reg2;
    } else {
      hmin = min(hmin, __double2hiint(r2));
    }
  };

  // target side only: every source of the tile, read by all lanes at once
  auto one_sided = [&](auto rules_tag) {
    constexpr bool R = decltype(rules_tag)::value;
#pragma unroll
    for (int q = 0; q < ND; ++q)
#pragma unroll
      for (int k = 0; k < 2; ++k) acc[q][k][0] = acc[q][k][1] = acc[q][k][2] = 0.0;
    for (int s = 0; s < cnt; ++s) {
      const double p0 = s_x[0][s], p1 = s_x[1][s], p2 = s_x[2][s];
      double sd[ND][3];
#pragma unroll
      for (int q = 0; q < ND; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) sd[q][c] = s_d[q][c][s];
      double n0 = 0.0, n1 = 0.0, n2 = 0.0;
      if (kNrm) {
        n0 = s_n[0][s];
        n1 = s_n[1][s];
        n2 = s_n[2][s];
      }
      int32_t gj = 0;
      if (R && kGrp) gj = s_grp[s];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double dx = tx[k][0] - p0, dy = tx[k][1] - p1, dz = tx[k][2] - p2;
        double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        bool skip = false;
        if (R) skip = kGrp ? (gj == tg[k]) : (diag && s == tid + k * kSymThreads);
        rules(rules_tag, r2, skip);
        if (KIND == F3D_KERNEL_OSEEN) {
          double ri = rsqrt_refined(r2);
          if (R) ri = skip ? 0.0 : ri;
          const double ri3 = ri * ri * ri;
#pragma unroll
          for (int q = 0; q < ND; ++q) {
            const double g = ri3 * fma(dx, sd[q][0], fma(dy, sd[q][1], dz * sd[q][2]));
            acc[q][k][0] = fma(g, dx, fma(ri, sd[q][0], acc[q][k][0]));
            acc[q][k][1] = fma(g, dy, fma(ri, sd[q][1], acc[q][k][1]));
            acc[q][k][2] = fma(g, dz, fma(ri, sd[q][2], acc[q][k][2]));
          }
        } else {
          const double qq = fma(dx, sd[0][0], fma(dy, sd[0][1], dz * sd[0][2])) * fma(dx, n0, fma(dy, n1, dz * n2));
          double f = times_rsqrt5(qq, r2);
          if (R) f = skip ? 0.0 : f;
          acc[0][k][0] = fma(f, dx, acc[0][k][0]);
          acc[0][k][1] = fma(f, dy, acc[0][k][1]);
          acc[0][k][2] = fma(f, dz, acc[0][k][2]);
        }
      }
    }
  };

  // both sides: tile J's sources rotate through the warp 32 at a time
  auto rotating = [&](auto rules_tag) {
    constexpr bool R = decltype(rules_tag)::value;
#pragma unroll
    for (int q = 0; q < ND; ++q)
#pragma unroll
      for (int k = 0; k < 2; ++k) acc[q][k][0] = acc[q][k][1] = acc[q][k][2] = 0.0;
    const int from = (lane + 1) & 31;
    for (int sb = 0; sb < cnt; sb += 32) {
      int m = lane;
      double px = s_x[0][sb + m], py = s_x[1][sb + m], pz = s_x[2][sb + m];
      double aj[ND][3];
#pragma unroll
      for (int q = 0; q < ND; ++q) aj[q][0] = aj[q][1] = aj[q][2] = 0.0;
#pragma unroll 2
      for (int st = 0; st < 32; ++st) {
        const int js = sb + m;
        double sd[ND][3];
#pragma unroll
        for (int q = 0; q < ND; ++q)
#pragma unroll
          for (int c = 0; c < 3; ++c) sd[q][c] = s_d[q][c][js];
        double n0 = 0.0, n1 = 0.0, n2 = 0.0;
        if (kNrm) {
          n0 = s_n[0][js];
          n1 = s_n[1][js];
          n2 = s_n[2][js];
        }
        int32_t gj = 0;
        if (R && kGrp) gj = s_grp[js];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const double dx = tx[k][0] - px, dy = tx[k][1] - py, dz = tx[k][2] - pz;
          double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
          const bool skip = R && kGrp && (gj == tg[k]);
          rules(rules_tag, r2, skip);
          if (KIND == F3D_KERNEL_OSEEN) {
            double ri = rsqrt_refined(r2);
            if (R) ri = skip ? 0.0 : ri;
            const double ri3 = ri * ri * ri;
#pragma unroll
            for (int q = 0; q < ND; ++q) {
              const double g = ri3 * fma(dx, sd[q][0], fma(dy, sd[q][1], dz * sd[q][2]));
              const double h = ri3 * fma(dx, td[q][k][0], fma(dy, td[q][k][1], dz * td[q][k][2]));
              acc[q][k][0] = fma(g, dx, fma(ri, sd[q][0], acc[q][k][0]));
              acc[q][k][1] = fma(g, dy, fma(ri, sd[q][1], acc[q][k][1]));
              acc[q][k][2] = fma(g, dz, fma(ri, sd[q][2], acc[q][k][2]));
              aj[q][0] = fma(h, dx, fma(ri, td[q][k][0], aj[q][0]));
              aj[q][1] = fma(h, dy, fma(ri, td[q][k][1], aj[q][1]));
              aj[q][2] = fma(h, dz, fma(ri, td[q][k][2], aj[q][2]));
            }
          } else {
            double R5 = rsqrt5(r2);
            if (R) R5 = skip ? 0.0 : R5;
            const double f =
                (fma(dx, sd[0][0], fma(dy, sd[0][1], dz * sd[0][2])) * fma(dx, n0, fma(dy, n1, dz * n2))) * R5;
            const double h = (fma(dx, td[0][k][0], fma(dy, td[0][k][1], dz * td[0][k][2])) *
                              fma(dx, tn[k][0], fma(dy, tn[k][1], dz * tn[k][2]))) *
                             R5;
            acc[0][k][0] = fma(f, dx, acc[0][k][0]);
            acc[0][k][1] = fma(f, dy, acc[0][k][1]);
            acc[0][k][2] = fma(f, dz, acc[0][k][2]);
            aj[0][0] = fma(-h, dx, aj[0][0]);
            aj[0][1] = fma(-h, dy, aj[0][1]);
            aj[0][2] = fma(-h, dz, aj[0][2]);
          }
        }
        // hand the source (position and its running sums) to lane - 1
        px = __shfl_sync(0xffffffffu, px, from);
        py = __shfl_sync(0xffffffffu, py, from);
        pz = __shfl_sync(0xffffffffu, pz, from);
#pragma unroll
        for (int q = 0; q < ND; ++q)
#pragma unroll
          for (int c = 0; c < 3; ++c) aj[q][c] = __shfl_sync(0xffffffffu, aj[q][c], from);
        m = (m + 1) & 31;
      }
      // after a full turn lane l holds source sb + l again
#pragma unroll
      for (int q = 0; q < ND; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) s_accj[q][warp][sb + lane][c] = aj[q][c];
    }
  };

  using Plain = std::integral_constant<bool, false>;
  using Careful = std::integral_constant<bool, true>;
  if (diag) {
    one_sided(Careful{});
  } else {
    // the plain pass, redone with the rules if a pair within eps was met
    bool redo = careful;
    if (!careful) {
      if (extra)
        one_sided(Plain{});
      else
        rotating(Plain{});
      redo = __syncthreads_or(hmin <= eps2_hi);
    }
    if (redo) {
      __syncthreads();
      if (extra)
        one_sided(Careful{});
      else
        rotating(Careful{});
    }
  }
  __syncthreads();
  const int64_t slot_stride = static_cast<int64_t>(kSymTile) * 3;
#pragma unroll
  for (int q = 0; q < ND; ++q) {
    double *const part = q == 0 ? a.partial : a.partial2;
    // tile J's partial from this item (slot I): the two warps' sums, in warp order
    if (!diag && !extra) {
      double *pj = part + (static_cast<int64_t>(J) * T + I) * slot_stride;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int s = tid + k * kSymThreads;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double v = s_accj[q][0][s][c];
#pragma unroll
          for (int w = 1; w < kSymWarps; ++w) v += s_accj[q][w][s][c];
          __stcg(pj + 3 * s + c, v);
        }
      }
    }
    // tile I's partial from this item (slot J)
    double *pi = part + (static_cast<int64_t>(I - a.tile0) * S + J) * slot_stride;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) __stcg(pi + 3 * (tid + k * kSymThreads) + c, acc[q][k][c]);
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    int f = 0;
    if (atomicAdd(&a.counters[I - a.tile0], 1u) == static_cast<unsigned>(S - 1)) f |= 1;
    if (!diag && !extra && atomicAdd(&a.counters[J], 1u) == static_cast<unsigned>(T - 1)) f |= 2;
    s_flags = f;
  }
  __syncthreads();
  const int flags = s_flags;
  for (int which = 0; which < 2; ++which) {
    if (!(flags & (1 << which))) continue;
    __threadfence();
    const int X = which == 0 ? I : J;
    const int64_t xbase =
        X < T ? static_cast<int64_t>(X) * kSymTile : (a.xt ? 0 : a.n) + static_cast<int64_t>(X - T) * kSymTile;
    const int64_t xend = X < T ? a.n : a.nt;
    // A slot is the tile's 128 x 3 sums in output order; thread tid sums the
    // pairs of doubles tid, tid + 64 and tid + 128 of every slot (16-byte
    // loads, eight slots in flight), in slot order.
    const int nvals = 3 * static_cast<int>(min(static_cast<int64_t>(kSymTile), xend - xbase));
#pragma unroll
    for (int q = 0; q < ND; ++q) {
      const double2 *p =
          reinterpret_cast<const double2 *>((q == 0 ? a.partial : a.partial2) +
                                            static_cast<int64_t>(X - a.tile0) * S * slot_stride);
      double2 v[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) v[m] = make_double2(0.0, 0.0);
      constexpr int kPairsPerSlot = kSymTile * 3 / 2;
      int slot = 0;
      for (; slot + 8 <= S; slot += 8) {
        double2 r[8][3];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int m = 0; m < 3; ++m) r[u][m] = __ldcg(p + (slot + u) * kPairsPerSlot + tid + m * kSymThreads);
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            v[m].x += r[u][m].x;
            v[m].y += r[u][m].y;
          }
      }
      for (; slot < S; ++slot)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          const double2 r = __ldcg(p + slot * kPairsPerSlot + tid + m * kSymThreads);
          v[m].x += r.x;
          v[m].y += r.y;
        }
      double *const o = (q == 0 ? a.out : a.out2) + 3 * xbase;
      const bool vec = (reinterpret_cast<uintptr_t>(o) & 15) == 0;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const int f = 2 * (tid + m * kSymThreads);
        double2 w = make_double2(v[m].x * a.scale, v[m].y * a.scale);
        if (vec && f + 1 < nvals) {
          double2 *o2 = reinterpret_cast<double2 *>(o + f);
          if (a.accumulate) {
            const double2 old = *o2;
            w.x += old.x;
            w.y += old.y;
          }
          *o2 = w;
        } else {
          if (f < nvals) o[f] = a.accumulate ? o[f] + w.x : w.x;
          if (f + 1 < nvals) o[f + 1] = a.accumulate ? o[f + 1] + w.y : w.y;
        }
      }
    }
    if (tid == 0) a.counters[X - a.tile0] = 0u;
  }
}

template <int KIND, int MODE, bool DUAL>
static int sym_launch_one(const SymArgs &a, int *occupancy, cudaStream_t st) {
  auto kfn = pair_sym_kernel<KIND, MODE, DUAL>;
  if (occupancy)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, kfn, kSymThreads, 0) == cudaSuccess
               ? F3D_OK
               : F3D_ERR_CUDA;
  const int64_t items = a.xt ? static_cast<int64_t>(a.nextra) * tile_slots(a.n, a.sub)
                             : static_cast<int64_t>(a.ntiles) * (a.ntiles + 1) / 2 +
                                   static_cast<int64_t>(a.nextra) * a.ntiles;
  kfn<<<static_cast<unsigned>(items), kSymThreads, 0, st>>>(a);
  return launch_status();
}

// The symmetric self-sum (kernel OSEEN or STRESSLET, FP64, mode SKIP_INDEX or
// SKIP_GROUP) over the first n of nt points, the rest summed as targets only;
// with dens2/out2 (Oseen only) the two-density form.  partial:
// sym_partial_bytes(n, nt) of workspace, twice that for two densities;
// counters: the pair workspace's counter region.  With occupancy non-null,
// only reports the kernel's resident CTAs per SM.
int pair_sym_launch(int kernel, int self_mode, const double *x, const double *dens, const double *nrm,
                    const int32_t *grp, double *out, int64_t n, int64_t nt, double eta, double reg, double eps,
                    int accumulate, double *partial, unsigned *counters, int *occupancy, cudaStream_t st,
                    const double *dens2, double *out2, bool dual) {
  SymArgs a{};
  a.x = x;
  a.dens = dens;
  a.dens2 = dens2;
  a.nrm = nrm;
  a.grp = grp;
  a.out = out;
  a.out2 = out2;
  a.partial = partial;
  a.partial2 = partial ? partial + sym_partial_bytes(n, nt) / sizeof(double) : nullptr;
  a.counters = counters;
  a.n = n;
  a.nt = nt;
  a.ntiles = static_cast<int>(sym_tiles(n));
  a.nextra = static_cast<int>(sym_tiles(nt - n));
  a.accumulate = accumulate ? 1 : 0;
  a.eps2 = eps * eps;
  a.reg2 = reg * reg;
  a.scale = (kernel == F3D_KERNEL_STRESSLET) ? -3.0 / (4.0 * kPi * eta) : 1.0 / (8.0 * kPi * eta);
  if (kernel == F3D_KERNEL_OSEEN && dual) {
    return self_mode == F3D_SELF_SKIP_INDEX
               ? sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX, true>(a, occupancy, st)
               : sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_GROUP, true>(a, occupancy, st);
  }
  if (kernel == F3D_KERNEL_OSEEN) {
    return self_mode == F3D_SELF_SKIP_INDEX
               ? sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX, false>(a, occupancy, st)
               : sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_GROUP, false>(a, occupancy, st);
  }
  return self_mode == F3D_SELF_SKIP_INDEX
             ? sym_launch_one<F3D_KERNEL_STRESSLET, F3D_SELF_SKIP_INDEX, false>(a, occupancy, st)
             : sym_launch_one<F3D_KERNEL_STRESSLET, F3D_SELF_SKIP_GROUP, false>(a, occupancy, st);
}

// The tile form of a plain source -> target sum (kernel OSEEN or STRESSLET,
// FP64, close pairs regularised as F3D_SELF_REGULARISE does): ns sources in
// xs, nt targets in xt; with dens2/out2 (Oseen only) the two-density form.
// partial: tile_partial_bytes(ns, nt) of workspace, twice that for two
// densities.  With occupancy non-null, only reports resident CTAs per SM.
int pair_tile_launch(int kernel, const double *xs, const double *dens, const double *nrm, const double *xt,
                     double *out, int64_t ns, int64_t nt, double eta, double reg, double eps, int accumulate,
                     double *partial, unsigned *counters, int *occupancy, cudaStream_t st, const double *dens2,
                     double *out2, bool dual, int sub) {
  SymArgs a{};
  a.x = xs;
  a.xt = xt;
  a.dens = dens;
  a.dens2 = dens2;
  a.nrm = nrm;
  a.out = out;
  a.out2 = out2;
  a.partial = partial;
  a.partial2 = partial ? partial + tile_partial_bytes(ns, nt, sub) / sizeof(double) : nullptr;
  a.counters = counters;
  a.n = ns;
  a.nt = nt;
  a.ntiles = static_cast<int>(sym_tiles(ns));
  a.nextra = static_cast<int>(sym_tiles(nt));
  a.tile0 = a.ntiles;
  a.sub = sub == 2 ? 2 : 1;
  a.accumulate = accumulate ? 1 : 0;
  a.eps2 = eps * eps;
  a.reg2 = reg * reg;
  a.scale = (kernel == F3D_KERNEL_STRESSLET) ? -3.0 / (4.0 * kPi * eta) : 1.0 / (8.0 * kPi * eta);
  // the target-side items skip nothing and regularise close pairs in every mode
  if (kernel == F3D_KERNEL_OSEEN)
    return dual ? sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX, true>(a, occupancy, st)
                : sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX, false>(a, occupancy, st);
  return sym_launch_one<F3D_KERNEL_STRESSLET, F3D_SELF_SKIP_INDEX, false>(a, occupancy, st);
}

}  // namespace f3d
