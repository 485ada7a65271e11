// Symmetric evaluation of the all-pairs self-sums over one point set: the
// Oseen sum of oseen_kernel_times_density_numba (python/kernels/kernels.py:
// 214-287) and the stresslet sum of stresslet_kernel_times_normal_times_
// density_numba (kernels.py:1123-1183), j == i skipped, and the same sums
// with the pairs of one group (fiber) skipped (tstep_utils.py:653-700,
// 812-851).
//
// A pair (i, j) contributes to target i through source j's density (and
// normal) and to target j through source i's; both terms share r = x_i - x_j,
// |r| and its powers, which is most of the arithmetic.  Each unordered pair
// is therefore evaluated once:
//   Oseen:     u_i += d_j/r + (r.d_j) r/r^3,   u_j += d_i/r + (r.d_i) r/r^3
//   stresslet: v_i += (r.d_j)(r.n_j) r/r^5,    v_j -= (r.d_i)(r.n_i) r/r^5
// (the prefactor is applied once per target, as everywhere).  About 19-20
// FP64 instructions per ordered pair instead of 24-25.
//
// Decomposition: tiles of 128 points; one CTA per tile pair (I, J), I <= J.
// Thread t holds target i = 128 I + t and its partial sum in registers; tile
// J's sources are staged in shared memory (one array per component).  A warp
// meets the sources of tile J 32 at a time, rotating: at step s lane l pairs
// its target with source (l + s) mod 32 of the group, whose position and
// running source-side sum it holds in registers and hands to lane l - 1
// after the step (six shuffles per step), its density and normal read from
// shared memory.  After 32 steps lane l holds source l's sum over the warp's
// targets; the CTA's four warps' sums are added in shared memory.  Each CTA writes two partials: tile I's
// (slot J) and tile J's (slot I); a diagonal CTA (I == J) evaluates its tile
// from the target side only and writes slot I.  Each tile thus receives
// exactly T partials (T = number of tiles); the CTA that delivers the last
// one (a self-resetting counter per tile) sums them in slot order and
// writes the result, so the sum is the same run to run.
//
// Rules per pair (skip, regularisation of pairs closer than eps) are applied
// only where they can matter: in diagonal tiles, in tile pairs whose group-id
// ranges meet (SKIP_GROUP), and in tile pairs where a pair within eps is met
// (detected from the smallest r^2 of the plain pass, which is then redone).
#include <climits>

#include "f3d_common.cuh"
#include "f3d_pair_math.cuh"

namespace f3d {

constexpr int kSymTile = 128;
constexpr int kSymMaxTiles = 192;  // partial storage grows as T^2: 113 MB at 192 tiles

struct SymArgs {
  const double *x, *dens, *nrm;  // n x 3 (nrm: stresslet only)
  const int32_t *grp;            // n (SKIP_GROUP only)
  double *out;
  double *partial;               // [T][T][kSymTile][3]
  unsigned *counters;            // [T], zero on entry and on exit
  int *err;
  int64_t n;
  int ntiles;
  int accumulate;
  double eps2, reg2, scale;
};

size_t sym_partial_bytes(int64_t n) {
  const int64_t T = (n + kSymTile - 1) / kSymTile;
  return static_cast<size_t>(T) * T * kSymTile * 3 * sizeof(double);
}

bool sym_fits(int64_t n) { return (n + kSymTile - 1) / kSymTile <= kSymMaxTiles; }

template <int KIND, int MODE>
__global__ void __launch_bounds__(kSymTile) pair_sym_kernel(const SymArgs a) {
  constexpr bool kNrm = (KIND == F3D_KERNEL_STRESSLET);
  // sources of tile J, one array per component (conflict-free when the
  // lanes of a warp read different sources)
  __shared__ __align__(16) double s_x[3][kSymTile];
  __shared__ __align__(16) double s_d[3][kSymTile];
  __shared__ __align__(16) double s_n[kNrm ? 3 : 1][kSymTile];
  __shared__ int32_t s_grp[kSymTile];
  __shared__ __align__(16) double s_accj[kSymTile / 32][kSymTile][3];
  __shared__ int s_flags;
  __shared__ int s_range[kSymTile / 32][4];

  // item -> (I, J), I <= J:  item = J (J + 1) / 2 + I
  const int64_t item = blockIdx.x;
  int J = static_cast<int>((sqrt(8.0 * static_cast<double>(item) + 1.0) - 1.0) * 0.5);
  while (static_cast<int64_t>(J + 1) * (J + 2) / 2 <= item) ++J;
  while (static_cast<int64_t>(J) * (J + 1) / 2 > item) --J;
  const int I = static_cast<int>(item - static_cast<int64_t>(J) * (J + 1) / 2);
  const int T = a.ntiles;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // this thread's target, with its own density and normal for the terms it
  // sends to the sources
  const int64_t i = static_cast<int64_t>(I) * kSymTile + tid;
  const bool iv = i < a.n;
  double xi0 = 0.0, xi1 = 0.0, xi2 = 0.0, di0 = 0.0, di1 = 0.0, di2 = 0.0, ni0 = 0.0, ni1 = 0.0, ni2 = 0.0;
  int32_t gi = INT32_MIN;
  if (iv) {
    xi0 = a.x[3 * i]; xi1 = a.x[3 * i + 1]; xi2 = a.x[3 * i + 2];
    di0 = a.dens[3 * i]; di1 = a.dens[3 * i + 1]; di2 = a.dens[3 * i + 2];
    if (kNrm) { ni0 = a.nrm[3 * i]; ni1 = a.nrm[3 * i + 1]; ni2 = a.nrm[3 * i + 2]; }
    if (MODE == F3D_SELF_SKIP_GROUP) gi = a.grp[i];
  }
  // tile J's sources
  const int64_t j0 = static_cast<int64_t>(J) * kSymTile;
  const int cnt = static_cast<int>(min(static_cast<int64_t>(kSymTile), a.n - j0));
  {
    // past the end: far away, zero density and normal (their terms vanish)
    const bool sv = tid < cnt;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s_x[c][tid] = sv ? a.x[3 * (j0 + tid) + c] : 1e30;
      s_d[c][tid] = sv ? a.dens[3 * (j0 + tid) + c] : 0.0;
      if (kNrm) s_n[c][tid] = sv ? a.nrm[3 * (j0 + tid) + c] : 0.0;
    }
  }
  if (MODE == F3D_SELF_SKIP_GROUP)
    s_grp[tid] = tid < cnt ? a.grp[j0 + tid] : INT32_MIN;
  __syncthreads();

  const long long eps2_bits = __double_as_longlong(a.eps2);
  const int eps2_hi = __double2hiint(a.eps2);
  const double reg2 = a.reg2;
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;

  if (I == J) {
    // one tile: every ordered pair from the target's side, with the rules
    for (int s = 0; s < cnt; ++s) {
      const double dx = xi0 - s_x[0][s], dy = xi1 - s_x[1][s], dz = xi2 - s_x[2][s];
      double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      bool skip = (s == tid);
      if (MODE == F3D_SELF_SKIP_GROUP) skip = skip || (s_grp[s] == gi);
      const bool close = !skip && (__double_as_longlong(r2) < eps2_bits);
      r2 = regularise(r2, close, reg2);
      const double d0 = s_d[0][s], d1 = s_d[1][s], d2 = s_d[2][s];
      if (KIND == F3D_KERNEL_OSEEN) {
        double ri = rsqrt_refined(r2);
        ri = skip ? 0.0 : ri;
        const double g = ri * ri * ri * fma(dx, d0, fma(dy, d1, dz * d2));
        acc0 = fma(g, dx, fma(ri, d0, acc0));
        acc1 = fma(g, dy, fma(ri, d1, acc1));
        acc2 = fma(g, dz, fma(ri, d2, acc2));
      } else {
        const double rd = fma(dx, d0, fma(dy, d1, dz * d2));
        const double rn = fma(dx, s_n[0][s], fma(dy, s_n[1][s], dz * s_n[2][s]));
        double f = times_rsqrt5(rd * rn, r2);
        f = skip ? 0.0 : f;
        acc0 = fma(f, dx, acc0);
        acc1 = fma(f, dy, acc1);
        acc2 = fma(f, dz, acc2);
      }
    }
  } else {
    // group ranges of the two tiles (SKIP_GROUP): pairs of one group can
    // occur only if they meet
    bool careful = false;
    if (MODE == F3D_SELF_SKIP_GROUP) {
      // group-id ranges of tile I (the targets) and tile J (the sources)
      int tlo = iv ? gi : INT32_MAX, thi = iv ? gi : INT32_MIN;
      int slo = tid < cnt ? s_grp[tid] : INT32_MAX, shi = tid < cnt ? s_grp[tid] : INT32_MIN;
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
      __syncthreads();
      int TL = s_range[0][0], TH = s_range[0][1], SL0 = s_range[0][2], SH = s_range[0][3];
#pragma unroll
      for (int w = 1; w < kSymTile / 32; ++w) {
        TL = min(TL, s_range[w][0]); TH = max(TH, s_range[w][1]);
        SL0 = min(SL0, s_range[w][2]); SH = max(SH, s_range[w][3]);
      }
      careful = (TL <= SH && SL0 <= TH);
    }
    // two passes at most: the plain one, then (if a rule can matter) the
    // careful one from scratch
    for (int pass = careful ? 1 : 0; pass < 2; ++pass) {
      const bool rules = (pass == 1);
      acc0 = acc1 = acc2 = 0.0;
      int hmin = INT32_MAX;
      for (int sb = 0; sb < cnt; sb += 32) {
        // the group's source at this lane: position and source-side sum rotate
        int m = lane;
        double px = s_x[0][sb + m], py = s_x[1][sb + m], pz = s_x[2][sb + m];
        double aj0 = 0.0, aj1 = 0.0, aj2 = 0.0;
        for (int st = 0; st < 32; ++st) {
          const int js = sb + m;
          const double dx = xi0 - px, dy = xi1 - py, dz = xi2 - pz;
          double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
          bool skip = !iv;
          if (rules) {
            if (MODE == F3D_SELF_SKIP_GROUP) skip = skip || (s_grp[js] == gi);
            if (!skip && __double_as_longlong(r2) < eps2_bits) r2 += reg2;
          } else if (iv) {
            hmin = min(hmin, __double2hiint(r2));
          }
          const double d0 = s_d[0][js], d1 = s_d[1][js], d2 = s_d[2][js];
          if (KIND == F3D_KERNEL_OSEEN) {
            double ri = rsqrt_refined(r2);
            ri = skip ? 0.0 : ri;
            const double ri3 = ri * ri * ri;
            const double g = ri3 * fma(dx, d0, fma(dy, d1, dz * d2));
            const double h = ri3 * fma(dx, di0, fma(dy, di1, dz * di2));
            acc0 = fma(g, dx, fma(ri, d0, acc0));
            acc1 = fma(g, dy, fma(ri, d1, acc1));
            acc2 = fma(g, dz, fma(ri, d2, acc2));
            aj0 = fma(h, dx, fma(ri, di0, aj0));
            aj1 = fma(h, dy, fma(ri, di1, aj1));
            aj2 = fma(h, dz, fma(ri, di2, aj2));
          } else {
            double R5 = rsqrt5(r2);
            R5 = skip ? 0.0 : R5;
            const double n0 = s_n[0][js], n1 = s_n[1][js], n2 = s_n[2][js];
            const double f = (fma(dx, d0, fma(dy, d1, dz * d2)) * fma(dx, n0, fma(dy, n1, dz * n2))) * R5;
            const double h = (fma(dx, di0, fma(dy, di1, dz * di2)) * fma(dx, ni0, fma(dy, ni1, dz * ni2))) * R5;
            acc0 = fma(f, dx, acc0);
            acc1 = fma(f, dy, acc1);
            acc2 = fma(f, dz, acc2);
            aj0 = fma(-h, dx, aj0);
            aj1 = fma(-h, dy, aj1);
            aj2 = fma(-h, dz, aj2);
          }
          // hand the source (position and its running sum) to lane - 1
          const int from = (lane + 1) & 31;
          px = __shfl_sync(0xffffffffu, px, from);
          py = __shfl_sync(0xffffffffu, py, from);
          pz = __shfl_sync(0xffffffffu, pz, from);
          aj0 = __shfl_sync(0xffffffffu, aj0, from);
          aj1 = __shfl_sync(0xffffffffu, aj1, from);
          aj2 = __shfl_sync(0xffffffffu, aj2, from);
          m = (m + 1) & 31;
        }
        // after a full turn lane l holds source sb + l again
        if (sb + lane < cnt) {
          s_accj[warp][sb + lane][0] = aj0;
          s_accj[warp][sb + lane][1] = aj1;
          s_accj[warp][sb + lane][2] = aj2;
        }
      }
      // a pair within eps met by the plain pass: redo with the rules
      if (pass == 0 && !__syncthreads_or(hmin <= eps2_hi)) break;
      if (pass == 0) __syncthreads();
    }
    __syncthreads();
    // tile J's partial from this CTA: the four warps' sums, in warp order
    if (tid < cnt) {
      double* pj = a.partial + ((static_cast<int64_t>(J) * T + I) * kSymTile + tid) * 3;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        double v = s_accj[0][tid][m];
#pragma unroll
        for (int w = 1; w < kSymTile / 32; ++w) v += s_accj[w][tid][m];
        __stcg(pj + m, v);
      }
    }
  }
  // tile I's partial from this CTA
  {
    double *pi = a.partial + ((static_cast<int64_t>(I) * T + J) * kSymTile + tid) * 3;
    __stcg(pi, acc0);
    __stcg(pi + 1, acc1);
    __stcg(pi + 2, acc2);
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    int f = 0;
    if (atomicAdd(&a.counters[I], 1u) == static_cast<unsigned>(T - 1)) f |= 1;
    if (I != J && atomicAdd(&a.counters[J], 1u) == static_cast<unsigned>(T - 1)) f |= 2;
    s_flags = f;
  }
  __syncthreads();
  const int flags = s_flags;
  for (int which = 0; which < 2; ++which) {
    if (!(flags & (1 << which))) continue;
    __threadfence();
    const int X = which == 0 ? I : J;
    const int64_t t = static_cast<int64_t>(X) * kSymTile + tid;
    if (t < a.n) {
      double v0 = 0.0, v1 = 0.0, v2 = 0.0;
      for (int slot = 0; slot < T; ++slot) {
        const double *p = a.partial + ((static_cast<int64_t>(X) * T + slot) * kSymTile + tid) * 3;
        v0 += __ldcg(p);
        v1 += __ldcg(p + 1);
        v2 += __ldcg(p + 2);
      }
      v0 *= a.scale; v1 *= a.scale; v2 *= a.scale;
      double *o = a.out + 3 * t;
      if (a.accumulate) { v0 += o[0]; v1 += o[1]; v2 += o[2]; }
      o[0] = v0; o[1] = v1; o[2] = v2;
    }
    if (tid == 0) a.counters[X] = 0u;
  }
}

template <int KIND, int MODE>
static int sym_launch_one(const SymArgs &a, int *occupancy, cudaStream_t st) {
  auto kfn = pair_sym_kernel<KIND, MODE>;
  if (occupancy)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, kfn, kSymTile, 0) == cudaSuccess
               ? F3D_OK
               : F3D_ERR_CUDA;
  const int64_t items = static_cast<int64_t>(a.ntiles) * (a.ntiles + 1) / 2;
  kfn<<<static_cast<unsigned>(items), kSymTile, 0, st>>>(a);
  return launch_status();
}

// The symmetric self-sum (kernel OSEEN or STRESSLET, FP64, mode SKIP_INDEX or
// SKIP_GROUP) over n points; partial: sym_partial_bytes(n) of workspace;
// counters: the pair workspace's counter region.  With occupancy non-null,
// only reports the kernel's resident CTAs per SM.
int pair_sym_launch(int kernel, int self_mode, const double *x, const double *dens, const double *nrm,
                    const int32_t *grp, double *out, int64_t n, double eta, double reg, double eps, int accumulate,
                    double *partial, unsigned *counters, int *occupancy, cudaStream_t st) {
  SymArgs a{};
  a.x = x; a.dens = dens; a.nrm = nrm; a.grp = grp; a.out = out;
  a.partial = partial; a.counters = counters; a.err = device_error_word();
  a.n = n;
  a.ntiles = static_cast<int>((n + kSymTile - 1) / kSymTile);
  a.accumulate = accumulate ? 1 : 0;
  a.eps2 = eps * eps;
  a.reg2 = reg * reg;
  a.scale = (kernel == F3D_KERNEL_STRESSLET) ? -3.0 / (4.0 * kPi * eta) : 1.0 / (8.0 * kPi * eta);
  if (kernel == F3D_KERNEL_OSEEN) {
    return self_mode == F3D_SELF_SKIP_INDEX ? sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX>(a, occupancy, st)
                                            : sym_launch_one<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_GROUP>(a, occupancy, st);
  }
  return self_mode == F3D_SELF_SKIP_INDEX ? sym_launch_one<F3D_KERNEL_STRESSLET, F3D_SELF_SKIP_INDEX>(a, occupancy, st)
                                          : sym_launch_one<F3D_KERNEL_STRESSLET, F3D_SELF_SKIP_GROUP>(a, occupancy, st);
}

}  // namespace f3d
