// All-pairs Stokes sums on sm_100a: Oseen (Stokeslet), stresslet (double
// layer) and rotlet, source -> target, FP64 or FP32-compensated.
//
// Reference semantics (fiber3d python/kernels/kernels.py):
//   oseen_kernel_source_target_numba            :794-846   (A1)
//   oseen_kernel_times_density_numba            :214-287   (A2, j == i skipped)
//   rotlet_kernel_source_target_numba           :856-908   (A6)
//   stresslet_kernel_times_normal_times_density :1123-1183 (A4, j == i skipped)
//   stresslet_kernel_source_target_numba        :1186-1217 (A3)
//   traction_kernel_times_normal_times_density  :1221-1264 (the normal of the target)
//   oseen_kernel_source_target_pycuda           :849 -> kernels_pycuda.py:22-66
//                                               (pairs closer than eps skipped)
// r = x_target - x_source.  A pair with |r| < epsilon_distance uses
// sqrt(|r|^2 + reg^2) in place of |r| (F3D_SELF_SKIP_CLOSE: contributes
// zero instead).  The prefactor (1/(8 pi eta) or -3/(4 pi eta)) is applied
// once per target.
//
// Design.  One CTA owns TPB = (kBlock / SL) * TPT targets (held in registers)
// and a contiguous range of source tiles (grid.y = source split).  Source
// tiles of kTile points are staged in shared memory with 1-D bulk copies
// (cp.async.bulk, TMA engine) completing on an mbarrier, double buffered, so
// the copy of tile i+2 overlaps the arithmetic on tile i.  Within a tile a
// target group of SL lanes strides the sources; lanes are reduced with warp
// shuffles.  With grid.y > 1 each CTA writes a partial sum to the workspace
// and the last CTA of a target block (self-resetting counter) adds the
// partials in split order, so results are deterministic run to run.
#include <algorithm>
#include <climits>
#include <type_traits>

#include "f3d_common.cuh"
#include "f3d_pair_math.cuh"

namespace f3d {

constexpr int kBlock = 128;  // threads per CTA
constexpr int kTile = 128;   // sources per staged tile

struct PairArgs {
  const double *rs, *rt, *dens, *nrm;  // nrm: source normals (traction: target normals)
  const double *dens2;  // dual sums: the second density (FP64 only)
  const float *packed;  // FP32C: [ns][12] packed source records
  const int32_t *gs, *gt;
  double *out;
  double *out2;             // dual sums: the second output
  double *partial;          // [nsplit][nt][3] (dual: a second such array follows)
  unsigned int *counters;   // [gridDim.x], zero on entry, zero on exit
  int *err;
  int64_t ns, nt;
  int64_t tiles_per_split;  // full tiles per split
  int nsplit;
  int use_tma;
  int accumulate;
  double eps2, reg2, scale;
  uint64_t wait_ns;  // limit of each bounded mbarrier wait
  int *occupancy;    // host: when set, report CTAs per SM of the chosen kernel instead of launching
};

// Shared-memory layout of one stage.
template <int KIND, int MODE, int PREC, bool DUAL = false>
struct Stage {
  static constexpr bool kNrm = (KIND == F3D_KERNEL_STRESSLET);
  static constexpr bool kGrp = (MODE == F3D_SELF_SKIP_GROUP);
  // FP64: pos[3T] dens[3T] (nrm[3T]) (dens2[3T]) (grp[T]);  FP32C: rec[12T] (grp[T])
  static constexpr size_t off_pos = 0;
  static constexpr size_t off_dens = 24 * kTile;
  static constexpr size_t off_nrm = 48 * kTile;
  static constexpr size_t off_dens2 = (kNrm ? 72 : 48) * kTile;
  static constexpr size_t off_rec = 0;
  static constexpr size_t data_bytes =
      (PREC == F3D_FP64) ? (kNrm ? 72 * kTile : 48 * kTile) + (DUAL ? 24 * kTile : 0) : 48 * kTile;
  static constexpr size_t off_grp = data_bytes;
  static constexpr size_t bytes = ((data_bytes + (kGrp ? 4 * kTile : 0)) + 127) / 128 * 128;
};

// Bytes of the FP64 accumulator snapshot: [TPT][3] (DUAL: twice) doubles per
// thread.
template <int PREC, int TPT, bool DUAL>
constexpr size_t snapshot_bytes() {
  return PREC == F3D_FP64 ? static_cast<size_t>(TPT) * 3 * (DUAL ? 2 : 1) * 8 * kBlock : 0;
}

template <int KIND, int MODE, int PREC, int TPT, bool DUAL = false>
constexpr size_t pair_smem_bytes() {
  return 128 + 2 * Stage<KIND, MODE, PREC, DUAL>::bytes + snapshot_bytes<PREC, TPT, DUAL>();
}

__device__ __forceinline__ void two_sum(float &s, float &c, float x) {
  const float t = s + x;
  const float bp = t - s;
  const float e = (s - (t - bp)) + (x - bp);
  s = t;
  c += e;
}

// Packed two-lane FP32 arithmetic (PTX f32x2, sm_100): one instruction
// applies the same IEEE round-to-nearest operation to two floats held in a
// 64-bit register pair, so a pair of sources costs one issue slot per
// operation instead of two.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void up2(f32x2 v, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// DUAL (FP64 Oseen only): the same pairs summed against two densities, dens
// into out and dens2 into out2, each with exactly the arithmetic of a single
// sum -- the geometry (r, 1/r, 1/r^3) is computed once for both.
template <int KIND, int MODE, int PREC, int TPT, int SL, bool DUAL = false>
__global__ void __launch_bounds__(kBlock, (PREC == F3D_FP64 && !DUAL) ? ((TPT == 1) ? 7 : (TPT == 2) ? 5 : 3) : 1)
    pair_kernel(const PairArgs a) {
  static_assert(!DUAL || (PREC == F3D_FP64 && KIND == F3D_KERNEL_OSEEN), "dual sums: FP64 Oseen");
  using St = Stage<KIND, MODE, PREC, DUAL>;
  constexpr int TG = kBlock / SL;
  constexpr int TPB = TG * TPT;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  unsigned char *stages = smem + 128;

  const int tid = threadIdx.x;
  const int tg = tid / SL;
  const int sl = tid % SL;
  const int64_t tb = static_cast<int64_t>(blockIdx.x) * TPB;

  // ---- targets in registers -------------------------------------------
  constexpr bool kTrac = (KIND == F3D_KERNEL_TRACTION);
  double txd[TPT], tyd[TPT], tzd[TPT];
  double tn0[TPT], tn1[TPT], tn2[TPT];  // traction: the target's normal
  float txh[TPT], tyh[TPT], tzh[TPT], txl[TPT], tyl[TPT], tzl[TPT];
  int32_t tgrp[TPT];
  int64_t tidx[TPT];
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    const int64_t t = tb + k * TG + tg;
    tidx[k] = t;
    double x = 0.0, y = 0.0, z = 0.0;
    int32_t g = -1;
    tn0[k] = tn1[k] = tn2[k] = 0.0;
    if (t < a.nt) {
      x = a.rt[3 * t + 0];
      y = a.rt[3 * t + 1];
      z = a.rt[3 * t + 2];
      if (MODE == F3D_SELF_SKIP_GROUP) g = a.gt[t];
      if (kTrac) {
        tn0[k] = a.nrm[3 * t + 0];
        tn1[k] = a.nrm[3 * t + 1];
        tn2[k] = a.nrm[3 * t + 2];
      }
    }
    tgrp[k] = g;
    if (PREC == F3D_FP64) {
      txd[k] = x; tyd[k] = y; tzd[k] = z;
    } else {
      txh[k] = static_cast<float>(x); txl[k] = static_cast<float>(x - static_cast<double>(txh[k]));
      tyh[k] = static_cast<float>(y); tyl[k] = static_cast<float>(y - static_cast<double>(tyh[k]));
      tzh[k] = static_cast<float>(z); tzl[k] = static_cast<float>(z - static_cast<double>(tzh[k]));
    }
  }
  // FP32C: each target coordinate (and traction normal) twice, against a
  // pair of sources
  f32x2 pxh[TPT], pyh[TPT], pzh[TPT], pxl[TPT], pyl[TPT], pzl[TPT];
  f32x2 pn0[TPT], pn1[TPT], pn2[TPT];
  if (PREC != F3D_FP64) {
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      pxh[k] = pk2(txh[k], txh[k]); pyh[k] = pk2(tyh[k], tyh[k]); pzh[k] = pk2(tzh[k], tzh[k]);
      pxl[k] = pk2(txl[k], txl[k]); pyl[k] = pk2(tyl[k], tyl[k]); pzl[k] = pk2(tzl[k], tzl[k]);
      const float m0 = static_cast<float>(tn0[k]), m1 = static_cast<float>(tn1[k]),
                  m2 = static_cast<float>(tn2[k]);
      pn0[k] = pk2(m0, m0); pn1[k] = pk2(m1, m1); pn2[k] = pk2(m2, m2);
    }
  }

  double acc[TPT][3], acc2[TPT][3];
  float fs[TPT][3], fc[TPT][3];
  f32x2 ft[TPT][3];  // FP32C tile sums: {even sources, odd sources}
#pragma unroll
  for (int k = 0; k < TPT; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      acc[k][c] = 0.0; acc2[k][c] = 0.0; fs[k][c] = 0.f; fc[k][c] = 0.f; ft[k][c] = 0ull;
    }

  const double reg2 = a.reg2;
  const long long eps2_bits = __double_as_longlong(a.eps2);
  const float eps2f = static_cast<float>(a.eps2), reg2f = static_cast<float>(a.reg2);

  // ---- FP64: which tiles need the per-pair rules ----------------------------
  // A tile runs the "careful" loop (skip rule, regularisation of close pairs,
  // per pair) only where a skipped pair can occur: for SKIP_INDEX a tile whose
  // source indices meet this warp's target indices, for SKIP_GROUP one whose
  // group-id range meets this warp's, always for SKIP_CLOSE and for a tail
  // tile.  Every other tile runs the plain arithmetic and tracks the smallest
  // r^2 it met (its high word, on the integer pipe); if that could be below
  // eps^2, the thread's accumulators are restored from a shared-memory
  // snapshot and the tile is redone carefully.  The result is the careful
  // loop's in every case.
  const int lane = tid & 31;
  const int eps2_hi = __double2hiint(a.eps2);
  int64_t w_lo = INT64_MAX, w_hi = INT64_MIN;  // SKIP_INDEX: this warp's target index range
  int w_glo = INT32_MAX, w_ghi = INT32_MIN;    // SKIP_GROUP: its target group-id range
  if (PREC == F3D_FP64 && MODE == F3D_SELF_SKIP_INDEX) {
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      w_lo = min(w_lo, tidx[k]);
      w_hi = max(w_hi, tidx[k]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      w_lo = min(w_lo, static_cast<int64_t>(__shfl_xor_sync(0xffffffffu, static_cast<long long>(w_lo), off)));
      w_hi = max(w_hi, static_cast<int64_t>(__shfl_xor_sync(0xffffffffu, static_cast<long long>(w_hi), off)));
    }
  }
  if (PREC == F3D_FP64 && MODE == F3D_SELF_SKIP_GROUP) {
    int glo = INT32_MAX, ghi = INT32_MIN;
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      glo = min(glo, tgrp[k]);
      ghi = max(ghi, tgrp[k]);
    }
    w_glo = __reduce_min_sync(0xffffffffu, glo);
    w_ghi = __reduce_max_sync(0xffffffffu, ghi);
  }
  double *snap = reinterpret_cast<double *>(stages + 2 * St::bytes) + tid;  // [TPT*3*(1+DUAL)][kBlock]

  // ---- one tile of `cnt` sources starting at global index `sbase` --------
  auto compute_tile = [&](const unsigned char *buf, int cnt, int64_t sbase) {
    if (PREC == F3D_FP64) {
      const double *pos = reinterpret_cast<const double *>(buf + St::off_pos);
      const double *den = reinterpret_cast<const double *>(buf + St::off_dens);
      const double *nrm = reinterpret_cast<const double *>(buf + St::off_nrm);
      const double *den2 = reinterpret_cast<const double *>(buf + St::off_dens2);
      const int32_t *grp = reinterpret_cast<const int32_t *>(buf + St::off_grp);
      // source s against this thread's targets; CAREFUL applies the skip and
      // close-pair rules, else the minimum high word of r^2 goes to hmin
      auto one_source = [&](int s, auto careful_tag, int &hmin) {
        constexpr bool CAREFUL = decltype(careful_tag)::value;
        const double sx = pos[3 * s], sy = pos[3 * s + 1], sz = pos[3 * s + 2];
        const double d0 = den[3 * s], d1 = den[3 * s + 1], d2 = den[3 * s + 2];
        double n0 = 0.0, n1 = 0.0, n2 = 0.0;
        if (KIND == F3D_KERNEL_STRESSLET) { n0 = nrm[3 * s]; n1 = nrm[3 * s + 1]; n2 = nrm[3 * s + 2]; }
        double e0 = 0.0, e1 = 0.0, e2 = 0.0;
        if (DUAL) { e0 = den2[3 * s]; e1 = den2[3 * s + 1]; e2 = den2[3 * s + 2]; }
        int32_t sg = 0;
        if (CAREFUL && MODE == F3D_SELF_SKIP_GROUP) sg = grp[s];
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
          const double dx = txd[k] - sx, dy = tyd[k] - sy, dz = tzd[k] - sz;
          double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
          // skipped pairs (and, in SKIP_CLOSE, close ones) are dropped by a
          // select on the final factor, so their r2 may stay 0
          bool skip = false;
          if (CAREFUL) {
            if (MODE == F3D_SELF_SKIP_INDEX) skip = (sbase + s == tidx[k]);
            if (MODE == F3D_SELF_SKIP_GROUP) skip = (sg == tgrp[k]);
            const bool close = !skip && (__double_as_longlong(r2) < eps2_bits);
            if (MODE == F3D_SELF_SKIP_CLOSE) skip = close;
            else r2 = regularise(r2, close, reg2);
          } else {
            hmin = min(hmin, __double2hiint(r2));
          }
          constexpr bool kSel = CAREFUL && (MODE != F3D_SELF_REGULARISE);
          if (KIND == F3D_KERNEL_OSEEN || KIND == F3D_KERNEL_ROTLET) {
            double ri = rsqrt_refined(r2);
            if (kSel) ri = skip ? 0.0 : ri;
            const double ri3 = ri * ri * ri;
            if (KIND == F3D_KERNEL_OSEEN) {
              const double rf = fma(dx, d0, fma(dy, d1, dz * d2));
              const double g = ri3 * rf;
              acc[k][0] = fma(g, dx, fma(ri, d0, acc[k][0]));
              acc[k][1] = fma(g, dy, fma(ri, d1, acc[k][1]));
              acc[k][2] = fma(g, dz, fma(ri, d2, acc[k][2]));
              if (DUAL) {
                const double re = fma(dx, e0, fma(dy, e1, dz * e2));
                const double g2 = ri3 * re;
                acc2[k][0] = fma(g2, dx, fma(ri, e0, acc2[k][0]));
                acc2[k][1] = fma(g2, dy, fma(ri, e1, acc2[k][1]));
                acc2[k][2] = fma(g2, dz, fma(ri, e2, acc2[k][2]));
              }
            } else {
              acc[k][0] = fma(ri3, dz * d1 - dy * d2, acc[k][0]);
              acc[k][1] = fma(ri3, dx * d2 - dz * d0, acc[k][1]);
              acc[k][2] = fma(ri3, dy * d0 - dx * d1, acc[k][2]);
            }
          } else {
            // stresslet: normal of the source; traction: normal of the target
            const double m0 = kTrac ? tn0[k] : n0, m1 = kTrac ? tn1[k] : n1, m2 = kTrac ? tn2[k] : n2;
            const double rd = fma(dx, d0, fma(dy, d1, dz * d2));
            const double rn = fma(dx, m0, fma(dy, m1, dz * m2));
            double f0 = times_rsqrt5(rd * rn, r2);
            if (kSel) f0 = skip ? 0.0 : f0;
            acc[k][0] = fma(f0, dx, acc[k][0]);
            acc[k][1] = fma(f0, dy, acc[k][1]);
            acc[k][2] = fma(f0, dz, acc[k][2]);
          }
        }
      };
      bool careful = (MODE == F3D_SELF_SKIP_CLOSE) || (cnt < kTile);
      if (MODE == F3D_SELF_SKIP_INDEX) careful = careful || (sbase <= w_hi && sbase + cnt > w_lo);
      if (MODE == F3D_SELF_SKIP_GROUP && !careful) {
        int glo = INT32_MAX, ghi = INT32_MIN;
        for (int s = lane; s < cnt; s += 32) {
          glo = min(glo, grp[s]);
          ghi = max(ghi, grp[s]);
        }
        glo = __reduce_min_sync(0xffffffffu, glo);
        ghi = __reduce_max_sync(0xffffffffu, ghi);
        careful = (glo <= w_ghi && ghi >= w_glo);
      }
      int hmin = INT32_MAX;
      if (!careful) {
#pragma unroll
        for (int k = 0; k < TPT; ++k)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            snap[(k * 3 + c) * kBlock] = acc[k][c];
            if (DUAL) snap[((TPT + k) * 3 + c) * kBlock] = acc2[k][c];
          }
#pragma unroll 1
        for (int s = sl; s < kTile; s += SL) one_source(s, std::false_type{}, hmin);
        if (hmin <= eps2_hi) {
          // a pair within eps (or r^2 = 0) met without the rules: redo the tile
#pragma unroll
          for (int k = 0; k < TPT; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              acc[k][c] = snap[(k * 3 + c) * kBlock];
              if (DUAL) acc2[k][c] = snap[((TPT + k) * 3 + c) * kBlock];
            }
          careful = true;
        }
      }
      if (careful) {
        for (int s = sl; s < cnt; s += SL) one_source(s, std::true_type{}, hmin);
      }
    } else {
      // sources in pairs (2q, 2q + 1); a record of 6 x 16 bytes holds
      // {xh,yh},{zh,xl},{yl,zl},{d0,d1},{d2,n0},{n1,n2}, each component as
      // {even, odd}.  An odd count ends on the packer's pad source (far
      // away, zero density), whose terms are exactly zero.
      const ulonglong2 *rec = reinterpret_cast<const ulonglong2 *>(buf + St::off_rec);
      const int npair = (cnt + 1) >> 1;
      for (int q = sl; q < npair; q += SL) {
        const ulonglong2 u0 = rec[6 * q], u1 = rec[6 * q + 1], u2 = rec[6 * q + 2];
        const ulonglong2 u3 = rec[6 * q + 3], u4 = rec[6 * q + 4];
        const f32x2 sxh = u0.x, syh = u0.y, szh = u1.x, sxl = u1.y, syl = u2.x, szl = u2.y;
        const f32x2 d0 = u3.x, d1 = u3.y, d2 = u4.x;
        f32x2 n0 = 0ull, n1 = 0ull, n2 = 0ull;
        if (KIND == F3D_KERNEL_STRESSLET) {
          const ulonglong2 u5 = rec[6 * q + 5];
          n0 = u4.y; n1 = u5.x; n2 = u5.y;
        }
        int2 sg = make_int2(0, 0);
        if (MODE == F3D_SELF_SKIP_GROUP) sg = reinterpret_cast<const int2 *>(buf + St::off_grp)[q];
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
          const f32x2 dx = add2(sub2(pxh[k], sxh), sub2(pxl[k], sxl));
          const f32x2 dy = add2(sub2(pyh[k], syh), sub2(pyl[k], syl));
          const f32x2 dz = add2(sub2(pzh[k], szh), sub2(pzl[k], szl));
          float ra, rb;
          up2(fma2(dx, dx, fma2(dy, dy, mul2(dz, dz))), ra, rb);
          // SKIP_CLOSE drops r <= eps here, so that a coincident pair is
          // dropped even when eps^2 underflows in float
          const bool ca = (MODE == F3D_SELF_SKIP_CLOSE) ? !(ra > eps2f) : (ra < eps2f);
          const bool cb = (MODE == F3D_SELF_SKIP_CLOSE) ? !(rb > eps2f) : (rb < eps2f);
          if (MODE != F3D_SELF_SKIP_CLOSE) {
            ra = ca ? ra + reg2f : ra;
            rb = cb ? rb + reg2f : rb;
          }
          float ia = rsqrtf(ra), ib = rsqrtf(rb);
          if (MODE == F3D_SELF_SKIP_CLOSE) {
            ia = ca ? 0.f : ia;
            ib = cb ? 0.f : ib;
          }
          if (MODE == F3D_SELF_SKIP_INDEX) {
            const int64_t s0 = sbase + 2 * q;
            ia = (s0 == tidx[k]) ? 0.f : ia;
            ib = (s0 + 1 == tidx[k]) ? 0.f : ib;
          }
          if (MODE == F3D_SELF_SKIP_GROUP) {
            ia = (sg.x == tgrp[k]) ? 0.f : ia;
            ib = (sg.y == tgrp[k]) ? 0.f : ib;
          }
          const f32x2 ri = pk2(ia, ib);
          if (KIND == F3D_KERNEL_OSEEN) {
            const f32x2 rf = fma2(dx, d0, fma2(dy, d1, mul2(dz, d2)));
            const f32x2 g = mul2(mul2(mul2(ri, ri), ri), rf);
            ft[k][0] = fma2(g, dx, fma2(ri, d0, ft[k][0]));
            ft[k][1] = fma2(g, dy, fma2(ri, d1, ft[k][1]));
            ft[k][2] = fma2(g, dz, fma2(ri, d2, ft[k][2]));
          } else if (KIND == F3D_KERNEL_ROTLET) {
            const f32x2 g = mul2(mul2(ri, ri), ri);
            ft[k][0] = fma2(g, sub2(mul2(dz, d1), mul2(dy, d2)), ft[k][0]);
            ft[k][1] = fma2(g, sub2(mul2(dx, d2), mul2(dz, d0)), ft[k][1]);
            ft[k][2] = fma2(g, sub2(mul2(dy, d0), mul2(dx, d1)), ft[k][2]);
          } else {
            const f32x2 ri2 = mul2(ri, ri);
            const f32x2 rd = fma2(dx, d0, fma2(dy, d1, mul2(dz, d2)));
            const f32x2 rn = kTrac ? fma2(dx, pn0[k], fma2(dy, pn1[k], mul2(dz, pn2[k])))
                                   : fma2(dx, n0, fma2(dy, n1, mul2(dz, n2)));
            const f32x2 f0 = mul2(mul2(rd, rn), mul2(mul2(ri2, ri2), ri));
            ft[k][0] = fma2(f0, dx, ft[k][0]);
            ft[k][1] = fma2(f0, dy, ft[k][1]);
            ft[k][2] = fma2(f0, dz, ft[k][2]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < TPT; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float e, o;
          up2(ft[k][c], e, o);
          two_sum(fs[k][c], fc[k][c], e + o);
          ft[k][c] = 0ull;
        }
    }
  };

  // ---- plain (non-bulk) cooperative tile load ----------------------------
  auto load_plain = [&](unsigned char *buf, int64_t s0, int cnt) {
    if (PREC == F3D_FP64) {
      double *pos = reinterpret_cast<double *>(buf + St::off_pos);
      double *den = reinterpret_cast<double *>(buf + St::off_dens);
      double *nrm = reinterpret_cast<double *>(buf + St::off_nrm);
      double *den2 = reinterpret_cast<double *>(buf + St::off_dens2);
      for (int i = tid; i < 3 * cnt; i += kBlock) {
        pos[i] = a.rs[3 * s0 + i];
        den[i] = a.dens[3 * s0 + i];
        if (KIND == F3D_KERNEL_STRESSLET) nrm[i] = a.nrm[3 * s0 + i];
        if (DUAL) den2[i] = a.dens2[3 * s0 + i];
      }
    } else {
      // whole source pairs (the packer pads an odd count)
      float *rec = reinterpret_cast<float *>(buf + St::off_rec);
      const int cp = (cnt + 1) & ~1;
      for (int i = tid; i < 12 * cp; i += kBlock) rec[i] = a.packed[12 * s0 + i];
    }
    if (MODE == F3D_SELF_SKIP_GROUP) {
      int32_t *g = reinterpret_cast<int32_t *>(buf + St::off_grp);
      for (int i = tid; i < cnt; i += kBlock) g[i] = a.gs[s0 + i];
      if ((cnt & 1) && tid == 0) g[cnt] = INT32_MIN;  // the pad source's group
    }
  };

  // ---- bulk-copy issue of one full tile (thread 0 only) ------------------
  auto issue_tile = [&](int st, int64_t tile) {
    unsigned char *buf = stages + st * St::bytes;
    const int64_t s0 = tile * kTile;
    uint32_t bytes = (PREC == F3D_FP64) ? (St::kNrm ? 72u : 48u) * kTile : 48u * kTile;
    if (DUAL) bytes += 24u * kTile;
    if (MODE == F3D_SELF_SKIP_GROUP) bytes += 4u * kTile;
    mbar_arrive_expect_tx(&bars[st], bytes);
    if (PREC == F3D_FP64) {
      bulk_copy_g2s(buf + St::off_pos, a.rs + 3 * s0, 24u * kTile, &bars[st]);
      bulk_copy_g2s(buf + St::off_dens, a.dens + 3 * s0, 24u * kTile, &bars[st]);
      if (KIND == F3D_KERNEL_STRESSLET)
        bulk_copy_g2s(buf + St::off_nrm, a.nrm + 3 * s0, 24u * kTile, &bars[st]);
      if (DUAL) bulk_copy_g2s(buf + St::off_dens2, a.dens2 + 3 * s0, 24u * kTile, &bars[st]);
    } else {
      bulk_copy_g2s(buf + St::off_rec, a.packed + 12 * s0, 48u * kTile, &bars[st]);
    }
    if (MODE == F3D_SELF_SKIP_GROUP)
      bulk_copy_g2s(buf + St::off_grp, a.gs + s0, 4u * kTile, &bars[st]);
  };

  // ---- source range of this split ---------------------------------------
  const int split = blockIdx.y;
  const int64_t nfull = a.ns / kTile;
  const int64_t tile0 = static_cast<int64_t>(split) * a.tiles_per_split;
  const int64_t tile1 = min(tile0 + a.tiles_per_split, nfull);
  const int64_t ntl = (tile1 > tile0) ? (tile1 - tile0) : 0;
  const int tail = static_cast<int>(a.ns - nfull * kTile);
  const bool has_tail = (split == a.nsplit - 1) && tail > 0;

  bool ok_all = true;
  if (a.use_tma) {
    if (tid == 0) {
      mbar_init(&bars[0], 1);
      mbar_init(&bars[1], 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
      for (int st = 0; st < 2 && st < ntl; ++st) issue_tile(st, tile0 + st);
    }
    for (int64_t i = 0; i < ntl; ++i) {
      const int st = static_cast<int>(i & 1);
      const uint32_t parity = static_cast<uint32_t>((i >> 1) & 1);
      const bool ok = mbar_wait_bounded(&bars[st], parity, a.wait_ns);
      if (ok) compute_tile(stages + st * St::bytes, kTile, (tile0 + i) * kTile);
      if (__syncthreads_or(!ok)) { ok_all = false; break; }
      if (tid == 0 && i + 2 < ntl) {
        fence_proxy_async_smem();
        issue_tile(st, tile0 + i + 2);
      }
    }
    if (!ok_all) {
      // Give copies still in flight a bounded chance to land before exit.
      if (tid == 0) {
        record_error(a.err, F3D_ERR_TIMEOUT);
        for (int st = 0; st < 2; ++st) (void)mbar_wait_bounded(&bars[st], 0, a.wait_ns);
      }
      return;
    }
  } else {
    for (int64_t i = 0; i < ntl; ++i) {
      load_plain(stages, (tile0 + i) * kTile, kTile);
      __syncthreads();
      compute_tile(stages, kTile, (tile0 + i) * kTile);
      __syncthreads();
    }
  }
  if (has_tail) {
    load_plain(stages, nfull * kTile, tail);
    __syncthreads();
    compute_tile(stages, tail, nfull * kTile);
  }

  // ---- combine lanes of a target group -----------------------------------
  double res[TPT][3], res2[TPT][3];
#pragma unroll
  for (int k = 0; k < TPT; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double v = (PREC == F3D_FP64) ? acc[k][c]
                                    : static_cast<double>(fs[k][c]) + static_cast<double>(fc[k][c]);
      double v2 = acc2[k][c];
#pragma unroll
      for (int off = SL / 2; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
        if (DUAL) v2 += __shfl_xor_sync(0xffffffffu, v2, off);
      }
      res[k][c] = v;
      res2[k][c] = v2;
    }

  if (a.nsplit == 1) {
    if (sl == 0) {
#pragma unroll
      for (int k = 0; k < TPT; ++k) {
        const int64_t t = tidx[k];
        if (t < a.nt) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double v = a.scale * res[k][c];
            a.out[3 * t + c] = a.accumulate ? a.out[3 * t + c] + v : v;
            if (DUAL) {
              const double v2 = a.scale * res2[k][c];
              a.out2[3 * t + c] = a.accumulate ? a.out2[3 * t + c] + v2 : v2;
            }
          }
        }
      }
    }
    return;
  }

  // ---- multi-split: partials, then the last CTA of this target block sums --
  if (sl == 0) {
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      const int64_t t = tidx[k];
      if (t < a.nt) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          __stcg(&a.partial[(static_cast<int64_t>(split) * a.nt + t) * 3 + c], res[k][c]);
          if (DUAL)
            __stcg(&a.partial[(static_cast<int64_t>(a.nsplit + split) * a.nt + t) * 3 + c], res2[k][c]);
        }
      }
    }
  }
  __threadfence();
  __syncthreads();
  __shared__ int s_last;
  if (tid == 0) {
    const unsigned prev = atomicAdd(&a.counters[blockIdx.x], 1u);
    s_last = (prev == static_cast<unsigned>(a.nsplit - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int64_t nvals = ((a.nt - tb < TPB) ? (a.nt - tb) : static_cast<int64_t>(TPB)) * 3;
  for (int64_t i = tid; i < nvals; i += kBlock) {
    const int64_t gi = tb * 3 + i;
    double v = 0.0;
    for (int sp = 0; sp < a.nsplit; ++sp) v += __ldcg(&a.partial[static_cast<int64_t>(sp) * a.nt * 3 + gi]);
    v *= a.scale;
    a.out[gi] = a.accumulate ? a.out[gi] + v : v;
    if (DUAL) {
      double v2 = 0.0;
      for (int sp = 0; sp < a.nsplit; ++sp)
        v2 += __ldcg(&a.partial[static_cast<int64_t>(a.nsplit + sp) * a.nt * 3 + gi]);
      v2 *= a.scale;
      a.out2[gi] = a.accumulate ? a.out2[gi] + v2 : v2;
    }
  }
  if (tid == 0) a.counters[blockIdx.x] = 0u;
}

// Packs FP32C source records by pairs of sources (2q, 2q + 1): 24 floats
// {xh,yh,zh,xl,yl,zl,d0,d1,d2,n0,n1,n2} interleaved as {even, odd} per
// component, in the order the kernel reads them: {xh_e,xh_o,yh_e,yh_o},
// {zh_e,zh_o,xl_e,xl_o}, {yl_e,yl_o,zl_e,zl_o}, {d0_e,d0_o,d1_e,d1_o},
// {d2_e,d2_o,n0_e,n0_o}, {n1_e,n1_o,n2_e,n2_o}.  One thread per source;
// with an odd count the source index ns is a pad at 1e30 with zero density
// and normal, whose pair terms are exactly zero (r^2 overflows to inf,
// rsqrt gives 0, and every term carries a zero factor).
__global__ void pack_fp32_sources(const double *rs, const double *dens, const double *nrm,
                                  float *packed, int64_t ns) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t npad = (ns + 1) & ~static_cast<int64_t>(1);
  if (s >= npad) return;
  float v[12];
  if (s < ns) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double x = rs[3 * s + c];
      v[c] = static_cast<float>(x);
      v[3 + c] = static_cast<float>(x - static_cast<double>(v[c]));
      v[6 + c] = static_cast<float>(dens[3 * s + c]);
      v[9 + c] = nrm ? static_cast<float>(nrm[3 * s + c]) : 0.f;
    }
  } else {
#pragma unroll
    for (int c = 0; c < 12; ++c) v[c] = (c < 3) ? 1e30f : 0.f;
  }
  float *o = packed + 24 * (s >> 1) + (s & 1);
#pragma unroll
  for (int c = 0; c < 12; ++c) o[2 * c] = v[c];
}

// ---------------------------------------------------------------- host ----
// The symmetric self-sum (f3d_pairs_sym.cu).
size_t sym_partial_bytes(int64_t n, int64_t nt);
bool sym_fits(int64_t n, int64_t nt);
int pair_sym_launch(int kernel, int self_mode, const double *x, const double *dens, const double *nrm,
                    const int32_t *grp, double *out, int64_t n, int64_t nt, double eta, double reg, double eps,
                    int accumulate, double *partial, unsigned *counters, int *occupancy, cudaStream_t st,
                    const double *dens2, double *out2, bool dual);
// Its tile form for plain source -> target sums.
size_t tile_partial_bytes(int64_t ns, int64_t nt, int sub);
bool tile_fits(int64_t ns, int64_t nt, int sub);
int pair_tile_launch(int kernel, const double *xs, const double *dens, const double *nrm, const double *xt,
                     double *out, int64_t ns, int64_t nt, double eta, double reg, double eps, int accumulate,
                     double *partial, unsigned *counters, int *occupancy, cudaStream_t st, const double *dens2,
                     double *out2, bool dual, int sub);

struct Plan {
  int tpt, sl, nsplit, use_tma;
  bool sym;   // shape.sl == -1: the symmetric self-sum
  bool tile;  // shape.sl == -2: the tile form of a source -> target sum
  int64_t ntb, tiles_per_split;
  size_t off_counters, off_partial, off_packed, bytes;
};

static int make_plan(int kernel, int precision, int64_t ns, int64_t nt, const f3d_pair_shape *shape,
                     Plan *p, bool dual = false) {
  if (kernel < 0 || kernel > 3 || precision < 0 || precision > 1) return F3D_ERR_ARG;
  if (ns < 0 || nt < 0) return F3D_ERR_SHAPE;
  p->sym = false;
  p->tile = false;
  if (shape && shape->sl == -2) {
    // tile form: FP64 Oseen or stresslet, sources and targets in their own
    // arrays, two targets per thread on 128-point tiles (the symmetric
    // kernel's target-side items)
    if (precision != F3D_FP64 || !(kernel == F3D_KERNEL_OSEEN || kernel == F3D_KERNEL_STRESSLET))
      return F3D_ERR_ARG;
    // source sub-tiles: 1 (128 points, the default) or 2 (64 points: twice
    // the items, for sums too small to fill the GPU; on the 12000-node sphere
    // onto 4096 points, 2.5 waves of whole items, the halves measured slower)
    int sub = shape->nsplit == 0 ? 1 : shape->nsplit;
    if (sub != 1 && sub != 2) return F3D_ERR_ARG;
    if (!tile_fits(ns, nt, sub)) return F3D_ERR_TOO_LARGE;
    p->tile = true;
    p->tpt = 2;
    p->sl = -2;
    p->nsplit = sub;
    p->use_tma = 0;
    p->ntb = (nt + kBlock - 1) / kBlock;
    p->tiles_per_split = 0;
    p->off_counters = 0;
    p->off_partial = kCounterBytes;
    p->off_packed = kCounterBytes;
    p->bytes =
        (ns > 0 && nt > 0) ? kCounterBytes + round_up((dual ? 2 : 1) * tile_partial_bytes(ns, nt, sub), 256) : 0;
    return F3D_OK;
  }
  if (shape && shape->sl == -1) {
    // symmetric self-sum: FP64 Oseen or stresslet over one point set (the
    // first ns of the nt targets), further targets one-sided; the
    // two-density Oseen form keeps two partial arrays
    if (precision != F3D_FP64 || !(kernel == F3D_KERNEL_OSEEN || kernel == F3D_KERNEL_STRESSLET))
      return F3D_ERR_ARG;
    if (nt < ns) return F3D_ERR_SHAPE;
    if (!sym_fits(ns, nt)) return F3D_ERR_TOO_LARGE;
    p->sym = true;
    p->tpt = 1;
    p->sl = -1;
    p->nsplit = 1;
    p->use_tma = 0;
    p->ntb = (ns + kBlock - 1) / kBlock;
    p->tiles_per_split = 0;
    p->off_counters = 0;
    p->off_partial = kCounterBytes;
    p->off_packed = kCounterBytes;
    p->bytes = ns > 0 ? kCounterBytes + round_up((dual ? 2 : 1) * sym_partial_bytes(ns, nt), 256) : 0;
    return F3D_OK;
  }
  int tpt = shape && shape->tpt ? shape->tpt : 0;
  int sl = shape && shape->sl ? shape->sl : 0;
  if (sl == 0) sl = (nt >= 4096) ? 1 : (nt >= 512 ? 8 : 32);
  if (tpt == 0) tpt = 1;
  if (!(tpt == 1 || tpt == 2 || tpt == 4)) return F3D_ERR_ARG;
  if (tpt == 4 && precision != F3D_FP64) return F3D_ERR_ARG;  // four targets per thread: FP64 only
  if (!(sl == 1 || sl == 8 || sl == 32)) return F3D_ERR_ARG;
  if (sl != 1 && tpt != 1) return F3D_ERR_ARG;
  const int64_t tpb = static_cast<int64_t>(kBlock / sl) * tpt;
  const int64_t ntb = (nt + tpb - 1) / tpb;
  const int64_t nfull = ns / kTile;
  int64_t nsplit = shape && shape->nsplit > 0 ? shape->nsplit : 0;
  if (nsplit == 0) {
    const int64_t want = 8LL * sm_count();
    nsplit = ntb > 0 ? (want + ntb - 1) / ntb : 1;
  }
  nsplit = std::max<int64_t>(1, std::min<int64_t>(nsplit, std::max<int64_t>(nfull, 1)));
  nsplit = std::min<int64_t>(nsplit, 65535);
  int64_t tps = nfull > 0 ? (nfull + nsplit - 1) / nsplit : 0;
  if (tps > 0) nsplit = (nfull + tps - 1) / tps;
  if (nsplit < 1) nsplit = 1;
  if (ntb > kMaxCounters) {
    nsplit = 1;
    tps = nfull;
  }
  p->tpt = tpt;
  p->sl = sl;
  p->nsplit = static_cast<int>(nsplit);
  p->use_tma = (shape && shape->use_tma < 0) ? 0 : 1;
  p->ntb = ntb;
  p->tiles_per_split = tps;
  // The counter words live in a fixed region at the start of the workspace
  // that nothing else ever writes, so they stay zero between calls of any
  // shape (each kernel returns the words it used to zero).  The region is
  // reserved whenever the call uses the workspace at all, also by calls that
  // need no counters themselves (FP32C with one split packs its sources
  // behind it), because one workspace serves calls of every shape.
  size_t off = 0;
  p->off_counters = off;
  if (p->nsplit > 1 || precision == F3D_FP32C) off += kCounterBytes;
  p->off_partial = off;
  if (p->nsplit > 1)
    off += round_up(static_cast<size_t>(p->nsplit) * nt * 3 * sizeof(double) * (dual ? 2 : 1), 256);
  p->off_packed = off;
  if (precision == F3D_FP32C) off += round_up(static_cast<size_t>((ns + 1) & ~int64_t(1)) * 12 * sizeof(float), 256);
  p->bytes = off;
  return F3D_OK;
}

template <int KIND, int MODE, int PREC, int TPT, int SL, bool DUAL = false>
static int launch_one(const PairArgs &a, int64_t ntb, int nsplit, cudaStream_t st) {
  constexpr size_t smem = pair_smem_bytes<KIND, MODE, PREC, TPT, DUAL>();
  auto kfn = pair_kernel<KIND, MODE, PREC, TPT, SL, DUAL>;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev >= 0 && dev < 64 && !attr_set[dev]) {
    if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
      return F3D_ERR_CUDA;
    attr_set[dev] = true;
  }
  if (a.occupancy) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(a.occupancy, kfn, kBlock, smem) == cudaSuccess
               ? F3D_OK
               : F3D_ERR_CUDA;
  }
  dim3 grid(static_cast<unsigned>(ntb), static_cast<unsigned>(nsplit));
  kfn<<<grid, kBlock, smem, st>>>(a);
  return launch_status();
}

template <int KIND, int MODE, int PREC, bool DUAL = false>
static int dispatch_shape(const PairArgs &a, const Plan &p, cudaStream_t st) {
  if (p.sl == 1 && p.tpt == 1) return launch_one<KIND, MODE, PREC, 1, 1, DUAL>(a, p.ntb, p.nsplit, st);
  if (p.sl == 1 && p.tpt == 2) return launch_one<KIND, MODE, PREC, 2, 1, DUAL>(a, p.ntb, p.nsplit, st);
  if constexpr (PREC == F3D_FP64) {
    if (p.sl == 1 && p.tpt == 4) return launch_one<KIND, MODE, PREC, 4, 1, DUAL>(a, p.ntb, p.nsplit, st);
  }
  if (p.sl == 8) return launch_one<KIND, MODE, PREC, 1, 8, DUAL>(a, p.ntb, p.nsplit, st);
  return launch_one<KIND, MODE, PREC, 1, 32, DUAL>(a, p.ntb, p.nsplit, st);
}

template <int KIND, int PREC>
static int dispatch_mode(int mode, const PairArgs &a, const Plan &p, cudaStream_t st) {
  switch (mode) {
    case F3D_SELF_REGULARISE: return dispatch_shape<KIND, F3D_SELF_REGULARISE, PREC>(a, p, st);
    case F3D_SELF_SKIP_INDEX: return dispatch_shape<KIND, F3D_SELF_SKIP_INDEX, PREC>(a, p, st);
    case F3D_SELF_SKIP_GROUP: return dispatch_shape<KIND, F3D_SELF_SKIP_GROUP, PREC>(a, p, st);
    case F3D_SELF_SKIP_CLOSE: return dispatch_shape<KIND, F3D_SELF_SKIP_CLOSE, PREC>(a, p, st);
    default: return F3D_ERR_ARG;
  }
}

template <int KIND>
static int dispatch_prec(int prec, int mode, const PairArgs &a, const Plan &p, cudaStream_t st) {
  if (prec == F3D_FP64) return dispatch_mode<KIND, F3D_FP64>(mode, a, p, st);
  return dispatch_mode<KIND, F3D_FP32C>(mode, a, p, st);
}

// One sum, or with dens2/out2 the dual FP64 Oseen sum (both outputs from
// one pass over the pairs).
static int pair_sum_core(int kernel, int precision, int self_mode, const double *rs,
                         const double *rt, const double *dens, const double *nrm,
                         const int32_t *gs, const int32_t *gt, double *out, int64_t ns,
                         int64_t nt, double eta, double reg, double eps, int accumulate,
                         const f3d_pair_shape *shape, void *ws, size_t ws_bytes, cudaStream_t st,
                         const double *dens2, double *out2) {
  const bool dual = out2 != nullptr;
  if (dual && (kernel != F3D_KERNEL_OSEEN || precision != F3D_FP64)) return F3D_ERR_ARG;
  Plan p;
  int rc = make_plan(kernel, precision, ns, nt, shape, &p, dual);
  if (rc) return rc;
  if (self_mode < 0 || self_mode > 3) return F3D_ERR_ARG;
  if (dual && self_mode == F3D_SELF_SKIP_CLOSE) return F3D_ERR_ARG;
  if (p.sym && !(self_mode == F3D_SELF_SKIP_INDEX || self_mode == F3D_SELF_SKIP_GROUP)) return F3D_ERR_ARG;
  if (p.tile && self_mode != F3D_SELF_REGULARISE) return F3D_ERR_ARG;
  if (nt == 0) return F3D_OK;
  if (!rt || !out) return F3D_ERR_NULL;
  if (ns > 0 && (!rs || !dens)) return F3D_ERR_NULL;
  if (kernel == F3D_KERNEL_STRESSLET && ns > 0 && !nrm) return F3D_ERR_NULL;
  if (kernel == F3D_KERNEL_TRACTION && !nrm) return F3D_ERR_NULL;  // target normals
  if (self_mode == F3D_SELF_SKIP_GROUP && (!gt || (ns > 0 && !gs))) return F3D_ERR_NULL;
  if (self_mode == F3D_SELF_SKIP_INDEX && nt < ns) return F3D_ERR_SHAPE;
  if (!aligned(rs, 8) || !aligned(rt, 8) || !aligned(dens, 8) || !aligned(nrm, 8) ||
      !aligned(out, 8) || !aligned(gs, 4) || !aligned(gt, 4))
    return F3D_ERR_ALIGN;
  if (dual && (!out2 || (ns > 0 && !dens2))) return F3D_ERR_NULL;
  if (dual && (!aligned(out2, 8) || !aligned(dens2, 8))) return F3D_ERR_ALIGN;
  if (ns == 0) {
    if (!accumulate && cudaMemsetAsync(out, 0, static_cast<size_t>(nt) * 3 * sizeof(double), st) != cudaSuccess)
      return F3D_ERR_CUDA;
    if (dual && !accumulate &&
        cudaMemsetAsync(out2, 0, static_cast<size_t>(nt) * 3 * sizeof(double), st) != cudaSuccess)
      return F3D_ERR_CUDA;
    return F3D_OK;
  }
  if (p.bytes > 0 && (!ws || ws_bytes < p.bytes)) return F3D_ERR_WORKSPACE;
  if (ws && !aligned(ws, 256)) return F3D_ERR_ALIGN;
  unsigned char *w = static_cast<unsigned char *>(ws);
  if (p.sym) {
    // one point set: the sources are the first ns targets (and their group
    // ids the first ns target group ids), passed as the same arrays
    if (rs != rt || (self_mode == F3D_SELF_SKIP_GROUP && gs != gt)) return F3D_ERR_ARG;
    return pair_sym_launch(kernel, self_mode, rs, dens, nrm, gs, out, ns, nt, eta, reg, eps, accumulate,
                           reinterpret_cast<double *>(w + p.off_partial), reinterpret_cast<unsigned *>(w),
                           nullptr, st, dens2, out2, dual);
  }
  if (p.tile)
    return pair_tile_launch(kernel, rs, dens, nrm, rt, out, ns, nt, eta, reg, eps, accumulate,
                            reinterpret_cast<double *>(w + p.off_partial), reinterpret_cast<unsigned *>(w), nullptr,
                            st, dens2, out2, dual, p.nsplit);

  PairArgs a{};
  a.rs = rs; a.rt = rt; a.dens = dens; a.nrm = nrm;
  a.gs = gs; a.gt = gt;
  a.out = out;
  a.dens2 = dens2;
  a.out2 = out2;
  a.partial = p.nsplit > 1 ? reinterpret_cast<double *>(w + p.off_partial) : nullptr;
  a.counters = p.nsplit > 1 ? reinterpret_cast<unsigned *>(w + p.off_counters) : nullptr;
  a.packed = precision == F3D_FP32C ? reinterpret_cast<float *>(w + p.off_packed) : nullptr;
  a.err = device_error_word();
  a.wait_ns = wait_limit_ns();
  a.ns = ns; a.nt = nt;
  a.tiles_per_split = p.tiles_per_split;
  a.nsplit = p.nsplit;
  a.accumulate = accumulate ? 1 : 0;
  a.eps2 = eps * eps;
  a.reg2 = reg * reg;
  a.scale = (kernel == F3D_KERNEL_STRESSLET || kernel == F3D_KERNEL_TRACTION) ? -3.0 / (4.0 * kPi * eta)
                                                                                : 1.0 / (8.0 * kPi * eta);
  // Bulk copies need 16-byte aligned sources; otherwise stage with plain loads.
  a.use_tma = p.use_tma;
  if (precision == F3D_FP64 && (!aligned(rs, 16) || !aligned(dens, 16) ||
                                (kernel == F3D_KERNEL_STRESSLET && !aligned(nrm, 16)) ||
                                (dual && !aligned(dens2, 16))))
    a.use_tma = 0;
  if (self_mode == F3D_SELF_SKIP_GROUP && !aligned(gs, 16)) a.use_tma = 0;

  if (precision == F3D_FP32C) {
    const int64_t nb = (ns + 1 + 255) / 256;
    pack_fp32_sources<<<static_cast<unsigned>(nb), 256, 0, st>>>(
        rs, dens, kernel == F3D_KERNEL_STRESSLET ? nrm : nullptr, const_cast<float *>(a.packed), ns);
    if ((rc = launch_status())) return rc;
  }
  if (dual) {
    switch (self_mode) {
      case F3D_SELF_REGULARISE:
        return dispatch_shape<F3D_KERNEL_OSEEN, F3D_SELF_REGULARISE, F3D_FP64, true>(a, p, st);
      case F3D_SELF_SKIP_INDEX:
        return dispatch_shape<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX, F3D_FP64, true>(a, p, st);
      default:
        return dispatch_shape<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_GROUP, F3D_FP64, true>(a, p, st);
    }
  }
  switch (kernel) {
    case F3D_KERNEL_OSEEN: return dispatch_prec<F3D_KERNEL_OSEEN>(precision, self_mode, a, p, st);
    case F3D_KERNEL_STRESSLET: return dispatch_prec<F3D_KERNEL_STRESSLET>(precision, self_mode, a, p, st);
    case F3D_KERNEL_TRACTION: return dispatch_prec<F3D_KERNEL_TRACTION>(precision, self_mode, a, p, st);
    default: return dispatch_prec<F3D_KERNEL_ROTLET>(precision, self_mode, a, p, st);
  }
}

int pair_sum_impl(int kernel, int precision, int self_mode, const double *rs, const double *rt,
                  const double *dens, const double *nrm, const int32_t *gs, const int32_t *gt,
                  double *out, int64_t ns, int64_t nt, double eta, double reg, double eps,
                  int accumulate, const f3d_pair_shape *shape, void *ws, size_t ws_bytes,
                  cudaStream_t st) {
  return pair_sum_core(kernel, precision, self_mode, rs, rt, dens, nrm, gs, gt, out, ns, nt, eta,
                       reg, eps, accumulate, shape, ws, ws_bytes, st, nullptr, nullptr);
}

}  // namespace f3d

extern "C" {

int f3d_pair_workspace_bytes(int kernel, int precision, int64_t ns, int64_t nt,
                             const f3d_pair_shape *shape, size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  f3d::Plan p;
  int rc = f3d::make_plan(kernel, precision, ns, nt, shape, &p);
  if (rc) return rc;
  *bytes = p.bytes;
  return F3D_OK;
}

int f3d_pair_sum(int kernel, int precision, int self_mode, const double *r_source,
                 const double *r_target, const double *density, const double *normal,
                 const int32_t *src_group, const int32_t *trg_group, double *out, int64_t ns,
                 int64_t nt, double eta, double reg, double epsilon_distance, int accumulate,
                 const f3d_pair_shape *shape, void *workspace, size_t workspace_bytes,
                 void *stream) {
  return f3d::pair_sum_impl(kernel, precision, self_mode, r_source, r_target, density, normal,
                            src_group, trg_group, out, ns, nt, eta, reg, epsilon_distance,
                            accumulate, shape, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int f3d_oseen_source_target(const double *r_source, const double *r_target,
                            const double *density, double *u, int64_t ns, int64_t nt,
                            double eta, double reg, double epsilon_distance, int precision,
                            void *workspace, size_t workspace_bytes, void *stream) {
  return f3d::pair_sum_impl(F3D_KERNEL_OSEEN, precision, F3D_SELF_REGULARISE, r_source, r_target,
                            density, nullptr, nullptr, nullptr, u, ns, nt, eta, reg,
                            epsilon_distance, 0, nullptr, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int f3d_oseen_times_density(const double *r_vectors, const double *density, double *u,
                            int64_t n, double eta, double reg, double epsilon_distance,
                            int precision, void *workspace, size_t workspace_bytes,
                            void *stream) {
  return f3d::pair_sum_impl(F3D_KERNEL_OSEEN, precision, F3D_SELF_SKIP_INDEX, r_vectors,
                            r_vectors, density, nullptr, nullptr, nullptr, u, n, n, eta, reg,
                            epsilon_distance, 0, nullptr, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int f3d_rotlet_source_target(const double *r_source, const double *r_target,
                             const double *density, double *u, int64_t ns, int64_t nt,
                             double eta, double reg, double epsilon_distance, int precision,
                             void *workspace, size_t workspace_bytes, void *stream) {
  return f3d::pair_sum_impl(F3D_KERNEL_ROTLET, precision, F3D_SELF_REGULARISE, r_source, r_target,
                            density, nullptr, nullptr, nullptr, u, ns, nt, eta, reg,
                            epsilon_distance, 0, nullptr, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int f3d_stresslet_source_target(const double *r_source, const double *r_target,
                                const double *normal, const double *density, double *v,
                                int64_t ns, int64_t nt, double eta, double reg,
                                double epsilon_distance, int precision, void *workspace,
                                size_t workspace_bytes, void *stream) {
  return f3d::pair_sum_impl(F3D_KERNEL_STRESSLET, precision, F3D_SELF_REGULARISE, r_source,
                            r_target, density, normal, nullptr, nullptr, v, ns, nt, eta, reg,
                            epsilon_distance, 0, nullptr, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int f3d_stresslet_times_normal_times_density(const double *r_vectors, const double *normal,
                                             const double *density, double *v, int64_t n,
                                             double eta, double reg, double epsilon_distance,
                                             int precision, void *workspace,
                                             size_t workspace_bytes, void *stream) {
  return f3d::pair_sum_impl(F3D_KERNEL_STRESSLET, precision, F3D_SELF_SKIP_INDEX, r_vectors,
                            r_vectors, density, normal, nullptr, nullptr, v, n, n, eta, reg,
                            epsilon_distance, 0, nullptr, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int f3d_pair_occupancy(int kernel, int precision, int self_mode, int dual, const f3d_pair_shape *shape,
                       int *ctas_per_sm) {
  if (!ctas_per_sm) return F3D_ERR_NULL;
  f3d::Plan p;
  int rc = f3d::make_plan(kernel, precision, 1, 1, shape, &p, dual != 0);
  if (rc) return rc;
  if (self_mode < 0 || self_mode > 3) return F3D_ERR_ARG;
  if (dual && (kernel != F3D_KERNEL_OSEEN || precision != F3D_FP64 || self_mode == F3D_SELF_SKIP_CLOSE))
    return F3D_ERR_ARG;
  if (shape && shape->sl == -1) {
    if (precision != F3D_FP64 || !(kernel == F3D_KERNEL_OSEEN || kernel == F3D_KERNEL_STRESSLET) ||
        !(self_mode == F3D_SELF_SKIP_INDEX || self_mode == F3D_SELF_SKIP_GROUP))
      return F3D_ERR_ARG;
    return f3d::pair_sym_launch(kernel, self_mode, nullptr, nullptr, nullptr, nullptr, nullptr, 1, 1, 1.0, 0.0, 0.0,
                                0, nullptr, nullptr, ctas_per_sm, nullptr, nullptr, nullptr, dual != 0);
  }
  if (shape && shape->sl == -2) {
    if (self_mode != F3D_SELF_REGULARISE) return F3D_ERR_ARG;
    return f3d::pair_tile_launch(kernel, nullptr, nullptr, nullptr, nullptr, nullptr, 1, 1, 1.0, 0.0, 0.0, 0,
                                 nullptr, nullptr, ctas_per_sm, nullptr, nullptr, nullptr, dual != 0, 1);
  }
  // the shape's own tpt/sl (make_plan picks defaults for a 1-target sum)
  if (shape && shape->tpt) p.tpt = shape->tpt;
  if (shape && shape->sl) p.sl = shape->sl;
  f3d::PairArgs a{};
  a.occupancy = ctas_per_sm;
  if (dual) {
    switch (self_mode) {
      case F3D_SELF_REGULARISE:
        return f3d::dispatch_shape<F3D_KERNEL_OSEEN, F3D_SELF_REGULARISE, F3D_FP64, true>(a, p, nullptr);
      case F3D_SELF_SKIP_INDEX:
        return f3d::dispatch_shape<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_INDEX, F3D_FP64, true>(a, p, nullptr);
      default:
        return f3d::dispatch_shape<F3D_KERNEL_OSEEN, F3D_SELF_SKIP_GROUP, F3D_FP64, true>(a, p, nullptr);
    }
  }
  switch (kernel) {
    case F3D_KERNEL_OSEEN: return f3d::dispatch_prec<F3D_KERNEL_OSEEN>(precision, self_mode, a, p, nullptr);
    case F3D_KERNEL_STRESSLET: return f3d::dispatch_prec<F3D_KERNEL_STRESSLET>(precision, self_mode, a, p, nullptr);
    case F3D_KERNEL_TRACTION: return f3d::dispatch_prec<F3D_KERNEL_TRACTION>(precision, self_mode, a, p, nullptr);
    default: return f3d::dispatch_prec<F3D_KERNEL_ROTLET>(precision, self_mode, a, p, nullptr);
  }
}

int f3d_oseen_dual_workspace_bytes(int64_t ns, int64_t nt, const f3d_pair_shape *shape,
                                   size_t *bytes) {
  if (!bytes) return F3D_ERR_NULL;
  f3d::Plan p;
  int rc = f3d::make_plan(F3D_KERNEL_OSEEN, F3D_FP64, ns, nt, shape, &p, true);
  if (rc) return rc;
  *bytes = p.bytes;
  return F3D_OK;
}

int f3d_oseen_dual(int self_mode, const double *r_source, const double *r_target,
                   const double *density, const double *density2, const int32_t *src_group,
                   const int32_t *trg_group, double *out, double *out2, int64_t ns, int64_t nt,
                   double eta, double reg, double epsilon_distance, int accumulate,
                   const f3d_pair_shape *shape, void *workspace, size_t workspace_bytes,
                   void *stream) {
  if (!out2) return F3D_ERR_NULL;
  return f3d::pair_sum_core(F3D_KERNEL_OSEEN, F3D_FP64, self_mode, r_source, r_target, density, nullptr,
                            src_group, trg_group, out, ns, nt, eta, reg, epsilon_distance, accumulate,
                            shape, workspace, workspace_bytes, static_cast<cudaStream_t>(stream),
                            density2, out2);
}

}  // extern "C"
