// FP64 pair arithmetic shared by the all-pairs kernels (f3d_pairs.cu) and
// their symmetric self-sum form (f3d_pairs_sym.cu).
#pragma once

#include "f3d_common.cuh"

namespace f3d {

// Reciprocal square roots in FP64.  y0 = rsqrt.approx.ftz.f64(x) (PTX; about
// 2^-22 relative error) is a seed; with u = y0^2 and e = 1 - x u (one FMA,
// exact to rounding), x^(-1/2) = y0 (1 - e)^(-1/2) and x^(-5/2) =
// y0 u^2 (1 - e)^(-5/2).  The binomial series to second order,
//   (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8,   (1 - e)^(-5/2) = 1 + 5e/2 + 35e^2/8,
// leaves O(e^3) ~ 2^-66: below double rounding.  (The first is one
// Halley-type step for 1/sqrt(x); folding the second into the power r^-5
// that the stresslet needs saves the separate refinement.)  For x = 0 the
// result is not finite; callers discard such pairs with a select.
__device__ __forceinline__ double rsqrt_seed(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

__device__ __forceinline__ double rsqrt_refined(double x) {
  const double y = rsqrt_seed(x);
  const double e = fma(-x, y * y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}

// q * x^(-5/2) for x > 0.
__device__ __forceinline__ double times_rsqrt5(double q, double x) {
  const double y = rsqrt_seed(x);
  const double u = y * y;
  const double e = fma(-x, u, 1.0);
  const double qy5 = (q * y) * (u * u);
  return fma(qy5 * e, fma(4.375, e, 2.5), qy5);
}

// x^(-5/2) for x > 0 (the same series as times_rsqrt5).
__device__ __forceinline__ double rsqrt5(double x) {
  const double y = rsqrt_seed(x);
  const double u = y * y;
  const double e = fma(-x, u, 1.0);
  const double y5 = y * (u * u);
  return fma(y5 * e, fma(4.375, e, 2.5), y5);
}

// Adds reg2 to r2 where close (r2 < eps2).  Such pairs are rare, so the add
// sits in a branch that a warp enters only when one of its lanes needs it.
// The vote covers exactly the lanes executing it, and each lane's own
// predicate is part of its vote, so the result does not depend on
// convergence.
__device__ __forceinline__ double regularise(double r2, bool close, double reg2) {
  if (__any_sync(__activemask(), close)) {
    if (close) r2 += reg2;
  }
  return r2;
}

}  // namespace f3d
