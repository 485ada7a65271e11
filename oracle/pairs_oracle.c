/*
 * C restatement of fiber3d's numba pair sums — TEST ORACLE and timed CPU
 * baseline (never linked into the product library).
 *
 * Loop structure follows the reference: a parallel loop over targets
 * (numba prange -> OpenMP), an inner scalar loop over sources, sqrt and
 * divisions as written in python/kernels/kernels.py:
 *   kind 0 Oseen      oseen_kernel_source_target_numba          :794-846
 *                     oseen_kernel_times_density_numba (skip)   :214-287
 *   kind 1 stresslet  stresslet_kernel_source_target_numba      :1186-1217
 *                     stresslet_..._times_density_numba (skip)  :1123-1183
 *   kind 2 rotlet     rotlet_kernel_source_target_numba         :856-908
 * self_mode 0: all pairs, |r| < eps regularised; 1: pair yn == xn skipped;
 * 2: pairs with equal group id skipped (fused flow_fibers/self_flow_fibers).
 */
#include <math.h>
#include <stdint.h>
#include <omp.h>

int oracle_max_threads(void) { return omp_get_max_threads(); }

void oracle_pair_sum(int kind, int self_mode, const double *rs, const double *rt,
                     const double *dens, const double *nrm, const int32_t *gs,
                     const int32_t *gt, double *out, int64_t ns, int64_t nt, double eta,
                     double reg, double eps, int nthreads) {
  const double pi = 3.14159265358979323846;
  const double factor = (kind == 1) ? -3.0 / (4.0 * pi * eta) : 1.0 / (8.0 * pi * eta);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t xn = 0; xn < nt; ++xn) {
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
    const double tx = rt[3 * xn], ty = rt[3 * xn + 1], tz = rt[3 * xn + 2];
    for (int64_t yn = 0; yn < ns; ++yn) {
      if (self_mode == 1 && yn == xn) continue;
      if (self_mode == 2 && gs[yn] == gt[xn]) continue;
      const double x = tx - rs[3 * yn];
      const double y = ty - rs[3 * yn + 1];
      const double z = tz - rs[3 * yn + 2];
      double r_norm = sqrt(x * x + y * y + z * z);
      if (r_norm < eps) r_norm = sqrt(r_norm * r_norm + reg * reg);
      const double d0 = dens[3 * yn], d1 = dens[3 * yn + 1], d2 = dens[3 * yn + 2];
      if (kind == 0) {
        const double fr = factor / r_norm;
        const double gr = factor / (r_norm * r_norm * r_norm);
        const double Mxx = fr + gr * x * x, Mxy = gr * x * y, Mxz = gr * x * z;
        const double Myy = fr + gr * y * y, Myz = gr * y * z, Mzz = fr + gr * z * z;
        u0 += Mxx * d0 + Mxy * d1 + Mxz * d2;
        u1 += Mxy * d0 + Myy * d1 + Myz * d2;
        u2 += Mxz * d0 + Myz * d1 + Mzz * d2;
      } else if (kind == 2) {
        const double fr = factor / (r_norm * r_norm * r_norm);
        u0 += fr * z * d1 - fr * y * d2;
        u1 += -fr * z * d0 + fr * x * d2;
        u2 += fr * y * d0 - fr * x * d1;
      } else {
        const double r_inv5 = 1.0 / (r_norm * r_norm * r_norm * r_norm * r_norm);
        const double f0 = factor * (x * d0 + y * d1 + z * d2) *
                          (x * nrm[3 * yn] + y * nrm[3 * yn + 1] + z * nrm[3 * yn + 2]) * r_inv5;
        u0 += f0 * x;
        u1 += f0 * y;
        u2 += f0 * z;
      }
    }
    out[3 * xn] = u0;
    out[3 * xn + 1] = u1;
    out[3 * xn + 2] = u2;
  }
}
