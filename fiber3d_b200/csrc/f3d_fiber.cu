// Fiber discretisation on the device: per-point derivatives, per-fiber
// operator + right-hand side assembly with the 14 boundary rows, the force
// operator, and the fiber rows of the GMRES matvec.
//
// Reference (fiber3d, python/):
//   derivatives xs..xsss = D_k x                tstep/tstep.py:703-709
//   operator A (4N x 4N)                        fiber/fiber.py:322-448 (form_linear_operator)
//   right-hand side                             fiber/fiber.py:473-582 (compute_RHS)
//   rectangular collocation + BC rows           fiber/fiber.py:810-961 (apply_BC_rectangular)
//   force operator f = -E X_ssss + (T X_s)_s    fiber/fiber.py:1399-1432
//   trapezoid weights (L/2) w0                  tstep/fiber_matrices.py:70-73, 135
//   fiber rows of the matvec                    tstep/tstep.py:1147-1173
//
// Per-resolution matrices (computed once on the host by fiber3d_b200.fibers
// and uploaded): D1_0..D4_0 (N x N, on alpha = linspace(-1,1,N)), P_X
// ((N-4) x N), P_T ((N-2) x N), w0 (N).  D_k = D_k_0 (2/L)^k.  The D_k are
// finite-difference matrices whose row k is non-zero only on a window of at
// most `band` + 1 consecutive columns containing k, so every product with a
// D_k loops over |k - j| <= band only.
//
// Layouts: points of all fibers are concatenated (pt_off[f] .. pt_off[f+1]);
// per-point vectors are (npts, 3) xyz-interleaved; per-fiber unknown blocks
// are [X_x(N), X_y(N), X_z(N), T(N)] at 4*pt_off[f]; operator blocks are
// row-major 4N x 4N at mat_off[f].
#include "f3d_common.cuh"

namespace f3d {

enum FiberBC { BC_FORCE = 0, BC_TORQUE = 1, BC_VELOCITY = 2, BC_ANGULAR_VELOCITY = 3 };

struct FiberSet {
  int nfib;
  const int32_t *n;        // points per fiber
  const int64_t *pt_off;   // first point of each fiber
  const int64_t *mat_off;  // operator block offsets
  const int64_t *res_off;  // offset of the fiber's resolution block in `mats`
  const double *length;    // per fiber
  const int32_t *bc;       // 4 codes per fiber: start_0, start_1, end_0, end_1
  const int32_t *pt_fib;   // fiber index of each point
  const double *mats;      // per-resolution matrices, see ResLayout
  int band;                // finite-difference half-window (n_fd + 3)
};

// Offsets inside one resolution block of `mats`.
struct ResLayout {
  int64_t d1, d2, d3, d4, px, pt, w0;
  __host__ __device__ explicit ResLayout(int n) {
    const int64_t nn = static_cast<int64_t>(n) * n;
    d1 = 0; d2 = nn; d3 = 2 * nn; d4 = 3 * nn;
    px = 4 * nn;
    pt = px + static_cast<int64_t>(n - 4) * n;
    w0 = pt + static_cast<int64_t>(n - 2) * n;
  }
};

struct FiberPhys {
  double E, dt, c0, c1, penalty;
};

// ---------------------------------------------------------------- geometry --
// geo[p] = {xs, xss, xsss} (9 doubles per point).
__global__ void fiber_geometry_kernel(FiberSet fs, const double *__restrict__ x, double *geo,
                                      int64_t npts) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int f = fs.pt_fib[p];
  const int n = fs.n[f];
  const int64_t p0 = fs.pt_off[f];
  const int k = static_cast<int>(p - p0);
  const double *m = fs.mats + fs.res_off[f];
  const ResLayout R(n);
  const double s1 = 2.0 / fs.length[f];
  const double sc[3] = {s1, s1 * s1, s1 * s1 * s1};
  const int64_t doff[3] = {R.d1, R.d2, R.d3};
  const int j0 = max(0, k - fs.band), j1 = min(n - 1, k + fs.band);
  double out[9];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = j0; j <= j1; ++j) {
      const double w = m[doff[d] + static_cast<int64_t>(k) * n + j];
      a0 = fma(w, x[3 * (p0 + j) + 0], a0);
      a1 = fma(w, x[3 * (p0 + j) + 1], a1);
      a2 = fma(w, x[3 * (p0 + j) + 2], a2);
    }
    out[3 * d + 0] = a0 * sc[d];
    out[3 * d + 1] = a1 * sc[d];
    out[3 * d + 2] = a2 * sc[d];
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) geo[9 * p + i] = out[i];
}

// ------------------------------------------------------------- assembly ----
// Element (r, col) of [P_cheb A; B] for one fiber.
__device__ double assemble_element(int r, int col, int n, const double *__restrict__ m,
                                   const ResLayout &R, const double *__restrict__ g,
                                   const double *__restrict__ xss2, const int32_t *bc,
                                   const FiberPhys &ph, double s1, int band) {
  const double s2 = s1 * s1, s3 = s2 * s1, s4 = s3 * s1;
  const int bcb = col / n, j = col - bcb * n;
  const double E = ph.E, c0 = ph.c0, c1 = ph.c1;
  // geometry at point k: g[9k + 0..2] xs, 3..5 xss, 6..8 xsss
  auto D = [&](int64_t off, int k, int jj) { return m[off + static_cast<int64_t>(k) * n + jj]; };
  const int nrect = 4 * n - 14;
  if (r < nrect) {
    int br, i;
    if (r < n - 4) { br = 0; i = r; }
    else if (r < 2 * n - 8) { br = 1; i = r - (n - 4); }
    else if (r < 3 * n - 12) { br = 2; i = r - (2 * n - 8); }
    else { br = 3; i = r - (3 * n - 12); }
    const double *P = (br < 3) ? m + R.px + static_cast<int64_t>(i) * n : m + R.pt + static_cast<int64_t>(i) * n;
    const int k0 = max(0, j - band), k1 = min(n - 1, j + band);
    double s = 0.0;
    if (br < 3 && bcb < 3) {
      const int a = br, b = bcb;
      if (a == b) s += P[j] / ph.dt;
      for (int k = k0; k <= k1; ++k) {
        const double xa = g[9 * k + a], xb = g[9 * k + b];
        const double c = (a == b) ? E * c0 * (1.0 + xa * xa) + E * c1 * (1.0 - xa * xa)
                                  : (E * c0 - E * c1) * xa * xb;
        s = fma(P[k] * c, D(R.d4, k, j) * s4, s);
      }
    } else if (br < 3) {  // coordinate rows, tension columns
      const int a = br;
      s += P[j] * (-(c0 + c1) * g[9 * j + 3 + a]);
      for (int k = k0; k <= k1; ++k) s = fma(P[k] * (-2.0 * c0 * g[9 * k + a]), D(R.d1, k, j) * s1, s);
    } else if (bcb < 3) {  // tension rows, coordinate columns
      const int b = bcb;
      for (int k = k0; k <= k1; ++k) {
        const double t = -(c1 + 7.0 * c0) * E * g[9 * k + 3 + b] * D(R.d4, k, j) * s4 -
                         6.0 * c0 * E * g[9 * k + 6 + b] * D(R.d3, k, j) * s3 -
                         ph.penalty * g[9 * k + b] * D(R.d1, k, j) * s1;
        s = fma(P[k], t, s);
      }
    } else {  // tension-tension
      s += P[j] * (c1 + c0) * xss2[j];
      for (int k = k0; k <= k1; ++k) s = fma(P[k] * (-2.0 * c0), D(R.d2, k, j) * s2, s);
    }
    return s;
  }
  // 14 boundary rows
  const int b = r - nrect;
  const int last = n - 1;
  const double *g0 = g, *gl = g + 9 * last;
  if (b < 4) {
    if (bc[0] == BC_FORCE) {
      if (b < 3) return (bcb == b) ? E * D(R.d3, 0, j) * s3 : ((bcb == 3 && j == 0) ? -g0[b] : 0.0);
      return (bcb < 3) ? -E * D(R.d2, 0, j) * s2 * g0[3 + bcb] : ((j == 0) ? -1.0 : 0.0);
    }
    if (bc[0] == BC_VELOCITY) {
      if (b < 3) return (bcb == b && j == 0) ? 1.0 / ph.dt : 0.0;
      return (bcb < 3) ? 6.0 * E * c0 * g0[3 + bcb] * D(R.d3, 0, j) * s3 : 2.0 * c0 * D(R.d1, 0, j) * s1;
    }
    return 0.0;
  }
  if (b < 7) {
    const int a = b - 4;
    if (bc[1] == BC_TORQUE) return (bcb == a) ? D(R.d2, 0, j) * s2 : 0.0;
    if (bc[1] == BC_ANGULAR_VELOCITY) return (bcb == a) ? D(R.d1, 0, j) * s1 / ph.dt : 0.0;
    return 0.0;
  }
  if (b < 11) {
    if (bc[2] == BC_FORCE) {
      if (b < 10) {
        const int a = b - 7;
        return (bcb == a) ? -E * D(R.d3, last, j) * s3 : ((bcb == 3 && j == last) ? gl[a] : 0.0);
      }
      return (bcb < 3) ? E * D(R.d2, last, j) * s2 * gl[3 + bcb] : ((j == last) ? 1.0 : 0.0);
    }
    if (bc[2] == BC_VELOCITY) {
      if (b < 10) return (bcb == b - 7 && j == last) ? 1.0 / ph.dt : 0.0;
      return (bcb < 3) ? 6.0 * E * c0 * gl[3 + bcb] * D(R.d3, last, j) * s3
                       : 2.0 * c0 * D(R.d1, last, j) * s1;
    }
    return 0.0;
  }
  const int a = b - 11;
  if (bc[3] == BC_TORQUE) return (bcb == a) ? D(R.d2, last, j) * s2 : 0.0;
  return 0.0;
}

// Collocation rows of the operator by columns.  Element (row i of row
// block br, column j of column block bcb) of the 4n - 14 collocation rows is
//   e P_br[i][j] + sum_{|k - j| <= band} P_br[i][k] w[k],
// P_br = P_X (br < 3) or P_T (br = 3), with e and w fixed by (br, column):
//   br, bcb < 3:     e = [br == bcb] / dt,        w[k] = c_ab(k) D4[k][j] s4,
//                    c_aa = E c0 (1 + xs_a^2) + E c1 (1 - xs_a^2), c_ab = (E c0 - E c1) xs_a xs_b
//   br < 3, bcb = 3: e = -(c0 + c1) xss_a(j),     w[k] = -2 c0 xs_a(k) D1[k][j] s1
//   br = 3, bcb < 3: e = 0,  w[k] = -(c1 + 7 c0) E xss_b(k) D4 s4 - 6 c0 E xsss_b(k) D3 s3
//                                   - penalty xs_b(k) D1 s1
//   br = 3, bcb = 3: e = (c1 + c0) |xss(j)|^2,   w[k] = -2 c0 D2[k][j] s2
// (the same terms as assemble_element, fiber.py:322-448 projected as in
// fiber.py:810-961).  A thread owns one column: it forms w for one row block
// at a time (2 band + 1 values) and sweeps that block's rows, reading the
// projection rows from shared memory.
constexpr int kAsmMaxBand = 7;

template <int MAXBAND>
__device__ void assemble_columns(int n, int col, int ph, int tpc, const double *__restrict__ m,
                                 const ResLayout &R, const double *__restrict__ g,
                                 const double *__restrict__ xss2, const double *__restrict__ sPx,
                                 const double *__restrict__ sPt, const FiberPhys &ph_, double s1,
                                 int band, double *Af, double *Ac) {
  constexpr int W = 2 * MAXBAND + 1;
  const int nn = 4 * n;
  const double s2 = s1 * s1, s3 = s2 * s1, s4 = s3 * s1;
  const double E = ph_.E, c0 = ph_.c0, c1 = ph_.c1;
  const int bcb = col / n, j = col - bcb * n;
  const int kbase = j - band;
  for (int br = 0; br < 4; ++br) {
    double w[W];
    double e = 0.0;
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const int k = kbase + q;
      double v = 0.0;
      if (q <= 2 * band && k >= 0 && k < n) {
        const double *gk = g + 9 * k;
        if (br < 3 && bcb < 3) {
          const double xa = gk[br], xb = gk[bcb];
          const double c = (br == bcb) ? E * c0 * (1.0 + xa * xa) + E * c1 * (1.0 - xa * xa)
                                       : (E * c0 - E * c1) * xa * xb;
          v = c * (m[R.d4 + static_cast<int64_t>(k) * n + j] * s4);
        } else if (br < 3) {
          v = (-2.0 * c0 * gk[br]) * (m[R.d1 + static_cast<int64_t>(k) * n + j] * s1);
        } else if (bcb < 3) {
          v = -(c1 + 7.0 * c0) * E * gk[3 + bcb] * (m[R.d4 + static_cast<int64_t>(k) * n + j] * s4) -
              6.0 * c0 * E * gk[6 + bcb] * (m[R.d3 + static_cast<int64_t>(k) * n + j] * s3) -
              ph_.penalty * gk[bcb] * (m[R.d1 + static_cast<int64_t>(k) * n + j] * s1);
        } else {
          v = (-2.0 * c0) * (m[R.d2 + static_cast<int64_t>(k) * n + j] * s2);
        }
      }
      w[q] = v;
    }
    if (br < 3 && bcb < 3) e = (br == bcb) ? 1.0 / ph_.dt : 0.0;
    else if (br < 3) e = -(c0 + c1) * g[9 * j + 3 + br];
    else if (bcb == 3) e = (c1 + c0) * xss2[j];
    const int rows = (br < 3) ? n - 4 : n - 2;
    const int r0 = br * (n - 4);
    const double *P = (br < 3) ? sPx : sPt;
    for (int i = ph; i < rows; i += tpc) {
      const double *Pi = P + i * n;
      double s = e * Pi[j];
#pragma unroll
      for (int q = 0; q < W; ++q) {
        const int k = kbase + q;
        const int kc = k < 0 ? 0 : (k >= n ? n - 1 : k);  // w is 0 outside the fiber
        s = fma(Pi[kc], w[q], s);
      }
      const int64_t idx = static_cast<int64_t>(r0 + i) * nn + col;
      Af[idx] = s;
      if (Ac) Ac[idx] = s;
    }
  }
}

// One CTA per fiber.  Writes the operator block to A (and to A_copy if
// non-null) and the right-hand side block to rhs.  BANDED: the collocation
// rows by columns (assemble_columns, projection matrices staged in shared
// memory; needs 4n <= blockDim and band <= kAsmMaxBand), else element by
// element.
template <bool BANDED>
__global__ void __launch_bounds__(256, 2) fiber_assemble_kernel(
    FiberSet fs, FiberPhys ph, const double *__restrict__ x, const double *__restrict__ geo,
    const double *__restrict__ flow, const double *__restrict__ force, double *A, double *A_copy,
    double *rhs) {
  const int f = blockIdx.x;
  const int n = fs.n[f];
  const int64_t p0 = fs.pt_off[f];
  const double *m = fs.mats + fs.res_off[f];
  const ResLayout R(n);
  const double L = fs.length[f];
  const double s1 = 2.0 / L;
  const int32_t bc[4] = {fs.bc[4 * f], fs.bc[4 * f + 1], fs.bc[4 * f + 2], fs.bc[4 * f + 3]};
  extern __shared__ double sm[];
  double *g = sm;                  // 9n geometry
  double *xss2 = g + 9 * n;        // n   |xss|^2
  double *rfull = xss2 + n;        // 4n  unprojected right-hand side
  double *sP = rfull + 4 * n;      // BANDED: P_X ((n-4) x n) then P_T ((n-2) x n)
  for (int i = threadIdx.x; i < 9 * n; i += blockDim.x) g[i] = geo[9 * p0 + i];
  if (BANDED)
    for (int i = threadIdx.x; i < (2 * n - 6) * n; i += blockDim.x) sP[i] = m[R.px + i];
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double *gk = g + 9 * k;
    xss2[k] = gk[3] * gk[3] + gk[4] * gk[4] + gk[5] * gk[5];
    // compute_RHS (fiber.py:473-582), first order, no growth term
    const double *xk = x + 3 * (p0 + k);
    const double *vk = flow + 3 * (p0 + k);
    const double *fk = force + 3 * (p0 + k);
    const double xf = gk[0] * fk[0] + gk[1] * fk[1] + gk[2] * fk[2];
    for (int a = 0; a < 3; ++a)
      rfull[a * n + k] = xk[a] / ph.dt + vk[a] + ph.c0 * (fk[a] + gk[a] * xf) + ph.c1 * (fk[a] - gk[a] * xf);
    double dv[3] = {0, 0, 0}, df[3] = {0, 0, 0};
    const int j0 = max(0, k - fs.band), j1 = min(n - 1, k + fs.band);
    for (int j = j0; j <= j1; ++j) {
      const double w = m[R.d1 + static_cast<int64_t>(k) * n + j] * s1;
      for (int a = 0; a < 3; ++a) {
        dv[a] = fma(w, flow[3 * (p0 + j) + a], dv[a]);
        df[a] = fma(w, force[3 * (p0 + j) + a], df[a]);
      }
    }
    const double xss_f = gk[3] * fk[0] + gk[4] * fk[1] + gk[5] * fk[2];
    rfull[3 * n + k] = -ph.penalty + (gk[0] * dv[0] + gk[1] * dv[1] + gk[2] * dv[2]) +
                       2.0 * ph.c0 * (gk[0] * df[0] + gk[1] * df[1] + gk[2] * df[2]) +
                       (ph.c0 - ph.c1) * xss_f;
  }
  __syncthreads();
  const int nn = 4 * n;
  double *Af = A + fs.mat_off[f];
  double *Ac = A_copy ? A_copy + fs.mat_off[f] : nullptr;
  if (BANDED) {
    const int tpc = blockDim.x / nn;  // threads per column
    const int col = threadIdx.x % nn, phs = threadIdx.x / nn;
    if (phs < tpc) {
      assemble_columns<kAsmMaxBand>(n, col, phs, tpc, m, R, g, xss2, sP, sP + (n - 4) * n, ph, s1, fs.band,
                                    Af, Ac);
      // the 14 boundary rows
      for (int r = nn - 14 + phs; r < nn; r += tpc) {
        const double v = assemble_element(r, col, n, m, R, g, xss2, bc, ph, s1, fs.band);
        Af[static_cast<int64_t>(r) * nn + col] = v;
        if (Ac) Ac[static_cast<int64_t>(r) * nn + col] = v;
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < nn * nn; idx += blockDim.x) {
      const int r = idx / nn, col = idx - r * nn;
      const double v = assemble_element(r, col, n, m, R, g, xss2, bc, ph, s1, fs.band);
      Af[idx] = v;
      if (Ac) Ac[idx] = v;
    }
  }
  // projected right-hand side and boundary values
  double *rf = rhs + 4 * p0;
  const int nrect = nn - 14;
  for (int r = threadIdx.x; r < nn; r += blockDim.x) {
    double s = 0.0;
    if (r < nrect) {
      int br, i;
      if (r < n - 4) { br = 0; i = r; }
      else if (r < 2 * n - 8) { br = 1; i = r - (n - 4); }
      else if (r < 3 * n - 12) { br = 2; i = r - (2 * n - 8); }
      else { br = 3; i = r - (3 * n - 12); }
      const double *P = (br < 3) ? m + R.px + static_cast<int64_t>(i) * n : m + R.pt + static_cast<int64_t>(i) * n;
      for (int k = 0; k < n; ++k) s = fma(P[k], rfull[br * n + k], s);
    } else {
      const int b = r - nrect;
      const int last = n - 1;
      const double *g0 = g, *gl = g + 9 * last;
      const double *x0 = x + 3 * p0, *xl = x + 3 * (p0 + last);
      const double *v0 = flow + 3 * p0, *vl = flow + 3 * (p0 + last);
      const double *f0 = force + 3 * p0, *fl = force + 3 * (p0 + last);
      if (b < 4) {
        if (bc[0] == BC_VELOCITY) {
          if (b < 3) s = x0[b] / ph.dt;
          else s = -(v0[0] * g0[0] + v0[1] * g0[1] + v0[2] * g0[2]) -
                   2.0 * ph.c0 * (f0[0] * g0[0] + f0[1] * g0[1] + f0[2] * g0[2]);
        }
      } else if (b < 7) {
        if (bc[1] == BC_ANGULAR_VELOCITY) s = g0[b - 4] / ph.dt;
      } else if (b < 11) {
        if (bc[2] == BC_FORCE) {
          s = (b < 10) ? fl[b - 7] : fl[0] * gl[0] + fl[1] * gl[1] + fl[2] * gl[2];
        } else if (bc[2] == BC_VELOCITY) {
          if (b < 10) s = xl[b - 7] / ph.dt;
          else s = -(vl[0] * gl[0] + vl[1] * gl[1] + vl[2] * gl[2]) -
                   2.0 * ph.c0 * (fl[0] * gl[0] + fl[1] * gl[1] + fl[2] * gl[2]);
        }
      }
    }
    rf[r] = s;
  }
}

// ------------------------------------------------------------------ forces --
// fw[p] = w_p * f_p with f = -E X_ssss + xss T + xs T_s (force operator times
// the fiber unknowns XT), w_p = (L/2) w0 the trapezoid weights.
__global__ void fiber_forces_kernel(FiberSet fs, double E, const double *__restrict__ geo,
                                    const double *__restrict__ XT, double *fw, int64_t npts,
                                    int weighted) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int f = fs.pt_fib[p];
  const int n = fs.n[f];
  const int64_t p0 = fs.pt_off[f];
  const int k = static_cast<int>(p - p0);
  const double *m = fs.mats + fs.res_off[f];
  const ResLayout R(n);
  const double L = fs.length[f];
  const double s1 = 2.0 / L, s4 = s1 * s1 * s1 * s1;
  const double *X = XT + 4 * p0;
  const int j0 = max(0, k - fs.band), j1 = min(n - 1, k + fs.band);
  double d4[3] = {0, 0, 0}, dT = 0.0;
  for (int j = j0; j <= j1; ++j) {
    const double w4 = m[R.d4 + static_cast<int64_t>(k) * n + j];
    const double w1 = m[R.d1 + static_cast<int64_t>(k) * n + j];
    d4[0] = fma(w4, X[j], d4[0]);
    d4[1] = fma(w4, X[n + j], d4[1]);
    d4[2] = fma(w4, X[2 * n + j], d4[2]);
    dT = fma(w1, X[3 * n + j], dT);
  }
  const double T = X[3 * n + k];
  const double *gk = geo + 9 * p;
  const double w = weighted ? m[R.w0 + k] * (L / 2.0) : 1.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    fw[3 * p + a] = w * (-E * d4[a] * s4 + gk[3 + a] * T + gk[a] * dT * s1);
}

// Per-point external force times the trapezoid weight.
__global__ void fiber_weight_kernel(FiberSet fs, const double *__restrict__ f, double *fw,
                                    int64_t npts) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  const int fi = fs.pt_fib[p];
  const int n = fs.n[fi];
  const ResLayout R(n);
  const double w = fs.mats[fs.res_off[fi] + R.w0 + (p - fs.pt_off[fi])] * (fs.length[fi] / 2.0);
  fw[3 * p] = w * f[3 * p];
  fw[3 * p + 1] = w * f[3 * p + 1];
  fw[3 * p + 2] = w * f[3 * p + 2];
}

// ---------------------------------------------------------------- residual --
// res = A XT - [P_cheb [v_x; v_y; v_z; xs . D1 v]; 0]   (tstep.py:1147-1173)
__global__ void __launch_bounds__(256) fiber_residual_kernel(FiberSet fs,
                                                             const double *__restrict__ A,
                                                             const double *__restrict__ geo,
                                                             const double *__restrict__ XT,
                                                             const double *__restrict__ v,
                                                             double *res) {
  const int f = blockIdx.x;
  const int n = fs.n[f];
  const int64_t p0 = fs.pt_off[f];
  const double *m = fs.mats + fs.res_off[f];
  const ResLayout R(n);
  const double s1 = 2.0 / fs.length[f];
  extern __shared__ double sm[];
  double *vT = sm;           // 4n
  double *xt = vT + 4 * n;   // 4n
  const int nn = 4 * n;
  for (int i = threadIdx.x; i < nn; i += blockDim.x) xt[i] = XT[4 * p0 + i];
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double *vk = v + 3 * (p0 + k);
    vT[k] = vk[0];
    vT[n + k] = vk[1];
    vT[2 * n + k] = vk[2];
    double dv[3] = {0, 0, 0};
    const int j0 = max(0, k - fs.band), j1 = min(n - 1, k + fs.band);
    for (int j = j0; j <= j1; ++j) {
      const double w = m[R.d1 + static_cast<int64_t>(k) * n + j] * s1;
      dv[0] = fma(w, v[3 * (p0 + j)], dv[0]);
      dv[1] = fma(w, v[3 * (p0 + j) + 1], dv[1]);
      dv[2] = fma(w, v[3 * (p0 + j) + 2], dv[2]);
    }
    const double *gk = geo + 9 * (p0 + k);
    vT[3 * n + k] = gk[0] * dv[0] + gk[1] * dv[1] + gk[2] * dv[2];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double *Af = A + fs.mat_off[f];
  const int nrect = nn - 14;
  for (int r = warp; r < nn; r += nw) {
    const double *row = Af + static_cast<int64_t>(r) * nn;
    double s = 0.0;
    for (int c = lane; c < nn; c += 32) s = fma(row[c], xt[c], s);
    if (r < nrect) {
      int br, i;
      if (r < n - 4) { br = 0; i = r; }
      else if (r < 2 * n - 8) { br = 1; i = r - (n - 4); }
      else if (r < 3 * n - 12) { br = 2; i = r - (2 * n - 8); }
      else { br = 3; i = r - (3 * n - 12); }
      const double *P = (br < 3) ? m + R.px + static_cast<int64_t>(i) * n : m + R.pt + static_cast<int64_t>(i) * n;
      for (int k = lane; k < n; k += 32) s = fma(-P[k], vT[br * n + k], s);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) res[4 * p0 + r] = s;
  }
}

static int check_set(const FiberSet &fs) {
  if (fs.nfib < 0) return F3D_ERR_SHAPE;
  if (fs.nfib == 0) return F3D_OK;
  if (!fs.n || !fs.pt_off || !fs.mat_off || !fs.res_off || !fs.length || !fs.bc || !fs.pt_fib ||
      !fs.mats)
    return F3D_ERR_NULL;
  if (fs.band < 0) return F3D_ERR_ARG;
  return F3D_OK;
}

}  // namespace f3d

extern "C" {

int f3d_fiber_geometry(const f3d_fiber_set *set, const double *x, double *geo, int64_t npts,
                       void *stream) {
  if (!set) return F3D_ERR_NULL;
  f3d::FiberSet fs{set->nfib, set->n, set->pt_off, set->mat_off, set->res_off, set->length,
                   set->bc, set->pt_fib, set->mats, set->band};
  int rc = f3d::check_set(fs);
  if (rc || npts == 0) return rc;
  if (!x || !geo) return F3D_ERR_NULL;
  f3d::fiber_geometry_kernel<<<static_cast<unsigned>((npts + 127) / 128), 128, 0,
                               static_cast<cudaStream_t>(stream)>>>(fs, x, geo, npts);
  return f3d::launch_status();
}

int f3d_fiber_assemble(const f3d_fiber_set *set, double E, double dt, double c0, double c1,
                       double penalty, const double *x, const double *geo, const double *flow,
                       const double *force, double *A, double *A_copy, double *rhs, int32_t max_n,
                       void *stream) {
  if (!set) return F3D_ERR_NULL;
  f3d::FiberSet fs{set->nfib, set->n, set->pt_off, set->mat_off, set->res_off, set->length,
                   set->bc, set->pt_fib, set->mats, set->band};
  int rc = f3d::check_set(fs);
  if (rc || fs.nfib == 0) return rc;
  if (!x || !geo || !flow || !force || !A || !rhs) return F3D_ERR_NULL;
  if (max_n < 5) return F3D_ERR_SHAPE;
  f3d::FiberPhys ph{E, dt, c0, c1, penalty};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  constexpr int kThreads = 256;
  if (4 * max_n <= kThreads && fs.band <= f3d::kAsmMaxBand) {
    // columns of every fiber fit one CTA: projection matrices staged in shared memory
    const size_t smem = (static_cast<size_t>(14) * max_n + static_cast<size_t>(2 * max_n - 6) * max_n) * sizeof(double);
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(f3d::fiber_assemble_kernel<true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess) return F3D_ERR_CUDA;
    }
    f3d::fiber_assemble_kernel<true><<<fs.nfib, kThreads, smem, st>>>(fs, ph, x, geo, flow, force, A, A_copy, rhs);
  } else {
    const size_t smem = static_cast<size_t>(14) * max_n * sizeof(double);
    f3d::fiber_assemble_kernel<false><<<fs.nfib, kThreads, smem, st>>>(fs, ph, x, geo, flow, force, A, A_copy,
                                                                        rhs);
  }
  return f3d::launch_status();
}

int f3d_fiber_forces(const f3d_fiber_set *set, double E, const double *geo, const double *XT,
                     double *fw, int64_t npts, int weighted, void *stream) {
  if (!set) return F3D_ERR_NULL;
  f3d::FiberSet fs{set->nfib, set->n, set->pt_off, set->mat_off, set->res_off, set->length,
                   set->bc, set->pt_fib, set->mats, set->band};
  int rc = f3d::check_set(fs);
  if (rc || npts == 0) return rc;
  if (!geo || !XT || !fw) return F3D_ERR_NULL;
  f3d::fiber_forces_kernel<<<static_cast<unsigned>((npts + 127) / 128), 128, 0,
                             static_cast<cudaStream_t>(stream)>>>(fs, E, geo, XT, fw, npts, weighted);
  return f3d::launch_status();
}

int f3d_fiber_weight(const f3d_fiber_set *set, const double *f, double *fw, int64_t npts,
                     void *stream) {
  if (!set) return F3D_ERR_NULL;
  f3d::FiberSet fs{set->nfib, set->n, set->pt_off, set->mat_off, set->res_off, set->length,
                   set->bc, set->pt_fib, set->mats, set->band};
  int rc = f3d::check_set(fs);
  if (rc || npts == 0) return rc;
  if (!f || !fw) return F3D_ERR_NULL;
  f3d::fiber_weight_kernel<<<static_cast<unsigned>((npts + 127) / 128), 128, 0,
                             static_cast<cudaStream_t>(stream)>>>(fs, f, fw, npts);
  return f3d::launch_status();
}

int f3d_fiber_residual(const f3d_fiber_set *set, const double *A, const double *geo,
                       const double *XT, const double *v, double *res, int32_t max_n,
                       void *stream) {
  if (!set) return F3D_ERR_NULL;
  f3d::FiberSet fs{set->nfib, set->n, set->pt_off, set->mat_off, set->res_off, set->length,
                   set->bc, set->pt_fib, set->mats, set->band};
  int rc = f3d::check_set(fs);
  if (rc || fs.nfib == 0) return rc;
  if (!A || !geo || !XT || !v || !res) return F3D_ERR_NULL;
  const size_t smem = static_cast<size_t>(8) * max_n * sizeof(double);
  f3d::fiber_residual_kernel<<<fs.nfib, 256, smem, static_cast<cudaStream_t>(stream)>>>(
      fs, A, geo, XT, v, res);
  return f3d::launch_status();
}

}  // extern "C"
