"""CPU restatement of fiber3d's fiber discretisation (test oracle).

* :func:`fornberg_weights` — finite-difference weights by Fornberg's
  recursion (B. Fornberg, SIAM Rev. 40 (1998) 685), with the stencil choice
  of python/utils/finite_diff.py:4-63.
* :func:`barycentric_matrix` — resampling matrix of python/utils/
  barycentricMatrix.py:12-45 (Driscoll & Hale rectangular collocation).
* :class:`FiberMatrices` — python/tstep/fiber_matrices.py:38-153.
* :func:`linear_operator`, :func:`rhs`, :func:`apply_bc_rectangular`,
  :func:`force_operator` — python/fiber/fiber.py:322-448, 473-582, 810-961,
  1399-1432.

Test infrastructure only.
"""
from __future__ import annotations

import numpy as np


def fornberg_weights(s: np.ndarray, m: int, n_s: int) -> np.ndarray:
    """D[i, j, k]: weight of s_j in the k-th derivative at s_i (k <= m), on a
    stencil of n_s consecutive nodes (finite_diff.py:4-63)."""
    n = s.size
    D = np.zeros((n, n, m + 1))
    half = (n_s - 1) // 2
    last = n_s - 1
    for i in range(n):
        if i < half:
            j0 = 0
        elif i > n - half - 2:
            j0 = n - last - 1
        else:
            j0 = i - half
        x = s[j0:j0 + last + 1]
        z = s[i]
        c = np.zeros((last + 1, m + 1))
        c[0, 0] = 1.0
        c1 = 1.0
        c4 = x[0] - z
        for a in range(1, last + 1):
            mn = min(a, m)
            c2 = 1.0
            c5 = c4
            c4 = x[a] - z
            for b in range(a):
                c3 = x[a] - x[b]
                c2 *= c3
                if b == a - 1:
                    for k in range(mn, 0, -1):
                        c[a, k] = c1 * (k * c[a - 1, k - 1] - c5 * c[a - 1, k]) / c2
                    c[a, 0] = -c1 * c5 * c[a - 1, 0] / c2
                for k in range(mn, 0, -1):
                    c[b, k] = (c4 * c[b, k] - k * c[b, k - 1]) / c3
                c[b, 0] = c4 * c[b, 0] / c3
            c1 = c2
        D[i, j0:j0 + last + 1, :] = c
    return D


def barycentric_matrix(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """P[j, k] resampling values at nodes x to points y with weights
    (1/2, -1, 1, -1, ..., -(-1)^N/2) (barycentricMatrix.py:12-45)."""
    x = np.asarray(x, dtype=np.float64).ravel()
    y = np.asarray(y, dtype=np.float64).ravel()
    N = x.size
    w = np.ones(N)
    w[1::2] = -1.0
    w[0] = 0.5
    w[-1] = -0.5 * (-1) ** N
    with np.errstate(divide="ignore", invalid="ignore"):
        yx = y[:, None] - x[None, :]
        wyx = w[None, :] / yx
        P = wyx / np.sum(wyx, axis=1)[:, None]
    P[yx == 0] = 1.0
    return P


class FiberMatrices:
    """Per-resolution matrices (fiber_matrices.py:38-104): D1..D4 on
    alpha = linspace(-1, 1, N) with supports n_fd+1..n_fd+4, trapezoid
    weights, P_X (N-4 interior midpoints), P_T (N-2), and the (4N-14) x 4N
    projector."""

    def __init__(self, N: int, n_fd: int = 4):
        self.N = N
        a = np.linspace(-1.0, 1.0, N)
        self.alpha = a
        nr, nt = N - 4, N - 2
        self.alpha_roots = 2 * (0.5 + np.arange(nr)) / nr - 1
        self.alpha_tension = 2 * (0.5 + np.arange(nt)) / nt - 1
        self.D0 = [fornberg_weights(a, k, n_fd + k)[:, :, k] for k in (1, 2, 3, 4)]
        w = np.full(N, 2.0)
        w[0] = w[-1] = 1.0
        self.weights0 = w / (N - 1)
        self.PX = barycentric_matrix(a, self.alpha_roots)
        self.PT = barycentric_matrix(a, self.alpha_tension)
        P = np.zeros((4 * N - 14, 4 * N))
        P[0:N - 4, 0:N] = self.PX
        P[N - 4:2 * N - 8, N:2 * N] = self.PX
        P[2 * N - 8:3 * N - 12, 2 * N:3 * N] = self.PX
        P[3 * N - 12:4 * N - 14, 3 * N:4 * N] = self.PT
        self.Pcheb = P

    def D(self, length: float):
        """Scaled derivative matrices D_k (2/L)^k (get_matrices 'Ds')."""
        return [d * (2.0 / length) ** (k + 1) for k, d in enumerate(self.D0)]

    def weights(self, length: float):
        return self.weights0 * (length / 2.0)


def mobility_constants(epsilon: float = 1e-3, eta: float = 1.0):
    """c0, c1 of slender-body theory (fiber.py:83-84)."""
    c0 = -np.log(np.e * epsilon**2) / (8.0 * np.pi * eta)
    c1 = 2.0 / (8.0 * np.pi * eta)
    return c0, c1


def derivatives(fm: FiberMatrices, x: np.ndarray, length: float):
    D1, D2, D3, D4 = fm.D(length)
    return D1 @ x, D2 @ x, D3 @ x, D4 @ x


def linear_operator(fm, x, length, E, dt, c0, c1, penalty=500.0, beta_tstep=1.0):
    """A (4N x 4N) of fiber.form_linear_operator (fiber.py:322-448), penalty
    inextensibility, no non-local term."""
    N = fm.N
    D1, D2, D3, D4 = fm.D(length)
    xs, xss, xsss, _ = derivatives(fm, x, length)
    I = np.eye(N)
    dg = lambda v, Dm: v[:, None] * Dm  # diag(v) @ Dm
    blocks = {}
    for a in range(3):
        for b in range(a, 3):
            if a == b:
                blocks[a, b] = beta_tstep * I / dt + E * c0 * dg(1 + xs[:, a] ** 2, D4) \
                    + E * c1 * dg(1 - xs[:, a] ** 2, D4)
            else:
                blocks[a, b] = (E * c0 - E * c1) * dg(xs[:, a] * xs[:, b], D4)
            blocks[b, a] = blocks[a, b]
    AT = [-c0 * (2.0 * dg(xs[:, a], D1) + np.diag(xss[:, a])) - c1 * np.diag(xss[:, a]) for a in range(3)]
    TA = [-(c1 + 7.0 * c0) * E * dg(xss[:, a], D4) - 6.0 * c0 * E * dg(xsss[:, a], D3)
          - penalty * dg(xs[:, a], D1) for a in range(3)]
    TT = -2.0 * c0 * D2 + (c1 + c0) * np.diag(np.sum(xss**2, axis=1))
    A = np.zeros((4 * N, 4 * N))
    for a in range(3):
        for b in range(3):
            A[a * N:(a + 1) * N, b * N:(b + 1) * N] = blocks[a, b]
        A[a * N:(a + 1) * N, 3 * N:] = AT[a]
        A[3 * N:, a * N:(a + 1) * N] = TA[a]
    A[3 * N:, 3 * N:] = TT
    return A


def rhs(fm, x, length, dt, c0, c1, force=None, flow=None, penalty=500.0, v_length=0.0):
    """RHS of fiber.compute_RHS (fiber.py:473-582), first order."""
    N = fm.N
    D1 = fm.D(length)[0]
    xs, xss, _, _ = derivatives(fm, x, length)
    R = np.zeros(4 * N)
    for a in range(3):
        R[a * N:(a + 1) * N] = x[:, a] / dt + (fm.alpha + 1.0) * (v_length * 0.5) * xs[:, a]
    R[3 * N:] = -penalty
    if flow is not None:
        for a in range(3):
            R[a * N:(a + 1) * N] += flow[:, a]
        R[3 * N:] += np.sum(xs * (D1 @ flow), axis=1)
    if force is not None:
        fs = D1 @ force
        xf = np.sum(xs * force, axis=1)
        for a in range(3):
            R[a * N:(a + 1) * N] += c0 * (force[:, a] + xs[:, a] * xf) + c1 * (force[:, a] - xs[:, a] * xf)
        R[3 * N:] += 2 * c0 * np.sum(xs * fs, axis=1) + (c0 - c1) * np.sum(xss * force, axis=1)
    return R


def bc_rows(fm, x, length, E, dt, c0, bc=("force", "torque", "force", "torque"),
            start_vec0=None, start_vec1=None, end_vec0=None, end_vec1=None,
            v_on_fiber=None, force_on_fiber=None, beta_tstep=1.0):
    """The 14 boundary-condition rows B (14 x 4N) and their right-hand side
    (fiber.apply_BC_rectangular, fiber.py:838-955)."""
    N = fm.N
    D1, D2, D3, _ = fm.D(length)
    xs, xss, _, _ = derivatives(fm, x, length)
    z3 = np.zeros(3)
    sv0 = z3 if start_vec0 is None else start_vec0
    sv1 = z3 if start_vec1 is None else start_vec1
    ev0 = z3 if end_vec0 is None else end_vec0
    ev1 = z3 if end_vec1 is None else end_vec1
    B = np.zeros((14, 4 * N))
    r = np.zeros(14)
    b0, b1, e0, e1 = bc
    if b0 == "force":
        for a in range(3):
            B[a, a * N:(a + 1) * N] = E * D3[0]
            B[a, 3 * N] = -xs[0, a]
            B[3, a * N:(a + 1) * N] = -E * D2[0] * xss[0, a]
        B[3, 3 * N] = -1.0
        r[0:3] = sv0
        r[3] = sv0 @ xs[0]
    elif b0 == "velocity":
        for a in range(3):
            B[a, a * N] = beta_tstep / dt
            B[3, a * N:(a + 1) * N] = 6.0 * E * c0 * xss[0, a] * D3[0]
            r[a] = x[0, a] / dt + sv0[a]
        B[3, 3 * N:] = 2.0 * c0 * D1[0]
        if v_on_fiber is not None:
            r[3] += -(v_on_fiber[0] @ xs[0])
        if force_on_fiber is not None:
            r[3] += -2 * c0 * (force_on_fiber[0] @ xs[0])
    if b1 == "torque":
        for a in range(3):
            B[4 + a, a * N:(a + 1) * N] = D2[0]
            r[4 + a] = sv1[a]
    elif b1 == "angular_velocity":
        for a in range(3):
            B[4 + a, a * N:(a + 1) * N] = beta_tstep * D1[0] / dt
        ld = x[0] / np.linalg.norm(x[0])
        om = sv1
        r[4] = xs[0, 0] / dt + om[1] * ld[2] - om[2] * ld[1]
        r[5] = xs[0, 1] / dt + om[2] * ld[0] - om[0] * ld[2]
        r[6] = xs[0, 2] / dt + om[0] * ld[1] - om[1] * ld[0]
    if e0 == "force":
        for a in range(3):
            B[7 + a, a * N:(a + 1) * N] = -E * D3[-1]
            B[7 + a, 4 * N - 1] = xs[-1, a]
            B[10, a * N:(a + 1) * N] = E * D2[-1] * xss[-1, a]
        B[10, 4 * N - 1] = 1.0
        r[7:10] = ev0
        r[10] = ev0 @ xs[-1]
    if e1 == "torque":
        for a in range(3):
            B[11 + a, a * N:(a + 1) * N] = D2[-1]
            r[11 + a] = ev1[a]
    if e0 == "velocity":
        for a in range(3):
            B[7 + a, a * N + N - 1] = beta_tstep / dt
            B[10, a * N:(a + 1) * N] = 6.0 * E * c0 * xss[-1, a] * D3[-1]
            r[7 + a] = x[-1, a] / dt + ev0[a]
        B[10, 3 * N:] = 2.0 * c0 * D1[-1]
        r[10] = 0.0
        if v_on_fiber is not None:
            r[10] += -(v_on_fiber[-1] @ xs[-1])
        if force_on_fiber is not None:
            r[10] += -2 * c0 * (force_on_fiber[-1] @ xs[-1])
    return B, r


def apply_bc_rectangular(fm, A, R, B, r):
    """[P_cheb A; B] and [P_cheb R; r] (fiber.py:835-836, 957-961)."""
    return np.vstack([fm.Pcheb @ A, B]), np.concatenate([fm.Pcheb @ R, r])


def force_operator(fm, x, length, E):
    """f = -E X_ssss + (T X_s)_s as a 3N x 4N matrix (fiber.py:1399-1432)."""
    N = fm.N
    D1, _, _, D4 = fm.D(length)
    xs, xss, _, _ = derivatives(fm, x, length)
    F = np.zeros((3 * N, 4 * N))
    for a in range(3):
        F[a * N:(a + 1) * N, a * N:(a + 1) * N] = -E * D4
        F[a * N:(a + 1) * N, 3 * N:] = np.diag(xss[:, a]) + xs[:, a][:, None] * D1
    return F


def self_mobility(xs: np.ndarray, c0: float, c1: float) -> np.ndarray:
    """fiber.self_mobility, fiber/fiber.py:964-993: the 3N x 3N local
    slender-body mobility in fiber3d's (x_all, y_all, z_all) ordering,
    M_ab = c0 (delta_ab I + diag(xs_a xs_b)) + c1 (delta_ab I - diag(xs_a xs_b))."""
    n = xs.shape[0]
    I = np.eye(n)
    M = np.zeros((3 * n, 3 * n))
    for a in range(3):
        for b in range(3):
            d = np.diag(xs[:, a] * xs[:, b])
            M[a * n:(a + 1) * n, b * n:(b + 1) * n] = c0 * ((a == b) * I + d) + c1 * ((a == b) * I - d)
    return M
