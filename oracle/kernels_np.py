"""numpy restatement of fiber3d's Green's-function sums (test oracle).

Each function follows the reference function named in its docstring
(``python/kernels/kernels.py`` of bioflume/fiber3d; the effective, i.e.
later, definitions).  Loops over targets are vectorised in chunks so memory
stays bounded; arithmetic is float64 throughout.  Test infrastructure only.
"""
from __future__ import annotations

import numpy as np

CHUNK = 512


def _pts(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    return a.reshape(a.size // 3, 3)


def _pair_geometry(xt: np.ndarray, xs: np.ndarray, reg: float, eps: float):
    """r = x_t - x_s and |r|, with |r| < eps replaced by sqrt(|r|^2 + reg^2)
    (kernels.py:826-829, the regularised branch of every numba kernel)."""
    r = xt[:, None, :] - xs[None, :, :]
    rn = np.sqrt(np.einsum("tsk,tsk->ts", r, r))
    close = rn < eps
    rn = np.where(close, np.sqrt(rn * rn + reg * reg), rn)
    return r, rn


def oseen_kernel_source_target(r_source, r_target, density, eta=1.0, reg=5e-3,
                               epsilon_distance=1e-5, skip_index=False, src_group=None,
                               trg_group=None):
    """oseen_kernel_source_target_numba, kernels.py:794-846 (skip_index=True gives
    oseen_kernel_times_density_numba, kernels.py:214-287, which skips yn == xn).
    With src_group/trg_group, pairs with equal group id are skipped (fused
    flow_fibers + self_flow_fibers, tstep_utils.py:653-700, 812-851)."""
    xs, xt, f = _pts(r_source), _pts(r_target), _pts(density)
    factor = 1.0 / (8.0 * np.pi * eta)
    u = np.zeros_like(xt)
    for t0 in range(0, xt.shape[0], CHUNK):
        t1 = min(t0 + CHUNK, xt.shape[0])
        r, rn = _pair_geometry(xt[t0:t1], xs, reg, epsilon_distance)
        fr = factor / rn
        gr = factor / rn**3
        if skip_index:
            idx = np.arange(t0, t1)
            fr[idx - t0, idx] = 0.0
            gr[idx - t0, idx] = 0.0
        if src_group is not None:
            same = np.asarray(trg_group)[t0:t1, None] == np.asarray(src_group)[None, :]
            fr[same] = 0.0
            gr[same] = 0.0
        rf = np.einsum("tsk,sk->ts", r, f)
        u[t0:t1] = fr @ f + np.einsum("ts,tsk->tk", gr * rf, r)
    return u.reshape(-1)


def oseen_kernel_times_density(r_vectors, density, eta=1.0, reg=5e-3, epsilon_distance=1e-5):
    """oseen_kernel_times_density_numba, kernels.py:214-287."""
    return oseen_kernel_source_target(r_vectors, r_vectors, density, eta, reg, epsilon_distance,
                                      skip_index=True)


def rotlet_kernel_source_target(r_source, r_target, density, eta=1.0, reg=5e-3,
                                epsilon_distance=1e-5):
    """rotlet_kernel_source_target_numba, kernels.py:856-908:
    u_x += fr (z tau_y - y tau_z), u_y += fr (x tau_z - z tau_x),
    u_z += fr (y tau_x - x tau_y), fr = 1/(8 pi eta r^3)."""
    xs, xt, tau = _pts(r_source), _pts(r_target), _pts(density)
    factor = 1.0 / (8.0 * np.pi * eta)
    u = np.zeros_like(xt)
    for t0 in range(0, xt.shape[0], CHUNK):
        t1 = min(t0 + CHUNK, xt.shape[0])
        r, rn = _pair_geometry(xt[t0:t1], xs, reg, epsilon_distance)
        fr = factor / rn**3
        x, y, z = r[..., 0], r[..., 1], r[..., 2]
        u[t0:t1, 0] = np.sum(fr * (z * tau[None, :, 1] - y * tau[None, :, 2]), axis=1)
        u[t0:t1, 1] = np.sum(fr * (x * tau[None, :, 2] - z * tau[None, :, 0]), axis=1)
        u[t0:t1, 2] = np.sum(fr * (y * tau[None, :, 0] - x * tau[None, :, 1]), axis=1)
    return u.reshape(-1)


def stresslet_kernel_source_target(r_source, r_target, normal, density, eta=1.0, reg=5e-3,
                                   epsilon_distance=1e-5, skip_index=False):
    """stresslet_kernel_source_target_numba, kernels.py:1186-1217:
    v_t = -3/(4 pi eta) sum_s (r.d_s)(r.n_s) r / r^5.  skip_index=True gives
    stresslet_kernel_times_normal_times_density_numba, kernels.py:1123-1183."""
    xs, xt, n, d = _pts(r_source), _pts(r_target), _pts(normal), _pts(density)
    factor = -3.0 / (4.0 * np.pi * eta)
    v = np.zeros_like(xt)
    for t0 in range(0, xt.shape[0], CHUNK):
        t1 = min(t0 + CHUNK, xt.shape[0])
        r, rn = _pair_geometry(xt[t0:t1], xs, reg, epsilon_distance)
        w = factor / rn**5 * np.einsum("tsk,sk->ts", r, d) * np.einsum("tsk,sk->ts", r, n)
        if skip_index:
            idx = np.arange(t0, t1)
            w[idx - t0, idx] = 0.0
        v[t0:t1] = np.einsum("ts,tsk->tk", w, r)
    return v.reshape(-1)


def stresslet_kernel_times_normal_times_density(r_vectors, normal, density, eta=1.0, reg=5e-3,
                                                epsilon_distance=1e-5):
    """stresslet_kernel_times_normal_times_density_numba, kernels.py:1123-1183."""
    return stresslet_kernel_source_target(r_vectors, r_vectors, normal, density, eta, reg,
                                          epsilon_distance, skip_index=True)


def stresslet_kernel_times_normal_dense(r_vectors, normal, eta=1.0, reg=5e-3,
                                        epsilon_distance=1e-5):
    """stresslet_kernel_times_normal_numba, kernels.py:1063-1120: block
    (i, j) = factor (r.n_j)/r^5 r r^T, r = x_i - x_j, zero diagonal blocks."""
    x, n = _pts(r_vectors), _pts(normal)
    N = x.shape[0]
    factor = -3.0 / (4.0 * np.pi * eta)
    r = x[:, None, :] - x[None, :, :]
    rn = np.sqrt(np.einsum("ijk,ijk->ij", r, r))
    rn = np.where(rn < epsilon_distance, np.sqrt(rn * rn + reg * reg), rn)
    s = factor * np.einsum("ijk,jk->ij", r, n) / rn**5
    np.fill_diagonal(s, 0.0)
    # M[i, a, j, b] = s_ij r_ij[a] r_ij[b]
    M = np.einsum("ij,ija,ijb->iajb", s, r, r)
    return M.reshape(3 * N, 3 * N)


def oseen_tensor(r_vectors, eta=1.0, reg=5e-3, epsilon_distance=1e-5, input_format='r'):
    """oseen_tensor, kernels.py:31-116 ('r' layout; 'xyz' input permuted)."""
    N = np.size(r_vectors) // 3
    if input_format == 'r':
        x = _pts(r_vectors)
    else:
        x = np.asarray(r_vectors, dtype=np.float64).reshape(3, N).T
    return oseen_tensor_source_target(x, x, eta, reg, epsilon_distance, input_format='r',
                                      _xyz=(input_format != 'r'))


def oseen_tensor_source_target(r_source, r_target, eta=1.0, reg=5e-3, epsilon_distance=1e-5,
                               input_format='r', _xyz=False):
    """oseen_tensor_source_target, kernels.py:119-211: r = x_s - x_t; dr > eps plain,
    dr <= eps regularised."""
    Ns, Nt = np.size(r_source) // 3, np.size(r_target) // 3
    if input_format == 'r':
        xs, xt = _pts(r_source), _pts(r_target)
    else:
        xs = np.asarray(r_source, dtype=np.float64).reshape(3, Ns).T
        xt = np.asarray(r_target, dtype=np.float64).reshape(3, Nt).T
        _xyz = True
    r = xs[None, :, :] - xt[:, None, :]
    dr = np.sqrt(np.einsum("tsk,tsk->ts", r, r))
    sel = dr > epsilon_distance
    d = np.where(sel, dr, np.sqrt(dr**2 + reg**2))
    fr = 1.0 / (8.0 * np.pi * eta * d)
    gr = 1.0 / (8.0 * np.pi * eta * d**3)
    G = fr[:, None, :, None] * np.eye(3)[None, :, None, :] + np.einsum("ts,tsa,tsb->tasb", gr, r, r)
    G = G.reshape(3 * Nt, 3 * Ns)
    if _xyz:
        pt = (np.arange(3)[:, None] + 3 * np.arange(Nt)[None, :]).reshape(-1)
        ps = (np.arange(3)[:, None] + 3 * np.arange(Ns)[None, :]).reshape(-1)
        G = G[pt][:, ps]
    return G


def complementary_kernel(r_vectors, normal):
    """complementary_kernel, kernels.py:1286-1295."""
    n = np.asarray(normal, dtype=np.float64).reshape(-1)
    return np.outer(n, n)


def complementary_kernel_times_density(r_vectors, normal, density):
    """complementary_kernel_times_density_numba, kernels.py:1267-1283."""
    n, d = _pts(normal), _pts(density)
    return (n * np.sum(n * d)).reshape(-1)


def traction_kernel_times_normal_times_density(r_vectors, normal, density, eta=1.0, reg=5e-3,
                                               epsilon_distance=1e-5):
    """traction_kernel_times_normal_times_density_numba, kernels.py:1221-1264:
    t_i = -3/(4 pi eta) sum_{j != i} (r.d_j)(r.n_i) r / r^5, r = x_i - x_j (the
    normal of the target; the eta = 1.0 at :1232 follows the prefactor)."""
    x, n, d = _pts(r_vectors), _pts(normal), _pts(density)
    factor = -3.0 / (4.0 * np.pi * eta)
    v = np.zeros_like(x)
    for t0 in range(0, x.shape[0], CHUNK):
        t1 = min(t0 + CHUNK, x.shape[0])
        r, rn = _pair_geometry(x[t0:t1], x, reg, epsilon_distance)
        w = factor / rn**5 * np.einsum("tsk,sk->ts", r, d) * np.einsum("tsk,tk->ts", r, n[t0:t1])
        idx = np.arange(t0, t1)
        w[idx - t0, idx] = 0.0
        v[t0:t1] = np.einsum("ts,tsk->tk", w, r)
    return v.reshape(-1)


def stresslet_kernel(r_vectors, eta=1.0, reg=5e-3, epsilon_distance=1e-5, input_format='r'):
    """stresslet_kernel, kernels.py:911-992: S[3i+a, 3j+b, c] = fr dr_a dr_b dr_c,
    dr = x_j - x_i, fr = -3/(4 pi eta dr^5) for dr > eps, -3/(4 pi eta
    (dr^2 + reg^2)^2.5) otherwise."""
    N = np.size(r_vectors) // 3
    x = _pts(r_vectors) if input_format == 'r' else np.asarray(r_vectors, dtype=np.float64).reshape(3, N).T
    dr = x[None, :, :] - x[:, None, :]
    d = np.sqrt(np.einsum("ijk,ijk->ij", dr, dr))
    fr = np.where(d > epsilon_distance, -3.0 / (4.0 * np.pi * eta * np.where(d > 0, d, 1.0) ** 5),
                  -3.0 / (4.0 * np.pi * eta * np.power(d**2 + reg**2, 2.5)))
    S = np.einsum("ij,ija,ijb,ijc->iajbc", fr, dr, dr, dr)
    return S.reshape(3 * N, 3 * N, 3)


def oseen_kernel_source_target_skip_close(r_source, r_target, density, eta=1.0, epsilon_distance=1e-5):
    """Oseen source -> target sum without regularisation in which pairs with
    |r| < epsilon_distance contribute nothing: fiber3d's PyCUDA kernel
    (kernels/kernels_pycuda.py:22-66, reached from kernels.py:849) and, with
    a vanishing epsilon_distance, the coincident-point exclusion of the
    STKFMM-backed sums (kernels.py:1298-1364)."""
    xs, xt, f = _pts(r_source), _pts(r_target), _pts(density)
    factor = 1.0 / (8.0 * np.pi * eta)
    u = np.zeros_like(xt)
    for t0 in range(0, xt.shape[0], CHUNK):
        t1 = min(t0 + CHUNK, xt.shape[0])
        r = xt[t0:t1, None, :] - xs[None, :, :]
        rn = np.sqrt(np.einsum("tsk,tsk->ts", r, r))
        keep = rn >= epsilon_distance
        rs = np.where(keep, rn, 1.0)
        fr = np.where(keep, factor / rs, 0.0)
        gr = np.where(keep, factor / rs**3, 0.0)
        u[t0:t1] = fr @ f + np.einsum("ts,tsk->tk", gr * np.einsum("tsk,sk->ts", r, f), r)
    return u.reshape(-1)


def stresslet_kernel_source_target_skip_close(r_source, r_target, normal, density, eta=1.0,
                                              epsilon_distance=1e-150):
    """Stresslet source -> target sum without regularisation, pairs with
    |r| < epsilon_distance left out: the direct-sum value of fiber3d's
    STKFMM double layer with its 2 (n (x) d) density (kernels.py:1367-1419)."""
    xs, xt, n, d = _pts(r_source), _pts(r_target), _pts(normal), _pts(density)
    factor = -3.0 / (4.0 * np.pi * eta)
    v = np.zeros_like(xt)
    for t0 in range(0, xt.shape[0], CHUNK):
        t1 = min(t0 + CHUNK, xt.shape[0])
        r = xt[t0:t1, None, :] - xs[None, :, :]
        rn = np.sqrt(np.einsum("tsk,tsk->ts", r, r))
        keep = rn >= epsilon_distance
        rs = np.where(keep, rn, 1.0)
        w = np.where(keep, factor / rs**5, 0.0) * np.einsum("tsk,sk->ts", r, d) * np.einsum("tsk,sk->ts", r, n)
        v[t0:t1] = np.einsum("ts,tsk->tk", w, r)
    return v.reshape(-1)
