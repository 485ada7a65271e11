"""Fiber discretisation set-up: per-resolution matrices and the device
descriptor of a set of fibers (``f3d_fiber_set`` in include/fiber3d_b200.h).

Per resolution N (computed once on the host, like fiber3d's
``tstep/fiber_matrices.py:38-104`` cache, and uploaded):

* D1_0..D4_0: finite-difference differentiation matrices on the equispaced
  parameter nodes alpha = linspace(-1, 1, N), derivative k on a stencil of
  n_fd + k points (Fornberg's weight recursion; stencil choice of
  ``utils/finite_diff.py:4-63``); D_k = D_k_0 (2/L)^k.
* P_X ((N-4) x N) and P_T ((N-2) x N): barycentric resampling onto the
  interior midpoints (``utils/barycentricMatrix.py:12-45``), the
  rectangular-collocation projectors.
* w0: trapezoid weights 2/(N-1) (1/(N-1) at the ends).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

N_FD = 4


def fd_weights(nodes: np.ndarray, order: int, support: int) -> np.ndarray:
    """(N, N) matrix of the `order`-th derivative on `support`-point stencils.

    Row i uses the `support` consecutive nodes centred on i, shifted inward
    at the ends; weights from Fornberg's recursion (B. Fornberg, Math. Comp.
    51 (1988) 699; SIAM Rev. 40 (1998) 685).
    """
    n = nodes.size
    out = np.zeros((n, n))
    half = (support - 1) // 2
    for i in range(n):
        j0 = min(max(i - half, 0), n - support)
        x = nodes[j0:j0 + support]
        z = nodes[i]
        c = np.zeros((support, order + 1))
        c[0, 0] = 1.0
        prod_prev = 1.0
        dz_prev = x[0] - z
        for a in range(1, support):
            mn = min(a, order)
            prod = 1.0
            dz_a_prev = dz_prev
            dz_prev = x[a] - z
            for b in range(a):
                d = x[a] - x[b]
                prod *= d
                if b == a - 1:
                    for k in range(mn, 0, -1):
                        c[a, k] = prod_prev * (k * c[a - 1, k - 1] - dz_a_prev * c[a - 1, k]) / prod
                    c[a, 0] = -prod_prev * dz_a_prev * c[a - 1, 0] / prod
                for k in range(mn, 0, -1):
                    c[b, k] = (dz_prev * c[b, k] - k * c[b, k - 1]) / d
                c[b, 0] = dz_prev * c[b, 0] / d
            prod_prev = prod
        out[i, j0:j0 + support] = c[:, order]
    return out


def barycentric(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Resampling matrix from nodes x to points y with weights
    (1/2, -1, 1, ..., -(-1)^N/2)."""
    n = x.size
    w = np.where(np.arange(n) % 2 == 1, -1.0, 1.0)
    w[0] = 0.5
    w[-1] = -0.5 * (-1) ** n
    d = y[:, None] - x[None, :]
    hit = d == 0
    with np.errstate(divide="ignore", invalid="ignore"):
        q = w[None, :] / d
        P = q / q.sum(axis=1, keepdims=True)
    P[hit] = 1.0
    return P


class Resolution:
    """Matrices of one fiber resolution N, packed as the device expects."""

    def __init__(self, n: int, n_fd: int = N_FD):
        if n < 6:
            raise ValueError("a fiber needs at least 6 points")
        self.n = n
        a = np.linspace(-1.0, 1.0, n)
        self.alpha = a
        self.D0 = [fd_weights(a, k, n_fd + k) for k in (1, 2, 3, 4)]
        roots = 2.0 * (0.5 + np.arange(n - 4)) / (n - 4) - 1.0
        tension = 2.0 * (0.5 + np.arange(n - 2)) / (n - 2) - 1.0
        self.PX = barycentric(a, roots)
        self.PT = barycentric(a, tension)
        w = np.full(n, 2.0 / (n - 1))
        w[0] = w[-1] = 1.0 / (n - 1)
        self.w0 = w

    def packed(self) -> np.ndarray:
        return np.concatenate([d.ravel() for d in self.D0] + [self.PX.ravel(), self.PT.ravel(), self.w0])

    def upsampling(self, rate: int = 2) -> np.ndarray:
        """[P_up (rate*N x N), w_up (rate*N)]: barycentric resampling onto
        rate*N equispaced nodes and their unit-length trapezoid weights
        (fiber3d's P_kerUp and weights_0_up, tstep/fiber_matrices.py:84-92)."""
        m = rate * self.n
        P = barycentric(self.alpha, np.linspace(-1.0, 1.0, m))
        w = np.full(m, 2.0 / (m - 1))
        w[0] = w[-1] = 1.0 / (m - 1)
        return np.concatenate([P.ravel(), w])


BC_CODES = {"force": 0, "torque": 1, "velocity": 2, "angular_velocity": 3}


class FiberSet:
    """Device arrays describing fibers of (possibly) different resolutions.

    ``positions``: list of (N_k, 3) arrays; ``lengths``: per fiber; ``bc``:
    per fiber 4 names (start translation, start rotation, end translation,
    end rotation), default free ends (force, torque, force, torque).
    """

    _res_cache: dict[int, Resolution] = {}

    def __init__(self, positions, lengths, bc=None, device=None, n_fd: int = N_FD):
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        dev = self.device
        self.npts = np.array([int(np.asarray(p).shape[0]) for p in positions], dtype=np.int64)
        self.nfib = len(positions)
        self.n_fd = n_fd
        self.pt_off_h = np.concatenate([[0], np.cumsum(self.npts)]).astype(np.int64)
        self.total = int(self.pt_off_h[-1])
        sizes = 4 * self.npts
        self.mat_off_h = np.concatenate([[0], np.cumsum(sizes * sizes)[:-1]]).astype(np.int64) \
            if self.nfib else np.zeros(0, np.int64)
        self.mat_total = int((sizes * sizes).sum())
        res_ids = sorted(set(self.npts.tolist()))
        blocks, offs, o = [], {}, 0
        for n in res_ids:
            r = self._res_cache.get(n)
            if r is None:
                r = Resolution(n, n_fd)
                self._res_cache[n] = r
            p = r.packed()
            offs[n] = o
            blocks.append(p)
            o += p.size
        self.resolutions = {n: self._res_cache[n] for n in res_ids}
        res_off = np.array([offs[n] for n in self.npts], dtype=np.int64)
        if bc is None:
            bc = [("force", "torque", "force", "torque")] * self.nfib
        bc_codes = np.array([[BC_CODES[b] for b in row] for row in bc], dtype=np.int32).reshape(-1)
        pt_fib = np.repeat(np.arange(self.nfib, dtype=np.int32), self.npts)
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
        self.n = t(self.npts.astype(np.int32), torch.int32)
        self.pt_off = t(self.pt_off_h, torch.int64)
        self.mat_off = t(self.mat_off_h, torch.int64)
        self.res_off = t(res_off, torch.int64)
        self.length = t(np.asarray(lengths, dtype=np.float64), torch.float64)
        self.bc = t(bc_codes, torch.int32)
        self.pt_fib = t(pt_fib, torch.int32)
        self.mats = t(np.concatenate(blocks) if blocks else np.zeros(1), torch.float64)
        self.max_n = int(self.npts.max()) if self.nfib else 0
        self._up = {}
        self.c = _lib.FiberSetC(self.nfib, _lib.ptr(self.n), _lib.ptr(self.pt_off), _lib.ptr(self.mat_off),
                                _lib.ptr(self.res_off), _lib.ptr(self.length), _lib.ptr(self.bc),
                                _lib.ptr(self.pt_fib), _lib.ptr(self.mats), n_fd + 3)

    def upsampling(self, rate: int = 2):
        """(up_mats, up_off) on the device: every resolution's
        Resolution.upsampling(rate) back to back, and each fiber's offset."""
        if rate not in self._up:
            blocks, offs, o = [], {}, 0
            for n, r in self.resolutions.items():
                p = r.upsampling(rate)
                offs[n] = o
                blocks.append(p)
                o += p.size
            up = torch.as_tensor(np.concatenate(blocks) if blocks else np.zeros(1), dtype=torch.float64,
                                 device=self.device)
            off = torch.as_tensor(np.array([offs[n] for n in self.npts], dtype=np.int64), device=self.device)
            self._up[rate] = (up, off)
        return self._up[rate]
