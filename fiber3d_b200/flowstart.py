"""GMRES warm start from a per-fiber network on geometry and background
flow: the fiber's 32 x 3 positions and the 32 x 3 background velocity at
them (the Oseen flow of the other fibers' forces, the double layers of the
bodies and the periphery, and the flow of the external forces) in; its 32
tensions and 32 x 3 force densities out.  The prediction becomes a guess for
the fiber unknowns of the coming step through the slender-body local
mobility of fiber3d (fiber.self_mobility, fiber/fiber.py:964-993):

    X^{n+1} = X^n + dt (M(X^n) f + u_bg),
    M f = c0 (f + x_s (x_s . f)) + c1 (f - x_s (x_s . f)),

c0 = -ln(e eps^2)/(8 pi eta), c1 = 2/(8 pi eta) (fiber.py:83-84), x_s the
unit tangent; the tensions are taken as predicted.  Periphery and body
unknowns take the quadratic extrapolation of the last solutions.

Training pairs come from the plain solver's own steps: the inputs of step
n+1 are the positions X^n and the background velocity of step n's solution
at step n's geometry; the targets are step n+1's tensions and force
densities f = F(X^n) x^{n+1} (the force operator of the geometry the step is
solved on).  The network is the library's FiberMLP (BF16 tensor-core GEMMs
with FP32 accumulation, its own backward pass and Adam) with 192 inputs.

fiber3d starts from zero (tstep.py:1209); GMRES still runs to the same
residual after this guess, so the answer does not depend on it.

The same guess built from the TRUE force densities and background velocity
of the step (``oracle_guess``) bounds what any network of this form can
reach: it measures how well the local-mobility map itself predicts X^{n+1}.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .warmstart import FiberMLP, NPTS, extrapolate, fiber_blocks, learnable

FLOW_LAYERS = (192, 256, 256, 256, 128)


def background_velocity(system, sol: torch.Tensor, precision: str = "fp32c") -> torch.Tensor:
    """(nfib, NPTS, 3) velocity at the fiber points from everything but the
    fiber itself, for solution `sol` at the system's current geometry: the
    pair sums of one matvec (other fibers' Oseen flow, body and periphery
    double layers) plus the explicit flow of the external forces."""
    tmp = torch.empty_like(sol)
    system.matvec(sol, tmp, precision=precision)
    v = system.v.view(-1, 3)[:system.nF] + system.flow_ext.view(-1, 3)
    return v.view(system.fs.nfib, NPTS, 3).clone()


def force_density(system, sol: torch.Tensor) -> torch.Tensor:
    """(nfib, NPTS, 3) force densities F(X) x of `sol` at the current geometry
    (fiber.force_operator, fiber/fiber.py:1399-1432)."""
    f = torch.empty((system.nF, 3), dtype=torch.float64, device=sol.device)
    _lib.call("f3d_fiber_forces", ctypes.byref(system.fs.c), system.p.E, _lib.ptr(system.geo),
              _lib.ptr(sol[system.o_fib:]), _lib.ptr(f), system.nF, 0, _lib.stream_handle(sol.device))
    return f.view(system.fs.nfib, NPTS, 3)


def positions(system, x: torch.Tensor) -> torch.Tensor:
    """(nfib, NPTS, 3) fiber positions held in the unknowns x."""
    return fiber_blocks(system, x)[:, :3].transpose(1, 2)


def tensions(system, x: torch.Tensor) -> torch.Tensor:
    return fiber_blocks(system, x)[:, 3]


def features(X: torch.Tensor, U: torch.Tensor) -> torch.Tensor:
    """(nfib, 192): positions about the fiber's centroid, background velocity."""
    Xc = X - X.mean(dim=1, keepdim=True)
    return torch.cat([Xc.flatten(1), U.flatten(1)], dim=1).float().contiguous()


def targets(T: torch.Tensor, f: torch.Tensor) -> torch.Tensor:
    """(nfib, 128): tensions, then force densities."""
    return torch.cat([T, f.flatten(1)], dim=1).float().contiguous()


class _Tangent:
    """Unit tangents x_s = (2/L) D1 X of equispaced fibers of NPTS points
    (fiber3d's finite-difference D1, as the device uses it)."""

    def __init__(self, system):
        res = system.fs.resolutions[NPTS]
        self.D1 = torch.as_tensor(res.D0[0], dtype=torch.float64, device=system.device)
        self.scale = (2.0 / system.fs.length).view(-1, 1, 1)

    def __call__(self, X: torch.Tensor) -> torch.Tensor:
        return torch.matmul(self.D1, X) * self.scale


def map_to_guess(system, x_base: torch.Tensor, X: torch.Tensor, U: torch.Tensor, T: torch.Tensor,
                 f: torch.Tensor, tangent: _Tangent) -> torch.Tensor:
    """x_base with its fiber unknowns replaced by X + dt (M(X) f + U) and T."""
    xs = tangent(X)
    xf = (xs * f).sum(dim=2, keepdim=True)
    c0, c1 = system.c0, system.c1
    Mf = c0 * (f + xs * xf) + c1 * (f - xs * xf)
    Xn = X + system.p.dt * (Mf + U)
    x0 = x_base.clone()
    B = fiber_blocks(system, x0)
    B[:, :3] = Xn.transpose(1, 2)
    B[:, 3] = T
    return x0


class FlowWarmStart:
    """FiberMLP on (positions, background velocity) -> (tensions, forces)."""

    def __init__(self, seed: int = 0, device=None):
        self.net = FiberMLP(seed=seed, device=device, layers=FLOW_LAYERS)
        self.device = self.net.device
        self._tangent = None

    def fit(self, X: torch.Tensor, Y: torch.Tensor, epochs=30, batch=1024, lr=1e-3, val_frac=0.1, seed=0):
        """Train on (features, targets); returns (loss history, relative
        error of the held-out predictions for tensions and forces)."""
        g = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(X.shape[0], generator=g).to(X.device)
        nval = max(1, int(val_frac * X.shape[0]))
        iv, it = perm[:nval], perm[nval:]
        self.net.set_normalisation(X[it], Y[it])
        hist = self.net.train(X[it].contiguous(), Y[it].contiguous(), epochs=epochs,
                              batch=min(batch, max(1, it.numel())), lr=lr, seed=seed)
        P = self.net.predict(X[iv].contiguous())
        Yv = Y[iv]
        rel = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        return hist, {"tension": rel(P[:, :NPTS], Yv[:, :NPTS]), "force": rel(P[:, NPTS:], Yv[:, NPTS:])}

    def guess(self, system, history, u_bg: torch.Tensor | None) -> torch.Tensor | None:
        """Extrapolated guess whose fiber unknowns come from the network (the
        extrapolation alone while there is no background velocity yet)."""
        x_q = extrapolate(history)
        if x_q is None or u_bg is None or not learnable(system):
            return x_q
        if self._tangent is None:
            self._tangent = _Tangent(system)
        X = positions(system, history[-1])
        Y = self.net.predict(features(X, u_bg)).double()
        T = Y[:, :NPTS]
        f = Y[:, NPTS:].view(-1, NPTS, 3)
        return map_to_guess(system, x_q, X, u_bg, T, f, self._tangent)


def oracle_guess(system, history, u_bg, T_true, f_true) -> torch.Tensor:
    """The same map with the step's true tensions and force densities (the
    best any network of this form can do; a diagnostic, not a method)."""
    x_q = extrapolate(history)
    X = positions(system, history[-1])
    return map_to_guess(system, x_q, X, u_bg, T_true, f_true, _Tangent(system))


def march(system, steps: int, guess: str = "extrapolate", net: FlowWarmStart | None = None, tol=1e-8,
          mixed=False, record=False, record_from: int = 2, restart=100, oracle_steps: int = 0):
    """Advance `system` `steps` steps with GMRES from `guess` ('zero',
    'extrapolate' or 'flow'); per step return iterations, solve time and the
    initial residual, and with `record` the network's training pairs.  The
    background velocity of each solution (one FP32C matvec at the solved
    geometry) is part of the timed step in 'flow' mode.  With oracle_steps,
    the first few steps from record_from on also report the initial
    residual of oracle_guess (an untimed extra solve each)."""
    history, stats, feats, targs = [], [], [], []
    u_bg = None
    can = learnable(system)
    for s in range(steps):
        X_in = positions(system, history[-1]) if (history and can) else None
        u_in = u_bg
        if guess == "zero":
            x0 = None
        elif guess == "flow" and net is not None:
            x0 = net.guess(system, history, u_bg)
        else:
            x0 = extrapolate(history)
        if s > 0:
            system.advance(history[-1], x0=x0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = system.solve(tol=tol, restart=restart, x0=x0, mixed=mixed)
        sol = res["x"]
        if guess == "flow" or record or oracle_steps:
            u_bg = background_velocity(system, sol) if can else None
        e1.record()
        e1.synchronize()
        st = {"iterations": res["iterations"], "ms": e0.elapsed_time(e1),
              "initial_rel_residual": res["history"][0]}
        if res["info"] != 0 or not bool(torch.isfinite(sol).all()):
            stats.append(st)
            break
        if can and s >= record_from and X_in is not None and u_in is not None:
            T_true = tensions(system, sol)
            f_true = force_density(system, sol).clone()
            if record:
                feats.append(features(X_in, u_in))
                targs.append(targets(T_true, f_true))
            if oracle_steps and s < record_from + oracle_steps:
                xo = oracle_guess(system, history, u_in, T_true, f_true)
                y = torch.empty_like(xo)
                system.matvec(xo, y)
                st["oracle_map_rel_residual"] = float(torch.linalg.vector_norm(system.rhs - y)
                                                      / torch.linalg.vector_norm(system.rhs))
        stats.append(st)
        history = (history + [sol])[-3:]
    if record:
        dev = system.device
        return (stats, torch.cat(feats) if feats else torch.zeros((0, FLOW_LAYERS[0]), device=dev),
                torch.cat(targs) if targs else torch.zeros((0, FLOW_LAYERS[-1]), device=dev))
    return stats
