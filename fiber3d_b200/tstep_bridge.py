"""Solver-level drop-in for fiber3d's hydrodynamic time step.

fiber3d builds its linear system inside ``tstep.time_step_hydro``
(python/tstep/tstep.py:628-1458) as two closures — the matvec
``A_body_fiber_hyd`` (:1003-1178) and the preconditioner ``P_inv``
(:950-994) — and solves it with ``bpm_utilities.gmres.gmres``
(:1209-1216).  :func:`install` replaces that ``gmres`` function with one that
builds the same system on the GPU from the time stepper's own state (fibers,
bodies, periphery, viscosity, time step), takes fiber3d's right-hand side
``b`` as given (so every explicit force fiber3d added is kept), and solves to
the same relative tolerance.  It returns ``(solution, info)`` in fiber3d's
unknown layout, so the rest of ``time_step_hydro`` runs unchanged.

The periphery preconditioner is built once per periphery and reused.

fiber3d starts GMRES from zero (tstep.py:1209).  With
``warm_start="extrapolate"`` the solver keeps the last three solutions of
its own calls and starts from their quadratic extrapolation
(``warmstart.extrapolate``); with ``warm_start="learned"`` and a trained
``warmstart.LearnedWarmStart`` as ``model``, from that extrapolation
corrected per fiber by the network once four solutions are known.  GMRES
still runs to fiber3d's tolerance, so a history that does not match the
step (a rejected step, a changed system) costs iterations, never accuracy.
The history is dropped whenever the system size changes.
"""
from __future__ import annotations

import numpy as np
import torch

from .hydro import Body, HydroSystem, Problem, Shell, ShellOperator


def _rotation(orientation) -> np.ndarray:
    return np.asarray(orientation.rotation_matrix(), dtype=np.float64)


def problem_from_tstep(ts) -> Problem:
    """Geometry and parameters of a fiber3d ``tstep`` object as a Problem
    (free fibers; fiber3d's fiber defaults epsilon / penalty_param)."""
    fibers = [np.asarray(f.x, dtype=np.float64) for f in ts.fibers]
    lengths = [float(f.length) for f in ts.fibers]
    f0 = ts.fibers[0] if ts.fibers else None
    bodies = [Body(np.asarray(b.location, dtype=np.float64), _rotation(b.orientation),
                   np.asarray(b.reference_configuration), np.asarray(b.reference_normals),
                   np.asarray(b.quadrature_weights)) for b in ts.bodies]
    shell = None
    if getattr(ts, "shell", None) is not None:
        shell = Shell(np.asarray(ts.trg_shell_surf).reshape(-1, 3),
                      np.asarray(ts.normals_shell).reshape(-1, 3),
                      np.asarray(ts.shell.quadrature_weights))
    return Problem(fibers, lengths, float(f0.E) if f0 else 1.0, float(ts.dt), float(ts.eta), bodies,
                   shell, None, epsilon=float(f0.epsilon) if f0 else 1e-3,
                   penalty=float(f0.penalty_param) if f0 else 500.0)


class GpuGmres:
    """Callable with the signature fiber3d uses for ``gmres.gmres``."""

    def __init__(self, ts, mixed: bool = False, restart: int = 100, warm_start: str | None = None,
                 model=None, shell_pc: str = "dense"):
        if warm_start not in (None, "extrapolate", "learned"):
            raise ValueError("warm_start must be None, 'extrapolate' or 'learned'")
        if warm_start == "learned" and model is None:
            raise ValueError("warm_start='learned' needs a trained warmstart.LearnedWarmStart as model")
        self.ts = ts
        self.model = model
        self.mixed = mixed
        self.restart = restart
        self.warm_start = warm_start
        self.shell_pc = shell_pc
        self._history = []
        self._shell = None
        self.last = None

    def __call__(self, A, b, x0=None, tol=1e-5, atol=0, restart=None, maxiter=None, M=None,
                 callback=None, **kw):
        P = problem_from_tstep(self.ts)
        if P.shell is not None and self._shell is None:
            self._shell = ShellOperator(P.shell, P.eta, P.reg, P.eps_dist, pc=self.shell_pc)
        sysd = HydroSystem(P, shell_op=self._shell)
        if sysd.size != np.size(b):
            raise ValueError(f"system size {sysd.size} != len(b) {np.size(b)}")
        sysd.rhs.copy_(torch.as_tensor(np.asarray(b, dtype=np.float64)))
        x0 = None
        if self.warm_start is not None:
            if self._history and self._history[-1].numel() != sysd.size:
                self._history = []
            if self._history:
                from .warmstart import extrapolate, learned_guess
                x0 = (learned_guess(sysd, self._history, self.model) if self.warm_start == "learned"
                      else extrapolate(self._history))
        res = sysd.solve(tol=tol, restart=min(restart or self.restart, 255), maxiter=maxiter or 200,
                         mixed=self.mixed, x0=x0)
        if self.warm_start is not None:
            from .warmstart import HISTORY
            self._history = (self._history + [res["x"]])[-HISTORY:]
        if callback is not None:
            for h in res["history"][1:]:
                callback(h)
        self.last = res
        return res["x"].cpu().numpy(), int(res["info"])


def install(ts, mixed: bool = False, warm_start: str | None = None, model=None, shell_pc: str = "dense"):
    """Route fiber3d's GMRES call through the GPU solver for time stepper `ts`."""
    import importlib
    gm = importlib.import_module("bpm_utilities.gmres")
    solver = GpuGmres(ts, mixed=mixed, warm_start=warm_start, model=model, shell_pc=shell_pc)
    gm.gmres = solver
    return solver
