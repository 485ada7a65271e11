"""Right-preconditioned restarted GMRES on the device, and mixed-precision
iterative refinement around it.

Replaces ``bpm_utilities/gmres.py:9-111`` (scipy.sparse.linalg.gmres on
A P^-1 y = b, then x = P^-1 y) as called at ``tstep/tstep.py:1209-1216``.

Arnoldi runs on the device: one step is ``z_k = P^-1 v_k``, ``w = A z_k``,
classical Gram-Schmidt applied twice (CGS2) against the basis, ``|w|`` and
``v_{k+1} = w / |w|`` — every vector stays in HBM and every reduction has a
fixed order.  The z_k are kept (as flexible GMRES keeps them), so the update
is ``x += Z y`` and a cycle applies the preconditioner once per iteration,
not once more for ``x += P^-1 (V y)``; the iterates are the same.  That step can be captured once as a CUDA graph (the basis
count lives in device memory) and replayed for every k.  The Hessenberg
column (k+2 numbers) comes back to the host each step, where the Givens
rotations and the residual estimate are updated in FP64, as scipy does.
Convergence uses the residual estimate, and is confirmed by a true residual
``|b - A x| / |b|`` before returning (a restart follows otherwise).

Mixed precision (``solve_system(mixed=True)``): outer iterative refinement
on residuals ``r = b - A x``; each correction is an inner GMRES solve whose
matvec uses the compensated-FP32 (FP32C) pair kernels and whose
preconditioner reads FP32/FP16 copies of the block inverses (Arnoldi and
Givens stay FP64).  The outer residual is itself evaluated with the FP32C
pair sums when that cannot change the convergence test: every other part of
the matvec is FP64, and the pair sums v carry a relative error below
``FP32C_PAIR_REL_ERR``; they enter the matvec through a linear map of norm
at most G (``system.v_gain``: 1 on periphery and body rows, the norm of the
projected value-and-derivative rows on fibers), so the residual is off by at
most ``e = FP32C_PAIR_REL_ERR * G * |v| / |b|`` (relative).  The solve stops when
``|r| / |b| + e <= tol``, which bounds the FP64 residual by tol as well;
while ``e <= tol / 2`` the residual stays FP32C, otherwise it is recomputed
in FP64 (and stays FP64 for the rest of the solve and for later solves of
the same system, whose |v| / |b| changes little from step to step).  When update(x0) already
summed the Oseen flow of the guess in FP64 (the dual pass), the first
residual adds only the stresslet flow in FP32C, and e counts only that part
of v.  After an inner solve
the new residual is bounded without a matvec: by the inner GMRES estimate
``|r - A32 d|`` plus e (0 for an FP64 residual) plus
``FP32C_PAIR_REL_ERR * G * sum_j |y_j| |v(z_j)|``
(the FP32C error of the matvecs that built d = sum_j y_j z_j); when that sum
is below tol the solve ends there, else the residual is computed.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from . import _lib

# Bound on |v_fp32c - v_fp64| / |v_fp64| (2-norms) of the FP32C pair sums:
# about 4x the largest value measured on the solver's own matvecs (4.3e-7);
# the tests hold the pair sums to a quarter of it.
FP32C_PAIR_REL_ERR = 2e-6


class DeviceGMRES:
    """GMRES workspace for systems of size n with restart length m."""

    def __init__(self, n: int, restart: int = 100, device=None):
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.n, self.m = n, int(restart)
        if self.m + 1 > 256:
            raise ValueError("restart must be <= 255")
        f = lambda *s: torch.zeros(*s, dtype=torch.float64, device=dev)
        self.V = f(self.m + 1, n)
        self.Z = f(self.m, n)  # z_k = P^-1 v_k
        self.cur = f(n)      # current basis vector (input of the Arnoldi step)
        self.z = f(n)
        self.w = f(n)
        self.h1 = f(self.m + 2)
        self.h2 = f(self.m + 2)
        self.beta = f(1)
        self.k = torch.zeros(1, dtype=torch.int32, device=dev)
        nb = ctypes.c_size_t(0)
        _lib.call("f3d_krylov_workspace_bytes", n, self.m + 1, ctypes.byref(nb))
        self.ws = torch.zeros(max(nb.value, 4096), dtype=torch.uint8, device=dev)
        self.wsn = torch.zeros(4096, dtype=torch.uint8, device=dev)
        self.aux = f(self.m + 2)      # aux[j + 1] = |aux vector| after the matvec of step j
        self.auxbeta = f(1)
        self.h_host = torch.zeros(3 * (self.m + 2) + 1, dtype=torch.float64).pin_memory()
        # y of the update x += Z y goes up through a pinned buffer
        self.y_host = torch.zeros(self.m, dtype=torch.float64).pin_memory()
        self.y_dev = f(self.m)
        self.y_done = torch.cuda.Event()
        # norms read back together (|b|, a residual's, the split residual's FP32C flow)
        self.pair = f(3)
        self.pair_host = torch.zeros(3, dtype=torch.float64).pin_memory()
        self.graph = {}
        self.last_aux_sum = 0.0

    # ------------------------------------------------------------ kernels --
    def _norm(self, w, beta):
        """beta = |w|_2 over all of w (any length, contiguous float64)."""
        if w.dtype != torch.float64 or not w.is_contiguous():
            raise ValueError("norm of a contiguous float64 vector")
        st = _lib.stream_handle(self.device)
        _lib.call("f3d_krylov_norm", _lib.ptr(w), w.numel(), None, None, _lib.ptr(beta), _lib.ptr(self.wsn),
                  self.wsn.numel(), st)

    def _arnoldi(self, matvec, pc, aux=None):
        """One Arnoldi step on the current stream (graph-capturable).  With
        `aux` (a device vector the matvec writes, e.g. its pair sums) its
        norm after the matvec is recorded for the step."""
        st = _lib.stream_handle(self.device)
        n, ldv = self.n, self.n
        pc(self.cur, self.z)
        _lib.call("f3d_krylov_store", _lib.ptr(self.z), _lib.ptr(self.k), -1, _lib.ptr(self.Z), n, n, st)
        matvec(self.z, self.w)
        if aux is not None:
            _lib.call("f3d_krylov_norm", _lib.ptr(aux), aux.numel(), _lib.ptr(self.k), _lib.ptr(self.aux),
                      _lib.ptr(self.auxbeta), _lib.ptr(self.wsn), self.wsn.numel(), st)
        for h in (self.h1, self.h2):
            _lib.call("f3d_krylov_multidot", _lib.ptr(self.V), ldv, _lib.ptr(self.w), _lib.ptr(self.k),
                      self.m + 1, _lib.ptr(h), n, 0, _lib.ptr(self.ws), self.ws.numel(), st)
            _lib.call("f3d_krylov_multiaxpy", _lib.ptr(self.V), ldv, _lib.ptr(h), _lib.ptr(self.k),
                      _lib.ptr(self.w), n, st)
        _lib.call("f3d_krylov_norm", _lib.ptr(self.w), n, _lib.ptr(self.k), _lib.ptr(self.h1),
                  _lib.ptr(self.beta), _lib.ptr(self.wsn), self.wsn.numel(), st)
        _lib.call("f3d_krylov_scale_into", _lib.ptr(self.w), _lib.ptr(self.beta), _lib.ptr(self.k),
                  _lib.ptr(self.V), ldv, n, 1, _lib.ptr(self.cur), st)
        m2 = self.m + 2
        self.h_host[:m2].copy_(self.h1, non_blocking=True)
        self.h_host[m2:2 * m2].copy_(self.h2, non_blocking=True)
        if aux is not None:
            self.h_host[2 * m2:3 * m2].copy_(self.aux, non_blocking=True)

    def _step(self, matvec, pc, key, use_graph, aux=None):
        if not use_graph:
            self._arnoldi(matvec, pc, aux)
            return
        key = (key, aux is not None)
        g = self.graph.get(key)
        if g is None:
            # warm-up outside capture on a side stream (allocations, lazy init)
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                saved = (self.k.clone(), self.cur.clone(), self.V.clone(), self.Z.clone())
                self._arnoldi(matvec, pc, aux)
                self.k.copy_(saved[0]); self.cur.copy_(saved[1]); self.V.copy_(saved[2])
                self.Z.copy_(saved[3])
            torch.cuda.current_stream(self.device).wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._arnoldi(matvec, pc, aux)
            self.graph[key] = g
        self.graph[key].replay()

    def start_cycle(self, r, beta_dev):
        """V[0] = cur = r / |r| with |r| read from the device scalar beta_dev; k = 0."""
        self.k.zero_()
        _lib.call("f3d_krylov_scale_into", _lib.ptr(r), _lib.ptr(beta_dev), _lib.ptr(self.k),
                  _lib.ptr(self.V), self.n, self.n, 1, _lib.ptr(self.cur), _lib.stream_handle(self.device))

    def read_pair(self):
        """The first two norms in self.pair, on the host (one synchronisation)."""
        return self.read_norms()[:2]

    def read_norms(self):
        """The three norms in self.pair, on the host (one synchronisation)."""
        self.pair_host.copy_(self.pair)
        h = self.pair_host.tolist()
        return h[0], h[1], h[2]

    # ------------------------------------------------------------- solve ---
    def solve(self, matvec, pc, b: torch.Tensor, x0: torch.Tensor | None = None, rtol=1e-8,
              maxiter=200, use_graph=True, key="default", bnorm=None, verify=True, aux=None,
              r0: torch.Tensor | None = None, rnorm0: float | None = None, first_step_done: bool = False):
        """Solve A x = b with right preconditioner pc = P^-1.

        Returns (x, info, iterations, history of relative residual estimates).
        info = 0 on convergence, else the iteration count reached.  With
        verify=False the first cycle whose residual estimate meets rtol
        returns without recomputing the true residual (the caller judges the
        result itself, as the mixed-precision refinement does).  With `aux`,
        ``self.last_aux_sum`` is set to sum_j |y_j| |aux after A z_j| over the
        correction x - x0 = sum_j y_j z_j (an error bound's ingredient).
        `r0` (optional) is b - A x0, already computed by the caller, and
        `rnorm0` (optional) the norm of the first residual (b itself when
        x0 is None) when the caller knows it.  With `first_step_done` the
        caller has already run start_cycle() on that residual and the first
        Arnoldi step (same matvec, pc, key and aux), and passes rnorm0.
        """
        self.last_aux_sum = 0.0
        n, m = self.n, self.m
        if b.numel() != n or (x0 is not None and x0.numel() != n):
            raise ValueError(f"right-hand side and guess must have {n} entries")
        dev = self.device
        # x starts as zero implicitly (the first update overwrites it) when x0 is None
        x_zero = x0 is None
        x = torch.empty(n, dtype=torch.float64, device=dev) if x_zero else x0.clone()
        r = torch.empty(n, dtype=torch.float64, device=dev)
        tmp = torch.empty(n, dtype=torch.float64, device=dev)
        if bnorm is None:
            self._norm(b, self.beta)
            bnorm = float(self.beta.item())
        if bnorm == 0.0:
            return torch.zeros_like(b), 0, 0, [0.0]
        its, hist = 0, []
        while True:
            # r = b - A x
            if x_zero:
                res = b
            elif r0 is not None and its == 0:
                res = r0
            else:
                matvec(x, tmp)
                torch.sub(b, tmp, out=r)
                res = r
            if its == 0 and rnorm0 is not None:
                rnorm = float(rnorm0)
                if not first_step_done:
                    self.beta.fill_(rnorm)
            else:
                self._norm(res, self.beta)
                rnorm = float(self.beta.item())
            hist.append(rnorm / bnorm)
            if rnorm <= rtol * bnorm or its >= maxiter:
                if x_zero:
                    x.zero_()
                return x, (0 if rnorm <= rtol * bnorm else its), its, hist
            # V[0] = r / |r|, cur = V[0], k = 1
            prestarted = first_step_done and its == 0
            if not prestarted:
                self.start_cycle(res, self.beta)
            # Givens rotations and the least-squares solve on the host, in
            # Python floats (a handful of scalar operations per step)
            m2 = m + 2
            hh = self.h_host.numpy()
            Hc = []            # Hc[k] = column k of the triangular factor (rows 0..k)
            cs, sn = [], []
            gv = [rnorm]
            j_done = 0
            for j in range(m):
                if not (prestarted and j == 0):
                    self._step(matvec, pc, key, use_graph, aux)
                torch.cuda.current_stream(dev).synchronize()
                col = (hh[:j + 1] + hh[m2:m2 + j + 1]).tolist()
                sub = float(hh[j + 1])           # subdiagonal |w|
                col.append(sub)
                for i in range(j):
                    t = cs[i] * col[i] + sn[i] * col[i + 1]
                    col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1]
                    col[i] = t
                den = math.hypot(col[j], col[j + 1])
                if den == 0.0:
                    c_, s_ = 1.0, 0.0
                else:
                    c_, s_ = col[j] / den, col[j + 1] / den
                cs.append(c_)
                sn.append(s_)
                col[j] = den
                gv.append(-s_ * gv[j])
                gv[j] = c_ * gv[j]
                Hc.append(col[:j + 1])
                its += 1
                j_done = j + 1
                est = abs(gv[j + 1]) / bnorm
                hist.append(est)
                if est <= rtol or its >= maxiter or sub == 0.0:
                    break
            # y = H^-1 g ; x += Z y  (= P^-1 (V y))
            y = [0.0] * j_done
            for i in range(j_done - 1, -1, -1):
                acc = gv[i]
                for k in range(i + 1, j_done):
                    acc -= Hc[k][i] * y[k]
                y[i] = acc / Hc[i][i]
            if aux is not None:
                an = hh[2 * m2:2 * m2 + j_done + 1].tolist()
                self.last_aux_sum += sum(abs(y[i]) * an[i + 1] for i in range(j_done))
            self.y_done.synchronize()  # the previous upload out of y_host has run
            self.y_host.numpy()[:j_done] = y
            self.y_dev[:j_done].copy_(self.y_host[:j_done], non_blocking=True)
            self.y_done.record()
            _lib.call("f3d_krylov_combine", _lib.ptr(self.Z), n, _lib.ptr(self.y_dev), j_done, _lib.ptr(x), n,
                      0 if x_zero else 1, _lib.stream_handle(dev))
            x_zero = False
            if not verify and hist[-1] <= rtol:
                return x, 0, its, hist


def solve_system(system, tol=1e-8, restart=100, maxiter=200, x0=None, mixed=False,
                 inner_tol=1e-5, max_refine=10, use_graph=True):
    """Solve system.matvec x = system.rhs to relative residual `tol`.

    Returns a dict with the solution and statistics.
    """
    dev = system.device
    n = system.size
    g = getattr(system, "_gmres", None)
    if g is None or g.n != n or g.m != restart:
        g = DeviceGMRES(n, restart, dev)
        system._gmres = g
    b = system.rhs
    t0 = time.perf_counter()
    # the Oseen flow of x0's fiber forces may already be summed (update(x0))
    pending = x0 is not None and hasattr(system, "pending_oseen") and system.pending_oseen(x0)
    if hasattr(system, "_pending_x0"):
        system._pending_x0 = None
    if not mixed:
        r0 = None
        if pending:
            r0 = torch.empty_like(b)
            system.matvec(x0, r0, "fp64", oseen_done=True)
            torch.sub(b, r0, out=r0)
        x, info, its, hist = g.solve(lambda a, o: system.matvec(a, o, "fp64"),
                                     lambda a, o: system.pc(a, o, "fp64"), b, x0=x0, rtol=tol,
                                     maxiter=maxiter, use_graph=use_graph, key="fp64", r0=r0)
        return {"x": x, "info": info, "iterations": its, "history": hist, "refinements": 0,
                "seconds": time.perf_counter() - t0}
    # mixed: FP32C inner solves; outer residuals FP32C while the bound holds
    x = torch.zeros(n, dtype=torch.float64, device=dev) if x0 is None else x0.clone()
    r = torch.empty(n, dtype=torch.float64, device=dev)
    tmp = torch.empty(n, dtype=torch.float64, device=dev)
    # |b| stays on the device until the first residual's norm is read with it
    g._norm(b, g.pair[0:1])
    bnorm = None

    def norm_rel(w):
        """|w| / |b| (reading |b| too on the first call)."""
        nonlocal bnorm
        if bnorm is None:
            g._norm(w, g.pair[1:2])
            bnorm, wn = g.read_pair()
        else:
            g._norm(w, g.beta)
            wn = float(g.beta.item())
        return wn / bnorm if bnorm > 0.0 else 0.0, wn

    mv32 = lambda a, o: system.matvec(a, o, "fp32c")
    pc32 = lambda a, o: system.pc(a, o, "fp32c")
    total_its, hist, ref = 0, [], 0
    info = 0
    # outer residuals start FP32C unless an earlier solve of this system found
    # their bound too loose (the ratio |v| / |b| changes little between steps)
    outer = "fp64" if getattr(system, "_outer_fp64", False) else "fp32c"
    fp64_residuals = 0
    # |A32 x - A64 x| <= eps_v |v(x)|: the pair-sum error times the gain of
    # the map from the pair sums to the matvec's rows
    eps_v = FP32C_PAIR_REL_ERR * getattr(system, "v_gain", 1.0)
    known = None  # a bound on the FP64 relative residual of x, when one is at hand
    first_bound = None
    while True:
        bound = 0.0  # bound on |r_computed - r_fp64| / |b|
        split_pending = False
        if known is not None:
            rel, bound = known
        elif x0 is None and ref == 0:
            r.copy_(b)
        elif pending and ref == 0 and not getattr(system, "_split_fp64", False):
            # the Oseen flow of x0 is FP64 already (update(x0)).  The
            # stresslet part in FP32C is bounded by its own flow,
            # eps_v |v - v_oseen|; when that bound is too loose, the fiber
            # targets' stresslet flow is FP64 and only the body and periphery
            # targets' is FP32C: their rows take it with gain 1, so the
            # bound is FP32C_PAIR_REL_ERR |(v - v_oseen) on those targets|.
            if not getattr(system, "_stress_fp64", False):
                system.matvec(x, tmp, "fp32c", oseen_done=True)
                bound = eps_v * norm_rel(system.v - system.v2)[0]
                if bound > 0.5 * tol:
                    system._stress_fp64 = True
            if getattr(system, "_stress_fp64", False):
                system.matvec(x, tmp, "split", oseen_done=True)
                nf3 = 3 * getattr(system, "nF", 0)
                # the norm stays on the device; it is read together with |r|
                # below, and the bound decided there
                g._norm((system.v - system.v2)[nf3:], g.pair[2:3])
                split_pending = True
            torch.sub(b, tmp, out=r)
        else:
            system.matvec(x, tmp, outer, oseen_done=pending and ref == 0)
            if outer == "fp32c":
                bound = eps_v * norm_rel(system.v)[0]
                if bound > 0.5 * tol:
                    outer, bound = "fp64", 0.0
                    system._outer_fp64 = True
                    system.matvec(x, tmp, outer, oseen_done=pending and ref == 0)
            if outer == "fp64":
                fp64_residuals += 1
            torch.sub(b, tmp, out=r)
        spec = False
        if known is None:
            # when the last solve of this system needed inner iterations, the
            # first one is launched before the host reads |r|, which it takes
            # from the device, so that read does not leave the GPU idle
            spec = ref == 0 and getattr(system, "_spec_first", False)
            if spec or split_pending:
                # |r| goes to pair[1], which the Arnoldi step does not write
                # (it overwrites beta with the next basis vector's norm); |b|,
                # |r| and the split residual's FP32C flow norm come back in
                # one read, after the speculative step has been launched
                g._norm(r, g.pair[1:2])
                if spec:
                    g.start_cycle(r, g.pair[1:2])
                    g._step(mv32, pc32, "fp32c", use_graph, aux=system.v)
                bn, rnorm, vrest = g.read_norms()
                if bnorm is None:
                    bnorm = bn
                rel = rnorm / bnorm if bnorm > 0.0 else 0.0
                if split_pending:
                    bound = FP32C_PAIR_REL_ERR * vrest / bnorm if bnorm > 0.0 else 0.0
                    if bound > 0.5 * tol:
                        # too loose: the residual in FP64; a speculative step
                        # taken on the split residual is dropped
                        bound, spec = 0.0, False
                        system._split_fp64 = True
                        system.matvec(x, tmp, "fp64", oseen_done=True)
                        fp64_residuals += 1
                        torch.sub(b, tmp, out=r)
                        rel, rnorm = norm_rel(r)
            else:
                rel, rnorm = norm_rel(r)
        known = None
        if first_bound is None:
            first_bound = bound
        hist.append(rel + bound)
        if rel + bound <= tol:  # the FP64 residual is <= tol as well
            break
        if ref >= max_refine or total_its >= maxiter:
            info = total_its
            break
        # inner tolerance relative to |r|: never ask beyond what is needed
        inner = max(inner_tol, 0.7 * (tol - bound) / rel)
        d, _, its, ihist = g.solve(mv32, pc32, r, rtol=inner,
                                   maxiter=maxiter - total_its, use_graph=use_graph, key="fp32c",
                                   verify=False, aux=system.v, bnorm=rnorm, rnorm0=rnorm,
                                   first_step_done=spec)
        total_its += its
        x += d
        ref += 1
        # |b - A64 (x + d)| <= |r - A32 d| + |r - r64| + |(A32 - A64) d|: the
        # inner GMRES estimate, the bound of the residual r (0 when FP64),
        # and the FP32C error of the matvecs that built d = sum_j y_j z_j
        # (linear in y); no further matvec when this settles convergence.
        est = ihist[-1] * rel
        bd = bound + eps_v * g.last_aux_sum / bnorm
        if est + bd <= tol:  # the same sum as the convergence test above
            known = (est, bd)
    system._spec_first = x0 is not None and hist[0] > 2.0 * tol
    return {"x": x, "info": info, "iterations": total_its, "history": hist, "refinements": ref,
            "outer_residuals": outer, "fp64_residuals": fp64_residuals, "first_residual_bound": first_bound,
            "seconds": time.perf_counter() - t0}
