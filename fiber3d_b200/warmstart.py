"""Learned GMRES warm start: a per-fiber network trained on the plain
solver's own time steps.

Network (per fiber of 32 points): input 192 = 32x3 positions (centred on the
fiber's mean point) + 32x3 background velocity; 3 hidden layers of 256 with
ReLU; output 128 = 32 tensions + 32x3 force densities.  Weights are kept in
FP32 (master copy, Adam) and rounded to BF16 when staged for the tensor
cores; every product runs in ``f3d_gemm_bf16`` (tcgen05, FP32 accumulation
in tensor memory), the backward pass included.

Warm start for step n+1 from the prediction (T^, f^) (fiber3d's first-order
scheme, tstep.py:628-1458):
  fiber positions  X^ = X^n + dt (u_bg + M f^),   M f = c0 (f + xs (xs.f)) + c1 (f - xs (xs.f))
                   (the local slender-body mobility, fiber.self_mobility, fiber.py:964-993)
  tensions         T^
  periphery / bodies: the previous step's values.
Plain GMRES then runs from this guess to the same relative residual, so the
converged answer does not depend on the network; what it changes is the
number of iterations.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

LAYERS = (192, 256, 256, 256, 128)


def _gemm(A, a_rs, a_cs, B, b_rs, b_cs, C, ldc, M, N, K, bias=None, relu=False, mask=None, ldm=0,
          pre=None, alpha=1.0, accumulate=False):
    _lib.call("f3d_gemm_bf16", _lib.ptr(A), a_rs, a_cs, _lib.ptr(B), b_rs, b_cs, _lib.ptr(C), ldc, M, N, K,
              _lib.ptr(bias), int(relu), _lib.ptr(mask), ldm, _lib.ptr(pre), float(alpha), int(accumulate),
              _lib.stream_handle(C.device))


def gemm(A: torch.Tensor, B: torch.Tensor, *, transpose_a=False, transpose_b=True, bias=None,
         relu=False, mask=None, pre=None) -> torch.Tensor:
    """C = op(A) op(B) on the tensor cores (BF16 operands, FP32 result).

    With the defaults C = A @ B^T (A: M x K, B: N x K)."""
    A = A.contiguous()
    B = B.contiguous()
    if transpose_a:
        K, M = A.shape
        a_rs, a_cs = 1, M
    else:
        M, K = A.shape
        a_rs, a_cs = K, 1
    if transpose_b:
        N, K2 = B.shape
        b_rs, b_cs = K2, 1
    else:
        K2, N = B.shape
        b_rs, b_cs = 1, N
    if K2 != K:
        raise ValueError("inner dimensions differ")
    C = torch.empty((M, N), dtype=torch.float32, device=A.device)
    _gemm(A, a_rs, a_cs, B, b_rs, b_cs, C, N, M, N, K, bias=bias, relu=relu, mask=mask,
          ldm=N if mask is not None else 0, pre=pre)
    return C


class FiberMLP:
    """The warm-start network with its own forward/backward/Adam kernels."""

    def __init__(self, seed: int = 0, device=None):
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []
        for k in range(len(LAYERS) - 1):
            fan_in, fan_out = LAYERS[k], LAYERS[k + 1]
            w = rng.normal(scale=np.sqrt(2.0 / fan_in), size=(fan_out, fan_in)).astype(np.float32)
            if k == len(LAYERS) - 2:
                w *= 0.1
            self.W.append(torch.as_tensor(w, device=dev))
            self.b.append(torch.zeros(fan_out, dtype=torch.float32, device=dev))
        self.params = self.W + self.b
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step = 0
        self.in_mean = torch.zeros(LAYERS[0], device=dev)
        self.in_std = torch.ones(LAYERS[0], device=dev)
        self.out_mean = torch.zeros(LAYERS[-1], device=dev)
        self.out_std = torch.ones(LAYERS[-1], device=dev)

    # ------------------------------------------------------------- passes --
    def forward(self, X: torch.Tensor, keep=False):
        """X: (B, 192) normalised inputs -> (B, 128) normalised outputs."""
        acts, pres = [X.contiguous()], []
        h = acts[0]
        L = len(self.W)
        for k in range(L):
            last = k == L - 1
            pre = torch.empty((h.shape[0], LAYERS[k + 1]), dtype=torch.float32, device=X.device) \
                if (keep and not last) else None
            h = gemm(h, self.W[k], bias=self.b[k], relu=not last, pre=pre)
            if keep:
                pres.append(pre)
                acts.append(h)
        return (h, acts, pres) if keep else h

    def grads(self, X: torch.Tensor, T: torch.Tensor):
        """Loss (mean squared error, normalised units) and parameter gradients."""
        Y, acts, pres = self.forward(X, keep=True)
        B = X.shape[0]
        D = torch.empty_like(Y)
        row = torch.empty(B, dtype=torch.float32, device=X.device)
        _lib.call("f3d_mse_grad", _lib.ptr(Y), _lib.ptr(T.contiguous()), _lib.ptr(D), _lib.ptr(row), B,
                  Y.shape[1], _lib.stream_handle(X.device))
        gW, gb = [None] * len(self.W), [None] * len(self.W)
        for k in range(len(self.W) - 1, -1, -1):
            Ain = acts[k]
            # dW = D^T Ain  (M = out, N = in, K = batch)
            gW[k] = gemm(D, Ain, transpose_a=True, transpose_b=False)
            gb[k] = torch.empty(self.b[k].shape, dtype=torch.float32, device=X.device)
            _lib.call("f3d_colsum", _lib.ptr(D), D.shape[1], B, D.shape[1], _lib.ptr(gb[k]), 0,
                      _lib.stream_handle(X.device))
            if k > 0:
                # dA = D W ; D_prev = dA * (pre_{k-1} > 0)
                D = gemm(D, self.W[k], transpose_b=False, mask=pres[k - 1])
        loss = row.sum() / (B * Y.shape[1])
        return loss, gW + gb

    def adam(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        st = _lib.stream_handle(self.device)
        for p, g, m, v in zip(self.params, grads, self.m, self.v):
            _lib.call("f3d_adam", _lib.ptr(p), _lib.ptr(g.contiguous()), _lib.ptr(m), _lib.ptr(v), p.numel(),
                      lr, b1, b2, eps, self.step, st)

    # ------------------------------------------------------------- data ----
    def set_normalisation(self, X: torch.Tensor, T: torch.Tensor):
        self.in_mean, self.in_std = X.mean(0), X.std(0) + 1e-6
        self.out_mean, self.out_std = T.mean(0), T.std(0) + 1e-6

    def train(self, X: torch.Tensor, T: torch.Tensor, epochs=30, batch=1024, lr=1e-3, seed=0):
        """Minibatch Adam on normalised data; returns the loss history."""
        Xn = ((X - self.in_mean) / self.in_std).float().contiguous()
        Tn = ((T - self.out_mean) / self.out_std).float().contiguous()
        g = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        n = Xn.shape[0]
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).to(Xn.device)
            tot = 0.0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                loss, gr = self.grads(Xn[idx].contiguous(), Tn[idx].contiguous())
                self.adam(gr, lr=lr)
                tot += float(loss)
            hist.append(tot / max(1, n // batch))
        return hist

    def predict(self, X: torch.Tensor) -> torch.Tensor:
        Xn = ((X - self.in_mean) / self.in_std).float().contiguous()
        return self.forward(Xn) * self.out_std + self.out_mean


# ---------------------------------------------------------------- features --
def fiber_features(x_fib: torch.Tensor, u_bg: torch.Tensor, npts: int = 32) -> torch.Tensor:
    """(nfib, 192): positions centred per fiber, and background velocity."""
    X = x_fib.view(-1, npts, 3)
    Xc = X - X.mean(1, keepdim=True)
    return torch.cat([Xc.reshape(-1, 3 * npts), u_bg.view(-1, 3 * npts)], dim=1).float()


def fiber_targets(T: torch.Tensor, f: torch.Tensor, npts: int = 32) -> torch.Tensor:
    """(nfib, 128): tensions and force densities."""
    return torch.cat([T.view(-1, npts), f.view(-1, 3 * npts)], dim=1).float()


# ------------------------------------------------------------ time marching --
def background_velocity(system, x_prev: torch.Tensor | None) -> torch.Tensor:
    """Velocity on every fiber point from everything except the fiber itself:
    the explicit flow of the external forces plus, when a previous solution
    is given, the flow of its fiber forces, body and periphery densities
    evaluated at the current geometry (one matvec's pair sums)."""
    u = system.flow_ext.clone()
    if x_prev is not None:
        y = torch.empty_like(x_prev)
        system.matvec(x_prev, y)
        u += system.v.view(-1, 3)[:system.nF]
    return u


def solution_targets(system, sol: torch.Tensor):
    """(T, f): tensions and force densities f = -E X_ssss + (T X_s)_s of the
    solved step, per fiber point (force operator at the solution)."""
    nF = system.nF
    f = torch.empty((nF, 3), dtype=torch.float64, device=sol.device)
    XT = sol[system.o_fib:]
    _lib.call("f3d_fiber_forces", ctypes.byref(system.fs.c), system.p.E, _lib.ptr(system.geo), _lib.ptr(XT),
              _lib.ptr(f), nF, 0, _lib.stream_handle(sol.device))
    n = int(system.fs.npts[0])
    T = XT.view(-1, 4, n)[:, 3, :].reshape(-1)
    return T, f


def guess_from_prediction(system, pred: torch.Tensor, u_bg: torch.Tensor,
                          x_prev: torch.Tensor | None) -> torch.Tensor:
    """GMRES initial guess from network output (T^, f^) per fiber:
    X^ = X^n + dt (u_bg + M f^) with the local slender-body mobility
    M f = c0 (f + xs (xs.f)) + c1 (f - xs (xs.f)); periphery and body
    unknowns from the previous solution (zero at the first step)."""
    n = int(system.fs.npts[0])
    nfib = system.fs.nfib
    x0 = x_prev.clone() if x_prev is not None else torch.zeros(system.size, dtype=torch.float64,
                                                               device=system.device)
    pred = pred.double()
    T = pred[:, :n]
    f = pred[:, n:].reshape(nfib * n, 3)
    xs = system.geo[:system.nF, 0:3]
    xf = (xs * f).sum(1, keepdim=True)
    Mf = system.c0 * (f + xs * xf) + system.c1 * (f - xs * xf)
    X = system.x_fib + system.p.dt * (u_bg + Mf)
    blk = x0[system.o_fib:].view(nfib, 4, n)
    blk[:, :3, :] = X.view(nfib, n, 3).transpose(1, 2)
    blk[:, 3, :] = T
    return x0


def march(system, steps: int, guess: str = "zero", net: FiberMLP | None = None, tol=1e-8,
          mixed=False, record=False, restart=100):
    """Advance `system` `steps` time steps; per step return iterations, time
    and (when record) the network's training pairs.

    guess: 'zero' (fiber3d's GMRES start), 'previous' (last solution) or
    'learned' (network prediction, then the same GMRES to the same residual).
    """
    x_prev = None
    stats, feats, targs = [], [], []
    n = int(system.fs.npts[0])
    for s in range(steps):
        if s > 0:
            system.advance(x_prev)
        u_bg = background_velocity(system, x_prev)
        X_feat = fiber_features(system.x_fib, u_bg, n)
        if guess == "learned" and net is not None:
            x0 = guess_from_prediction(system, net.predict(X_feat), u_bg, x_prev)
        elif guess in ("previous", "learned") and x_prev is not None:
            x0 = x_prev
        else:
            x0 = None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = system.solve(tol=tol, restart=restart, x0=x0, mixed=mixed)
        e1.record()
        e1.synchronize()
        sol = res["x"]
        st = {"iterations": res["iterations"], "solve_ms": e0.elapsed_time(e1),
              "initial_rel_residual": res["history"][0], "converged": res["info"] == 0}
        stats.append(st)
        if res["info"] != 0 or not bool(torch.isfinite(sol).all()):
            break  # a trajectory that stops converging ends here; its step is not recorded
        if record:
            T, f = solution_targets(system, sol)
            y = fiber_targets(T, f, n)
            if bool(torch.isfinite(X_feat).all() and torch.isfinite(y).all()):
                feats.append(X_feat)
                targs.append(y)
        x_prev = sol
    if record:
        empty = torch.zeros((0, 192), dtype=torch.float32, device=system.device)
        return (stats, torch.cat(feats) if feats else empty,
                torch.cat(targs) if targs else empty[:, :128])
    return stats
