"""Learned GMRES warm start: a per-fiber network, trained on the solver's
own time steps, that corrects the polynomial extrapolation of the last
solutions.

fiber3d starts every GMRES solve from zero (tstep/tstep.py:1209).  Along a
trajectory the solution changes smoothly, so the quadratic extrapolation
x_q = 3 x^n - 3 x^{n-1} + x^{n-2} of the last three solutions is already a
close guess; what is left is mostly per fiber (its bending and tension
dynamics).  The network predicts, per fiber of 32 points, the correction
x^{n+1} - x_q on that fiber's unknowns (positions and tensions) from the
fiber's recent differences, each in units of its own size so that nothing
depends on how fast the fiber moves:

  input  (260) = D2 X^n / s2_X (96),  D3 X^n / s2_X (96),
                 D2 T^n / s2_T (32),  D3 T^n / s2_T (32),
                 log10 of s3/s2 and s2/s1 for X and T (4)
  output (128) = (X^{n+1} - X_q) / s2_X (96),  (T^{n+1} - T_q) / s2_T (32)

where D1 X^n = X^n - X^{n-1}, D2 X^n = D1 X^n - D1 X^{n-1}, D3 X^n =
X^n - 3 X^{n-1} + 3 X^{n-2} - X^{n-3} (note X^{n+1} - X_q = D3 X^{n+1}, so
cubic extrapolation is the map output = D3 X^n / s2_X), and sk is the
root-mean-square of Dk over the fiber.  The correction is
projected on the first few Legendre modes along the fiber before it is used:
a point-to-point wiggle in a position guess is multiplied by the fourth
derivative in the bending operator, so the correction must be smooth to
lower the residual.  A gain per unknown group (positions, tensions), fitted
by least squares on held-out steps and kept in [0, 1], scales it, and a
factor per group is then chosen among a few candidates (0 included) by the
GMRES iterations it gives on held-out trajectories: a correction that does
not strictly shorten GMRES there is switched off, and where both are off the
guess is the extrapolation.
Periphery and body unknowns take x_q.  At inference the features, the
network (output statistics, smoothing and gains folded into its last
layer) and the guess take six kernel launches.

3 hidden layers of 256 with ReLU; weights kept in FP32 (master copy, Adam)
and rounded to BF16 when staged for the tensor cores; every product runs in
``f3d_gemm_bf16`` (tcgen05, FP32 accumulation in tensor memory), the
backward pass included.  GMRES then runs from the corrected guess to the
same relative residual, so the converged answer does not depend on the
network; what it changes is the number of iterations.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

LAYERS = (260, 256, 256, 256, 128)
NPTS = 32          # points per fiber the network is built for
CLIP = 50.0        # bound on normalised correction targets
MODES = 10         # Legendre modes kept in a correction along the fiber
HISTORY = 4        # solutions the features need


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
    """A per-fiber network (ReLU hidden layers) with its own forward,
    backward and Adam kernels; `layers` gives the widths, input first."""

    def __init__(self, seed: int = 0, device=None, layers=LAYERS):
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.layers = tuple(layers)
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []
        for k in range(len(self.layers) - 1):
            fan_in, fan_out = self.layers[k], self.layers[k + 1]
            w = rng.normal(scale=np.sqrt(2.0 / fan_in), size=(fan_out, fan_in)).astype(np.float32)
            if k == len(self.layers) - 2:
                w *= 0.1
            self.W.append(torch.as_tensor(w, device=dev))
            self.b.append(torch.zeros(fan_out, dtype=torch.float32, device=dev))
        self.params = self.W + self.b
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step = 0
        self.in_mean = torch.zeros(self.layers[0], device=dev)
        self.in_std = torch.ones(self.layers[0], device=dev)
        self.out_mean = torch.zeros(self.layers[-1], device=dev)
        self.out_std = torch.ones(self.layers[-1], device=dev)

    # ------------------------------------------------------------- passes --
    def forward(self, X: torch.Tensor, keep=False):
        """X: (B, layers[0]) normalised inputs -> (B, layers[-1]) normalised outputs."""
        acts, pres = [X.contiguous()], []
        h = acts[0]
        L = len(self.W)
        for k in range(L):
            last = k == L - 1
            pre = torch.empty((h.shape[0], self.layers[k + 1]), dtype=torch.float32, device=X.device) \
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
            # dW = D^T Ain  (M = out, N = in, K = batch); the GEMM's N is a
            # multiple of 16 up to 256, so a wider or ragged input layer
            # takes (Ain^T D)^T instead
            n_in = Ain.shape[1]
            if n_in <= 256 and n_in % 16 == 0:
                gW[k] = gemm(D, Ain, transpose_a=True, transpose_b=False)
            else:
                gW[k] = gemm(Ain, D, transpose_a=True, transpose_b=False).t().contiguous()
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


# ------------------------------------------------------- history features --
def fiber_blocks(system, x: torch.Tensor) -> torch.Tensor:
    """(nfib, 4, N) view of the fiber unknowns of x: rows X_x, X_y, X_z, T
    (fiber3d's layout, tstep_utils.py:906-931)."""
    return x[system.o_fib:].view(system.fs.nfib, 4, NPTS)


def learnable(system) -> bool:
    """The network applies to systems whose fibers all have NPTS points."""
    return system.fs.nfib > 0 and bool(np.all(system.fs.npts == NPTS))


def extrapolate(history) -> torch.Tensor | None:
    """Polynomial extrapolation of the last solutions (newest last):
    constant, linear or quadratic with one, two or three of them."""
    if not history:
        return None
    if len(history) == 1:
        return history[-1].clone()
    if len(history) == 2:
        return 2.0 * history[-1] - history[-2]
    return 3.0 * history[-1] - 3.0 * history[-2] + history[-3]


def history_features(system, history):
    """(nfib, 260) network input from the last four solutions, and the
    per-fiber scales s2_X (nfib, 1, 1) and s2_T (nfib, 1) of the targets."""
    B = [fiber_blocks(system, h) for h in history[-4:]][::-1]  # newest first
    X = [b[:, :3] for b in B]
    T = [b[:, 3] for b in B]
    d1X, d1T = X[0] - X[1], T[0] - T[1]
    d2X, d2T = d1X - (X[1] - X[2]), d1T - (T[1] - T[2])
    d3X = X[0] - 3.0 * X[1] + 3.0 * X[2] - X[3]
    d3T = T[0] - 3.0 * T[1] + 3.0 * T[2] - T[3]
    rmsX = lambda d: d.square().mean(dim=(1, 2), keepdim=True).sqrt() + 1e-300
    rmsT = lambda d: d.square().mean(dim=1, keepdim=True).sqrt() + 1e-300
    s1X, s2X, s3X = rmsX(d1X), rmsX(d2X), rmsX(d3X)
    s1T, s2T, s3T = rmsT(d1T), rmsT(d2T), rmsT(d3T)
    ratios = torch.cat([torch.log10(s3X / s2X).view(-1, 1), torch.log10(s3T / s2T),
                        torch.log10(s2X / s1X).view(-1, 1), torch.log10(s2T / s1T)], dim=1)
    feats = torch.cat([(d2X / s2X).flatten(1), (d3X / s2X).flatten(1), d2T / s2T, d3T / s2T, ratios], dim=1)
    return feats.float().contiguous(), s2X, s2T


def mode_projection(npts: int = NPTS, modes: int = MODES, device=None) -> torch.Tensor:
    """(npts, npts) orthogonal projection on the Legendre polynomials of
    degree < modes sampled at the fiber's equispaced parameter points."""
    s = np.linspace(-1.0, 1.0, npts)
    V = np.polynomial.legendre.legvander(s, modes - 1)
    Q, _ = np.linalg.qr(V)
    return torch.as_tensor(Q @ Q.T, dtype=torch.float32, device=device)


def correction_targets(system, x_new: torch.Tensor, x_q: torch.Tensor, sX, sT) -> torch.Tensor:
    """(nfib, 128) normalised correction x_new - x_q on the fiber unknowns."""
    d = fiber_blocks(system, x_new) - fiber_blocks(system, x_q)
    t = torch.cat([(d[:, :3] / sX).flatten(1), d[:, 3] / sT], dim=1)
    return t.clamp(-CLIP, CLIP).float().contiguous()


def apply_correction(system, x_q: torch.Tensor, corr: torch.Tensor, sX, sT) -> torch.Tensor:
    """x_q with a normalised correction (nfib, 128) added on the fiber unknowns."""
    x0 = x_q.clone()
    B = fiber_blocks(system, x0)
    c = corr.double()
    B[:, :3] += c[:, :3 * NPTS].view(-1, 3, NPTS) * sX
    B[:, 3] += c[:, 3 * NPTS:] * sT
    return x0


class LearnedWarmStart:
    """FiberMLP + smoothing projection + held-out gains: the learned
    correction of the quadratic extrapolation."""

    def __init__(self, seed: int = 0, device=None, modes: int = MODES):
        self.net = FiberMLP(seed=seed, device=device)
        self.device = self.net.device
        self.P = mode_projection(NPTS, modes, self.device)
        self.gain = torch.ones(2, dtype=torch.float32, device=self.device)
        self.scale = (1.0, 1.0)   # factors on the position / tension correction, chosen on held-out trajectories
        self._fold = None         # inference weights (see _folded)

    def smooth(self, Y: torch.Tensor) -> torch.Tensor:
        """Project each of the 4 rows (X, Y, Z, T) of a (B, 128) correction."""
        return (Y.view(-1, 4, NPTS) @ self.P.T).reshape(-1, 4 * NPTS)

    def predict(self, feats: torch.Tensor) -> torch.Tensor:
        """Smoothed, gain-scaled normalised correction (B, 128)."""
        C = self.smooth(self.net.predict(feats))
        C[:, :3 * NPTS] *= self.gain[0] * self.scale[0]
        C[:, 3 * NPTS:] *= self.gain[1] * self.scale[1]
        return C

    def fit(self, X: torch.Tensor, T: torch.Tensor, epochs=30, batch=1024, lr=1e-3, val_frac=0.1,
            seed=0):
        """Train on smoothed targets, then fit the gains on a held-out split.
        Returns the training loss history."""
        g = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(X.shape[0], generator=g).to(X.device)
        nval = max(1, int(val_frac * X.shape[0]))
        iv, it = perm[:nval], perm[nval:]
        Ts = self.smooth(T)
        self.net.set_normalisation(X[it], Ts[it])
        hist = self.net.train(X[it].contiguous(), Ts[it].contiguous(), epochs=epochs,
                              batch=min(batch, max(1, it.numel())), lr=lr, seed=seed)
        self.gain.fill_(1.0)
        C = self.smooth(self.net.predict(X[iv].contiguous()))
        Tv = T[iv]
        for k, sl in enumerate((slice(0, 3 * NPTS), slice(3 * NPTS, 4 * NPTS))):
            num = float((C[:, sl] * Tv[:, sl]).sum())
            den = float((C[:, sl] * C[:, sl]).sum())
            self.gain[k] = min(1.0, max(0.0, num / den)) if den > 0 else 0.0
        self._fold = None
        return hist

    def select_scale(self, make_systems, steps: int, candidates=(0.0, 0.5, 1.0), tol=1e-8,
                     count_from: int = HISTORY) -> dict:
        """Pick the (position, tension) correction factors with the fewest
        GMRES iterations over held-out trajectories, counted where the
        network acts.  ``make_systems()`` returns fresh systems at the
        trajectories' first steps; steps from `count_from` on are counted.
        A correction must strictly lower the
        iteration count to be kept: on a tie the smaller factors win, so a
        network that does not shorten GMRES is switched off (the guess is
        then the extrapolation)."""
        score = {}
        for cx in candidates:
            for ct in candidates:
                self.scale = (cx, ct)
                self._fold = None
                its, lr0 = 0, []
                for sysd in make_systems():
                    st = march(sysd, steps, guess="learned", net=self, tol=tol)
                    acting = st[max(count_from, HISTORY):]
                    its += sum(x["iterations"] for x in acting)
                    lr0 += [np.log(max(x["initial_rel_residual"], 1e-300)) for x in acting]
                score[(cx, ct)] = (its, cx + ct, float(np.exp(np.mean(lr0))) if lr0 else 1.0)
        self.scale = min(score, key=lambda c: score[c][:2])
        self._fold = None
        return {f"{c[0]},{c[1]}": {"iterations": v[0], "r0_geomean": v[2]} for c, v in score.items()}

    def _folded(self):
        """Inference weights: the output un-normalisation, the smoothing
        projection and the gains folded into the last layer (FP32 master
        values; the GEMM rounds them to BF16 like every weight)."""
        if self._fold is None:
            net = self.net
            Pi = torch.block_diag(self.P, self.P, self.P, self.P)
            g = torch.cat([self.gain[0].expand(3 * NPTS) * self.scale[0], self.gain[1].expand(NPTS) * self.scale[1]])
            M = g[:, None] * Pi
            W = list(net.W[:-1]) + [(M @ (net.out_std[:, None] * net.W[-1])).contiguous()]
            b = list(net.b[:-1]) + [(M @ (net.out_std * net.b[-1] + net.out_mean)).contiguous()]
            self._fold = (W, b)
        return self._fold

    def guess_reference(self, system, history) -> torch.Tensor | None:
        """The same guess from PyTorch ops around the network (test reference
        of :meth:`guess`)."""
        x_q = extrapolate(history)
        if len(history) < HISTORY or not learnable(system) or self.scale == (0.0, 0.0):
            return x_q
        f, sX, sT = history_features(system, history)
        return apply_correction(system, x_q, self.predict(f), sX, sT)

    def guess(self, system, history) -> torch.Tensor | None:
        """The warm start: quadratic extrapolation, corrected by the network
        once HISTORY solutions are known.  Six launches: the feature kernel
        (standardised inputs), four tensor-core GEMMs (the last one with the
        smoothing and gains folded in) and the guess kernel."""
        if len(history) < HISTORY or not learnable(system) or self.scale == (0.0, 0.0):
            return extrapolate(history)
        W, b = self._folded()
        h0, h1, h2, h3 = (h.contiguous() for h in history[-HISTORY:])
        nfib = system.fs.nfib
        dev = h3.device
        st = _lib.stream_handle(dev)
        feats = torch.empty((nfib, LAYERS[0]), dtype=torch.float32, device=dev)
        sx = torch.empty(nfib, dtype=torch.float64, device=dev)
        sT = torch.empty(nfib, dtype=torch.float64, device=dev)
        _lib.call("f3d_warmstart_features", _lib.ptr(h0), _lib.ptr(h1), _lib.ptr(h2), _lib.ptr(h3), h3.numel(),
                  system.o_fib, nfib, NPTS, _lib.ptr(self.net.in_mean), _lib.ptr(self.net.in_std), _lib.ptr(feats),
                  _lib.ptr(sx), _lib.ptr(sT), st)
        h = feats
        for k in range(len(W)):
            h = gemm(h, W[k], bias=b[k], relu=k < len(W) - 1)
        x0 = torch.empty_like(h3)
        _lib.call("f3d_warmstart_guess", _lib.ptr(h1), _lib.ptr(h2), _lib.ptr(h3), h3.numel(), system.o_fib, nfib,
                  NPTS, _lib.ptr(h), _lib.ptr(sx), _lib.ptr(sT), _lib.ptr(x0), st)
        return x0


def learned_guess(system, history, model: LearnedWarmStart | None) -> torch.Tensor | None:
    """Extrapolation plus the learned correction (plain extrapolation
    without a model)."""
    if model is None:
        return extrapolate(history)
    return model.guess(system, history)


# ------------------------------------------------------------ time marching --
def march(system, steps: int, guess: str = "zero", net: LearnedWarmStart | None = None, tol=1e-8,
          mixed=False, record=False, restart=100, record_from: int = 0):
    """Advance `system` `steps` time steps; per step return iterations, time
    and (when record) the network's training pairs from step `record_from`
    on.

    guess: 'zero' (fiber3d's GMRES start), 'previous' (last solution),
    'extrapolate' (quadratic extrapolation) or 'learned' (extrapolation plus
    the network's correction); GMRES then runs to the same residual.
    """
    if guess not in ("zero", "previous", "extrapolate", "learned"):
        raise ValueError(f"unknown guess {guess!r}")
    history = []
    stats, feats, targs = [], [], []
    can_learn = learnable(system)
    for s in range(steps):
        # the guess depends only on the previous solutions, so it is formed
        # before the geometry moves and handed to advance() (which then sums
        # its Oseen flow together with the explicit flow)
        x_q = extrapolate(history)
        f = None
        if can_learn and len(history) >= HISTORY and record and s >= record_from:
            f, sX, sT = history_features(system, history)
        if guess == "zero":
            x0 = None
        elif guess == "previous":
            x0 = history[-1] if history else None
        elif guess == "learned" and net is not None:
            x0 = net.guess(system, history)
        else:
            x0 = x_q
        if s > 0:
            system.advance(history[-1], x0=x0)
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
        if record and f is not None:
            y = correction_targets(system, sol, x_q, sX, sT)
            ok = torch.isfinite(f).all(dim=1) & torch.isfinite(y).all(dim=1)
            feats.append(f[ok])
            targs.append(y[ok])
        history = (history + [sol])[-HISTORY:]
    if record:
        empty = torch.zeros((0, LAYERS[0]), dtype=torch.float32, device=system.device)
        return (stats, torch.cat(feats) if feats else empty,
                torch.cat(targs) if targs else torch.zeros((0, LAYERS[-1]), dtype=torch.float32,
                                                           device=system.device))
    return stats
