"""Batched LU of uneven dense blocks on the GPU (the block-diagonal
preconditioner of fiber3d's GMRES, tstep/tstep.py:950-994).

:class:`BlockLU` packs a list of square blocks into one device buffer, factors
them all in one persistent launch and solves them all in one launch, through
``f3d_batched_lu_factor`` / ``f3d_batched_lu_solve``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


class BlockLU:
    """Factors of ``len(sizes)`` square blocks stored back to back.

    ``sizes`` fixes the layout; :meth:`load` (or :attr:`A` written by a device
    kernel) fills the blocks, :meth:`factor` factors them in place and
    :meth:`solve` solves ``block_b x_b = r_b`` for a packed right-hand side.
    """

    def __init__(self, sizes, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else device
        sizes = np.asarray(sizes, dtype=np.int64)
        self.sizes_h = sizes
        self.count = int(sizes.size)
        self.max_n = int(sizes.max()) if self.count else 0
        moff = np.concatenate([[0], np.cumsum(sizes * sizes)[:-1]]) if self.count else np.zeros(0, np.int64)
        voff = np.concatenate([[0], np.cumsum(sizes)[:-1]]) if self.count else np.zeros(0, np.int64)
        self.moff_h, self.voff_h = moff.astype(np.int64), voff.astype(np.int64)
        self.nvec = int(sizes.sum())
        dev = self.device
        self.moff = torch.as_tensor(self.moff_h, device=dev)
        self.voff = torch.as_tensor(self.voff_h, device=dev)
        self.sizes = torch.as_tensor(sizes.astype(np.int32), device=dev)
        self.order = torch.as_tensor(np.argsort(-sizes, kind="stable").astype(np.int32), device=dev)
        self.A = torch.zeros(int((sizes * sizes).sum()), dtype=torch.float64, device=dev)
        self.piv = torch.zeros(self.nvec, dtype=torch.int32, device=dev)
        self.info = torch.zeros(max(self.count, 1), dtype=torch.int32, device=dev)
        nb = ctypes.c_size_t(0)
        _lib.call("f3d_batched_lu_workspace_bytes", ctypes.byref(nb))
        self.ws = torch.zeros(nb.value, dtype=torch.uint8, device=dev)

    def block(self, b: int) -> torch.Tensor:
        n = int(self.sizes_h[b])
        o = int(self.moff_h[b])
        return self.A[o:o + n * n].view(n, n)

    def load(self, blocks) -> None:
        for b, M in enumerate(blocks):
            self.block(b).copy_(torch.as_tensor(np.asarray(M, dtype=np.float64)))

    panel = 0  # panel width of the factorisation (0: size-based default)

    def tune_panel(self, reps: int = 3) -> int:
        """Time the panel widths 8/16/32 on the current blocks and keep the
        fastest (restores the blocks afterwards)."""
        saved = self.A.clone()
        best, best_t = 0, float("inf")
        for p in (8, 16, 32):
            from ._lib import F3DError
            try:
                self.A.copy_(saved)
                self.panel = p
                self.factor()
                torch.cuda.synchronize()
                t = float("inf")
                for _ in range(reps):
                    self.A.copy_(saved)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    self.factor()
                    e1.record()
                    e1.synchronize()
                    t = min(t, e0.elapsed_time(e1))
            except F3DError:
                continue
            if t < best_t:
                best, best_t = p, t
        self.A.copy_(saved)
        self.panel = best
        return best

    def factor(self, blocks=None) -> None:
        """Factor every block, or only the listed block indices."""
        if self.count == 0:
            return
        if blocks is None:
            order, count = self.order, self.count
        else:
            key = tuple(int(b) for b in blocks)
            cached = getattr(self, "_subset", None)
            if cached is None or cached[0] != key:
                sel = np.asarray(key, dtype=np.int64)
                sel = sel[np.argsort(-self.sizes_h[sel], kind="stable")]
                self._subset = (key, torch.as_tensor(sel.astype(np.int32), device=self.device))
            order, count = self._subset[1], len(key)
            if count == 0:
                return
        mx = self.max_n if blocks is None else int(self.sizes_h[list(blocks)].max())
        _lib.call("f3d_batched_lu_factor_panel", _lib.ptr(self.A), _lib.ptr(self.moff), _lib.ptr(self.voff),
                  _lib.ptr(self.sizes), _lib.ptr(order), count, mx, int(self.panel),
                  _lib.ptr(self.piv), _lib.ptr(self.info), _lib.ptr(self.ws), self.ws.numel(),
                  _lib.stream_handle(self.device))

    def check(self) -> None:
        """Raise if any block had a zero pivot (synchronises)."""
        bad = torch.nonzero(self.info[:self.count]).flatten()
        if bad.numel():
            b = int(bad[0])
            raise ZeroDivisionError(f"block {b}: zero pivot at step {int(self.info[b])}")

    A32 = None  # FP32 copy of the inverses (invert(fp32=True))

    def invert(self, fp32: bool = True) -> None:
        """Replace every block by its explicit inverse (Gauss-Jordan, blocks up
        to 128), and with ``fp32`` also keep an FP32 copy; :meth:`apply` then
        evaluates the preconditioner as one streaming pass over the blocks."""
        if self.count == 0:
            return
        if fp32 and self.A32 is None:
            self.A32 = torch.zeros(self.A.numel(), dtype=torch.float32, device=self.device)
        _lib.call("f3d_batched_inverse", _lib.ptr(self.A), _lib.ptr(self.moff), _lib.ptr(self.sizes), self.count,
                  self.max_n, _lib.ptr(self.A32) if fp32 else None, _lib.ptr(self.info),
                  _lib.stream_handle(self.device))

    def apply(self, x: torch.Tensor, y: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
        """y = blockdiag(inverses) x after :meth:`invert` (x, y distinct,
        packed like the right-hand side of :meth:`solve`)."""
        if self.count:
            M = self.A if precision == "fp64" else self.A32
            if M is None:
                raise RuntimeError("no FP32 inverses: call invert(fp32=True)")
            _lib.call("f3d_block_gemv", _lib.PRECISION[precision], _lib.ptr(M), _lib.ptr(self.moff),
                      _lib.ptr(self.voff), _lib.ptr(self.sizes), self.count, self.max_n, _lib.ptr(x), _lib.ptr(y),
                      _lib.stream_handle(self.device))
        return y

    def solve(self, x: torch.Tensor) -> torch.Tensor:
        """Solve in place for a packed right-hand side of length sum(sizes)."""
        if x.numel() != self.nvec or x.dtype != torch.float64 or not x.is_contiguous():
            raise ValueError("right-hand side must be a contiguous float64 vector of length sum(sizes)")
        if self.count:
            _lib.call("f3d_batched_lu_solve", _lib.ptr(self.A), _lib.ptr(self.moff), _lib.ptr(self.voff),
                      _lib.ptr(self.sizes), _lib.ptr(self.order), self.count, self.max_n,
                      _lib.ptr(self.piv), _lib.ptr(x), _lib.ptr(self.ws), self.ws.numel(),
                      _lib.stream_handle(self.device))
        return x
