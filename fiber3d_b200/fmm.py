"""Fast multipole evaluation of the Stokes single- and double-layer sums on
the GPU: the counterpart of the STKFMM library calls on fiber3d's useFMM
path (python/kernels/kernels.py:1298-1485; tstep/tstep.py:116-137).

The device side (``f3d_fmm_*`` in include/fiber3d_b200.h, csrc/f3d_fmm.cu)
builds a uniform octree and runs the kernel-independent FMM passes.  This
module computes what the device side takes as given, once per expansion
order: the unit cube's surface grid (``order`` points per edge) and the two
pseudo-inverses that turn a check potential into an equivalent density
(host SVD), and wraps the handle for torch device tensors.

Equivalent densities have four components per surface point, a Stokeslet
and a potential source r / r^3: the double layer of a density whose tensor
D = 2 n (x) d has a trace carries a net flux that Stokeslets alone cannot
represent (a Stokeslet layer is divergence free and flux free).
"""
from __future__ import annotations

import ctypes
import functools

import numpy as np
import torch

from . import _lib

R_IN, R_OUT = 1.05, 2.95


def surface(order: int) -> np.ndarray:
    """The points of the order x order x order grid on [-1, 1]^3 that lie on
    the cube's surface, n = 6 (order - 1)^2 + 2 of them, in lexicographic
    order."""
    g = np.linspace(-1.0, 1.0, order)
    pts = [(a, b, c) for a in g for b in g for c in g if max(abs(a), abs(b), abs(c)) > 1.0 - 1e-12]
    return np.ascontiguousarray(np.array(pts, dtype=np.float64))


def k4(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """The far-field kernel [I/r + r r^T/r^3 | r/r^3] between points x (rows,
    3 per point) and y (columns, 4 per point), no constants."""
    r = x[:, None, :] - y[None, :, :]
    d2 = np.einsum("ijk,ijk->ij", r, r)
    d = np.sqrt(d2)
    s = np.eye(3)[None, None] / d[..., None, None] + r[..., :, None] * r[..., None, :] / (d2 * d)[..., None, None]
    q = r / (d2 * d)[..., None]
    g = np.concatenate([s, q[..., None]], axis=-1)  # (nx, ny, 3, 4)
    return g.transpose(0, 2, 1, 3).reshape(3 * len(x), 4 * len(y))


# The check-to-equivalent maps are ill-conditioned (condition numbers 3e8 at
# order 6, 7e10 at 8, 1e14 at 10, 4e16 at 12): singular values below 1e-10
# of the largest only amplify rounding.  With this cut-off the single-box
# round trips reach, relative L2, 5e-6 (order 8), 7e-7 (10) and 1.3e-7 (12)
# for the double layer's upward density, the hardest of the four; with
# 1e-14 orders 10 and 12 lose two orders of magnitude to the noise.
PINV_RCOND = 1e-10


def pinv(a: np.ndarray, rcond: float = PINV_RCOND) -> np.ndarray:
    """Least-norm pseudo-inverse through the SVD, singular values below
    rcond * the largest dropped."""
    u, s, vt = np.linalg.svd(a, full_matrices=False)
    keep = s > rcond * s[0]
    return (vt[keep].T / s[keep]) @ u[:, keep].T


@functools.lru_cache(maxsize=8)
def operators(order: int):
    """(surface, uc2ue, dc2de) for expansions of this order: uc2ue maps the
    velocity on the upward check surface (R_OUT) to the equivalent density on
    the upward equivalent surface (R_IN) of a unit box; dc2de the downward
    check surface (R_IN) to the downward equivalent surface (R_OUT)."""
    if order < 4 or order > 16 or order % 2:
        raise ValueError("order must be even, 4..16")
    s = surface(order)
    uc2ue = np.ascontiguousarray(pinv(k4(R_OUT * s, R_IN * s)))
    dc2de = np.ascontiguousarray(pinv(k4(R_IN * s, R_OUT * s)))
    return s, uc2ue, dc2de


def _dev(a, device, name, cols=3):
    if a is None:
        return None
    t = torch.as_tensor(a, dtype=torch.float64, device=device).reshape(-1, cols).contiguous()
    return t


class FMM:
    """A device FMM handle: ``set_points`` builds the tree for single-layer
    sources, double-layer sources and targets; ``evaluate`` sums the layers'
    velocities at the targets (the PVel kernel's velocity, divided by eta).
    The near field (the 27 neighbour leaves) is summed directly, coincident
    points excluded."""

    def __init__(self, order: int = 8, max_pts: int = 1000, device=None):
        self.order = int(order)
        self.max_pts = int(max_pts)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        s, uc2ue, dc2de = operators(self.order)
        self.nsurf = s.shape[0]
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("f3d_fmm_create", self.order, self.max_pts, s.ctypes.data, uc2ue.ctypes.data,
                      dc2de.ctypes.data, ctypes.byref(h))
        self._h = h
        self._pts = None

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().f3d_fmm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def set_box(self, lo, width: float):
        lo = np.ascontiguousarray(np.asarray(lo, dtype=np.float64).reshape(3))
        _lib.call("f3d_fmm_set_box", self._h, lo.ctypes.data, float(width))

    def set_points(self, src_sl=None, src_dl=None, trg=None):
        """Sources (n x 3 each, either may be None) and targets, any array
        type; kept on the device in the handle's sorted order."""
        dev = self.device
        sl, dl, tg = _dev(src_sl, dev, "src_sl"), _dev(src_dl, dev, "src_dl"), _dev(trg, dev, "trg")
        if tg is None:
            raise ValueError("targets are required")
        self._pts = (sl, dl, tg)
        nsl = 0 if sl is None else sl.shape[0]
        ndl = 0 if dl is None else dl.shape[0]
        with torch.cuda.device(dev):
            _lib.call("f3d_fmm_set_points", self._h, nsl, _lib.ptr(sl), ndl, _lib.ptr(dl), tg.shape[0],
                      _lib.ptr(tg), _lib.stream_handle(dev))
        self.nsl, self.ndl, self.ntrg = nsl, ndl, tg.shape[0]

    def evaluate(self, sl_density=None, dl_normal=None, dl_density=None, dl_tensor=None, eta: float = 1.0,
                 out: torch.Tensor | None = None) -> torch.Tensor:
        """Velocity at the targets (flat 3 * ntrg float64 device tensor)."""
        if self._pts is None:
            raise RuntimeError("set_points first")
        dev = self.device
        f = _dev(sl_density, dev, "sl_density")
        n = _dev(dl_normal, dev, "dl_normal")
        d = _dev(dl_density, dev, "dl_density")
        D = _dev(dl_tensor, dev, "dl_tensor", cols=9)
        if self.nsl and (f is None or f.shape[0] != self.nsl):
            raise ValueError("sl_density must have one row per single-layer source")
        if self.ndl:
            if D is None and (n is None or d is None):
                raise ValueError("double-layer sources need dl_tensor or dl_normal and dl_density")
            if D is not None and D.shape[0] != self.ndl:
                raise ValueError("dl_tensor must have one row per double-layer source")
            if D is None and (n.shape[0] != self.ndl or d.shape[0] != self.ndl):
                raise ValueError("dl_normal / dl_density must have one row per double-layer source")
        if out is None:
            out = torch.empty(3 * self.ntrg, dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            _lib.call("f3d_fmm_evaluate", self._h, _lib.ptr(f), _lib.ptr(n), _lib.ptr(d), _lib.ptr(D),
                      _lib.ptr(out), float(eta), _lib.stream_handle(dev))
        return out

    def tree_info(self) -> dict:
        depth = ctypes.c_int(0)
        ns, nt, m2l = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        box = (ctypes.c_double * 4)()
        _lib.call("f3d_fmm_tree_info", self._h, ctypes.byref(depth), ctypes.byref(ns), ctypes.byref(nt), box,
                  ctypes.byref(m2l))
        return {"depth": depth.value, "source_leaves": ns.value, "target_leaves": nt.value,
                "box_lo": list(box[:3]), "box_width": box[3], "m2l_pairs": m2l.value}

    def last_launches(self) -> int:
        """Kernels the last evaluate launched."""
        v = ctypes.c_int(0)
        _lib.call("f3d_fmm_last_launches", self._h, ctypes.byref(v))
        return v.value

    def far_field_flops(self) -> float:
        """Algorithmic FP64 flops of the interaction lists per evaluation:
        2 (3n)(4n) per non-empty entry (the dominant far-field work)."""
        return 2.0 * 3 * self.nsurf * 4 * self.nsurf * self.tree_info()["m2l_pairs"]
