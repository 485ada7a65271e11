"""The Python API of the STKFMM library as fiber3d calls it
(python/kernels/kernels.py:24-28, 1298-1485; tstep/tstep.py:116-137;
kernels/test_stkfmm.py), over this package's GPU FMM (``fmm.FMM``).

fiber3d's useFMM path imports ``stkfmm``; with

    import sys, fiber3d_b200.stkfmm
    sys.modules["stkfmm"] = fiber3d_b200.stkfmm

its ``*_stkfmm`` kernel functions run unchanged on the GPU.  Only what
those functions use is provided: the PVel kernel without periodicity,
velocity outputs (the pressure column of the target values is left at
zero: fiber3d reads only the velocity), single-layer source values
(f_x, f_y, f_z, TRD) with TRD = 0 (fiber3d passes zeros) and double-layer
values D_jk (9 per source, fiber3d passes 2 n (x) d).  Host numpy arrays in,
results written into the caller's ``trgValue`` array, as STKFMM does.
"""
from __future__ import annotations

import enum

import numpy as np
import torch

from .fmm import FMM


class KERNEL(enum.IntFlag):
    PVel = 1


class PAXIS(enum.IntEnum):
    NONE = 0


# (single-layer, double-layer, target) values per point of each kernel
_DIMS = {KERNEL.PVel: (4, 9, 4)}


class STKFMM:
    """STKFMM(order, max_pts, pbc, kernels): one handle per kernel set."""

    def __init__(self, order: int, max_pts: int, pbc, kernels):
        if PAXIS(pbc) != PAXIS.NONE:
            raise NotImplementedError("periodic boxes are not supported")
        if KERNEL(kernels) & ~KERNEL.PVel:
            raise NotImplementedError("only the PVel kernel is supported")
        self.fmm = FMM(order=order, max_pts=max_pts)
        self.box = None
        self.points = None
        self.tree = False

    @property
    def device(self):
        return self.fmm.device


def getKernelDimension(fmm: STKFMM, kernel) -> tuple[int, int, int]:
    return _DIMS[KERNEL(kernel)]


def setBox(fmm: STKFMM, xlow, xhigh, ylow, yhigh, zlow, zhigh):
    """The tree's box: the cube with the given lower corner whose side is the
    largest of the three extents (STKFMM's box is a cube)."""
    lo = np.array([xlow, ylow, zlow], dtype=np.float64)
    width = float(max(xhigh - xlow, yhigh - ylow, zhigh - zlow))
    fmm.fmm.set_box(lo, width)
    fmm.box = (lo, width)
    fmm.tree = False


def setPoints(fmm: STKFMM, nSL, srcSLCoord, nDL, srcDLCoord, nTrg, trgCoord):
    def pts(n, a):
        a = np.asarray(a, dtype=np.float64).reshape(-1)
        if n and a.size < 3 * n:
            raise ValueError("coordinate array shorter than 3 x count")
        return a[:3 * n].reshape(n, 3) if n else None
    fmm.points = (int(nSL), pts(nSL, srcSLCoord), int(nDL), pts(nDL, srcDLCoord), int(nTrg), pts(nTrg, trgCoord))
    fmm.tree = False


def setupTree(fmm: STKFMM, kernel):
    if fmm.points is None:
        raise RuntimeError("setPoints first")
    nsl, sl, ndl, dl, ntrg, trg = fmm.points
    fmm.fmm.set_points(sl, dl, trg)
    fmm.tree = True


def clearFMM(fmm: STKFMM, kernel):
    """Nothing to clear: every evaluation starts from zero."""


def evaluateFMM(fmm: STKFMM, nSL, srcSLValue, nDL, srcDLValue, nTrg, trgValue, kernel):
    """trgValue (nTrg x 4: pressure, velocity) += the PVel sums of the
    sources' values at the targets (the pressure column is not computed)."""
    if not fmm.tree:
        raise RuntimeError("setupTree first")
    nsl, ndl, ntrg = int(nSL), int(nDL), int(nTrg)
    if (nsl, ndl, ntrg) != (fmm.points[0], fmm.points[2], fmm.points[4]):
        raise ValueError("source / target counts differ from setPoints")
    f = D = None
    if nsl:
        v = np.asarray(srcSLValue, dtype=np.float64).reshape(nsl, 4)
        if np.any(v[:, 3] != 0.0):
            raise NotImplementedError("non-zero TRD single-layer values are not supported")
        f = np.ascontiguousarray(v[:, :3])
    if ndl:
        D = np.ascontiguousarray(np.asarray(srcDLValue, dtype=np.float64).reshape(ndl, 9))
    u = fmm.fmm.evaluate(sl_density=f, dl_tensor=D, eta=1.0)
    out = np.asarray(trgValue).reshape(ntrg, 4)
    out[:, 1:4] += u.view(ntrg, 3).cpu().numpy()
