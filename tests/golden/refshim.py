"""Import shims that let fiber3d's own Python modules run on Python 3.12 /
scipy 1.18 (used only by the fixture generators in this folder, which run
where the fiber3d sources are available; the fixtures they write are what
the tests read).

Shims, all outside the fiber3d tree:
* ``imp`` (removed in Python 3.12; kernels.py:6,18-22): ``find_module``
  raises ImportError, so the optional PyCUDA branch is skipped.
* ``stkfmm`` and ``mpi4py`` (tstep.py:10,30): empty stand-ins (the FMM path
  is not used; ``MPI.`` is never referenced).
* ``numba.errors`` -> ``numba.core.errors`` (tstep_utils.py:45).
* ``scipy.sparse.linalg.gmres(tol=...)`` -> ``rtol=...`` (bpm_utilities/
  gmres.py:92,105; scipy >= 1.14 removed ``tol``).
"""
from __future__ import annotations

import os
import sys
import types

REFERENCE_PY = os.environ.get("FIBER3D_REFERENCE")


def install() -> str:
    if not REFERENCE_PY:
        raise RuntimeError("set FIBER3D_REFERENCE to the python/ folder of a fiber3d checkout "
                           "(the fixture generators run fiber3d's own code)")
    if "imp" not in sys.modules:
        imp = types.ModuleType("imp")

        def find_module(*_a, **_k):
            raise ImportError("imp shim: no optional modules")

        imp.find_module = find_module
        sys.modules["imp"] = imp
    sys.modules.setdefault("stkfmm", types.ModuleType("stkfmm"))
    if "mpi4py" not in sys.modules:
        mpi = types.ModuleType("mpi4py")
        mpi.MPI = types.SimpleNamespace()
        sys.modules["mpi4py"] = mpi
    import numba.core.errors as nerr
    sys.modules.setdefault("numba.errors", nerr)
    import scipy.sparse.linalg as spla
    if not getattr(spla.gmres, "_f3d_shim", False):
        orig = spla.gmres

        def gmres(A, b, x0=None, *args, tol=None, rtol=None, **kw):
            if rtol is None:
                rtol = 1e-5 if tol is None else tol
            kw.setdefault("callback_type", "legacy")
            return orig(A, b, x0, *args, rtol=rtol, **kw)

        gmres._f3d_shim = True
        spla.gmres = gmres
    if REFERENCE_PY not in sys.path:
        sys.path.insert(0, REFERENCE_PY)
    return REFERENCE_PY
