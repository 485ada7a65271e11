"""ctypes access to the C/OpenMP pair-sum oracle (``oracle/pairs_oracle.c``).

Test infrastructure and timed CPU baseline only.  ``build()`` compiles the C
file with gcc into ``oracle/_build/liboracle_pairs.so``.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "pairs_oracle.c"
OUT = HERE / "_build" / "liboracle_pairs.so"

KINDS = {"oseen": 0, "stresslet": 1, "rotlet": 2}
MODES = {"regularise": 0, "skip_index": 1, "skip_group": 2}

_dll = None


def build(force: bool = False) -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if force or not OUT.exists() or OUT.stat().st_mtime < SRC.stat().st_mtime:
        cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", str(OUT), str(SRC), "-lm"]
        subprocess.run(cmd, check=True)
    return OUT


def _lib():
    global _dll
    if _dll is None:
        build()
        d = ctypes.CDLL(str(OUT))
        P, I64, D, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        d.oracle_pair_sum.argtypes = [I, I, P, P, P, P, P, P, P, I64, I64, D, D, D, I]
        d.oracle_pair_sum.restype = None
        d.oracle_max_threads.restype = I
        _dll = d
    return _dll


def max_threads() -> int:
    return _lib().oracle_max_threads()


def _c(a, dtype=np.float64):
    return None if a is None else np.ascontiguousarray(np.asarray(a, dtype=dtype))


def pair_sum(kind: str, r_source, r_target, density, normal=None, *, eta=1.0, reg=5e-3,
             epsilon_distance=1e-5, self_mode="regularise", src_group=None, trg_group=None,
             nthreads: int = 0) -> np.ndarray:
    rs, rt, d, n = _c(r_source), _c(r_target), _c(density), _c(normal)
    gs, gt = _c(src_group, np.int32), _c(trg_group, np.int32)
    ns, nt = rs.size // 3, rt.size // 3
    out = np.zeros(3 * nt)
    p = lambda a: None if a is None else a.ctypes.data
    _lib().oracle_pair_sum(KINDS[kind], MODES[self_mode], p(rs), p(rt), p(d), p(n), p(gs), p(gt),
                           p(out), ns, nt, float(eta), float(reg), float(epsilon_distance),
                           int(nthreads))
    return out
