"""Launch-shape autotuner for the pair kernels.

For a (kernel, precision, self mode, Ns bucket, Nt bucket) key it times a
set of candidate shapes (targets per thread, source lanes per target, CTA
count via source splits, bulk-copy staging on/off) with CUDA events on the
current stream and keeps the fastest.  Results are cached in memory and in a
JSON file (``$FIBER3D_B200_TUNE`` or ``~/.cache/fiber3d_b200/pair_shapes.json``)
keyed by GPU name.  Candidates differ only in launch shape, so every one
computes the same sum (bit-identical for a fixed split count; within
rounding otherwise).
"""
from __future__ import annotations

import json
import math
import os
import threading
from pathlib import Path

import torch

from . import _lib

_lock = threading.Lock()
_cache: dict[str, list[int]] = {}
_loaded = False


def _path() -> Path:
    p = os.environ.get("FIBER3D_B200_TUNE")
    if p:
        return Path(p)
    return Path.home() / ".cache" / "fiber3d_b200" / "pair_shapes.json"


def _bucket(n: int) -> int:
    """Power-of-two bucket of a point count."""
    return 0 if n <= 0 else 1 << int(math.ceil(math.log2(n)))


_names: dict[int, str] = {}


def _key(kernel, precision, self_mode, ns, nt, same=False) -> str:
    """Cache key: GPU, sum, size buckets, and whether the sum runs over one
    point set (the sources are the first ns targets, which allows the
    symmetric form)."""
    dev = torch.cuda.current_device()
    name = _names.get(dev)
    if name is None:
        name = _names[dev] = torch.cuda.get_device_name(dev).replace(" ", "_")
    one = "|self" if (same and nt >= ns) else ""
    return f"{name}|{kernel}|{precision}|{self_mode}|{_bucket(ns)}|{_bucket(nt)}{one}"


# the symmetric self-sum's launch shape (f3d_pair_shape.sl = -1)
SYMMETRIC = (1, -1, 0, -1)
SYM_MAX_POINTS = 1024 * 128
TILE = (1, -2, 0, -1)


def symmetric_eligible(kernel, precision, self_mode, ns, nt, same) -> bool:
    """Whether the symmetric form can run this sum: FP64 Oseen or stresslet
    with a self rule, over one array whose first ns points are the sources
    (further targets after them are summed one-sided in the same launch)."""
    return (same and nt >= ns and 0 < ns <= SYM_MAX_POINTS and precision == "fp64"
            and kernel in ("oseen", "stresslet") and self_mode in ("skip_index", "skip_group"))


def tile_eligible(kernel, precision, self_mode, ns, nt) -> bool:
    """Whether the tile form (the symmetric kernel's target-side items for a
    plain source -> target sum) can run this sum: FP64 Oseen or stresslet,
    close pairs regularised, at most 1024 source tiles."""
    return (0 < ns <= SYM_MAX_POINTS and nt > 0 and precision == "fp64"
            and kernel in ("oseen", "stresslet") and self_mode == "regularise")


def _same_array(a, b) -> bool:
    """b is a, or both are device tensors starting at the same address
    (a = b[:ns], the sources as the first points of the targets)."""
    if a is b:
        return True
    return (isinstance(a, torch.Tensor) and isinstance(b, torch.Tensor) and a.is_cuda and b.is_cuda
            and a.data_ptr() == b.data_ptr())


def _load():
    global _loaded
    if _loaded:
        return
    _loaded = True
    try:
        _cache.update(json.loads(_path().read_text()))
    except (OSError, ValueError):
        pass


def _save():
    try:
        p = _path()
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(f".{os.getpid()}.tmp")  # one per process: ranks may write at once
        tmp.write_text(json.dumps(_cache, indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass


def occupancy(kernel: str, precision: str, self_mode: str, tpt: int, sl: int) -> int:
    """Resident CTAs per SM of the pair kernel of this shape (0 if unknown)."""
    import ctypes
    n = ctypes.c_int(0)
    shp = _lib.PairShape(tpt, sl, 0, 0)
    rc = _lib.lib().f3d_pair_occupancy(_lib.KERNEL[kernel], _lib.PRECISION[precision], _lib.SELF_MODE[self_mode],
                                       0, ctypes.byref(shp), ctypes.byref(n))
    return n.value if rc == 0 else 0


def candidates(nt: int, sms: int, occ=None):
    """Candidate (tpt, sl, nsplit, use_tma) shapes for nt targets: source
    splits giving about 4, 8 or 16 CTAs per SM and, where the occupancy
    `occ(tpt, sl)` is known, splits that fill 1-4 whole waves of resident
    CTAs (no partly-filled last wave)."""
    out = []
    for tpt, sl in ((1, 1), (2, 1), (4, 1), (1, 8), (1, 32)):
        tpb = (128 // sl) * tpt
        ntb = max(1, -(-nt // tpb))
        splits = {max(1, -(-per_sm * sms // ntb)) for per_sm in (4, 8, 16)}
        slots = occ(tpt, sl) * sms if occ is not None else 0
        for waves in (1, 2, 3, 4):
            if slots:
                splits.add(max(1, (waves * slots) // ntb))
        for nsplit in splits:
            for tma in (0, -1):
                out.append((tpt, sl, nsplit, tma))
    return sorted(set(out))


def tune(kernel: str, r_source, r_target, density, normal=None, *, self_mode="regularise",
         src_group=None, trg_group=None, precision="fp64", eta=1.0, reg=5e-3,
         epsilon_distance=1e-5, reps: int = 3, force: bool = False) -> _lib.PairShape:
    """Best launch shape for this sum (times the candidates on first use)."""
    from . import kernels as K
    ns = int(r_source.shape[0] if hasattr(r_source, "shape") and len(r_source.shape) == 2 else len(r_source) // 3)
    nt = int(r_target.shape[0] if hasattr(r_target, "shape") and len(r_target.shape) == 2 else len(r_target) // 3)
    same = (nt >= ns and _same_array(r_source, r_target)
            and (self_mode != "skip_group" or _same_array(src_group, trg_group)))
    with _lock:
        _load()
        key = _key(kernel, precision, self_mode, ns, nt, same)
        if key in _cache and not force:
            return _lib.PairShape(*_cache[key])
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    kw = dict(self_mode=self_mode, src_group=src_group, trg_group=trg_group, precision=precision,
              eta=eta, reg=reg, epsilon_distance=epsilon_distance)
    out = K.pair_sum(kernel, r_source, r_target, density, normal, **kw)
    best, best_t = None, float("inf")
    occ = lambda tpt, sl: occupancy(kernel, precision, self_mode, tpt, sl)
    cands = candidates(nt, sms, occ)
    if symmetric_eligible(kernel, precision, self_mode, ns, nt, same):
        cands.append(SYMMETRIC)
    if tile_eligible(kernel, precision, self_mode, ns, nt):
        cands += [(1, -2, 1, -1), (1, -2, 2, -1)]  # whole or half source tiles
    for cand in cands:
        shp = _lib.PairShape(*cand)
        try:
            K.pair_sum(kernel, r_source, r_target, density, normal, shape=shp, out=out, **kw)
        except _lib.F3DError:
            continue  # a shape this sum cannot take
        torch.cuda.synchronize()
        t = float("inf")
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            K.pair_sum(kernel, r_source, r_target, density, normal, shape=shp, out=out, **kw)
            e1.record()
            e1.synchronize()
            t = min(t, e0.elapsed_time(e1))
        if t < best_t:
            best, best_t = cand, t
    with _lock:
        _cache[key] = list(best)
        _save()
    return _lib.PairShape(*best)


def cached(kernel: str, precision: str, self_mode: str, ns: int, nt: int,
           same: bool = False) -> _lib.PairShape | None:
    """The tuned shape of this sum's bucket if one is known (no tuning)."""
    with _lock:
        _load()
        v = _cache.get(_key(kernel, precision, self_mode, ns, nt, same))
    return _lib.PairShape(*v) if v is not None else None


def table() -> dict:
    """The cached shapes (for reports)."""
    with _lock:
        _load()
        return dict(_cache)
