"""Build recipe for the fiber3d_b200 shared library (sm_100a).

Compiles every ``csrc/*.cu`` with nvcc for ``compute_100a/sm_100a`` into
objects under ``_build/`` (parallel), then links ``fiber3d_b200/_lib/
libfiber3d_b200.so`` in-tree so that it travels with the repository
snapshot.  Cross-compiles without a GPU.

    python -m fiber3d_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIBDIR = PKG / "_lib"
LIBNAME = "libfiber3d_b200.so"
LIBPATH = LIBDIR / LIBNAME

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the fiber3d_b200 CUDA library cannot be built")
    return cand


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [_nvcc(), *NVCC_FLAGS, *extra, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile and link the library; returns the path of the .so."""
    extra = list(extra_flags or [])
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = _sources()
    hdrs = _headers()
    objs = []
    jobs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *hdrs]):
            jobs.append((s, o))
    if jobs:
        workers = max(1, min(len(jobs), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(workers) as ex:
            futs = {ex.submit(_compile, s, o, extra): s for s, o in jobs}
            for f in cf.as_completed(futs):
                f.result()
                if verbose:
                    print(f"compiled {futs[f].name}", file=sys.stderr)
    if force or jobs or _stale(LIBPATH, objs):
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
               "--cudart", "static", "-o", str(LIBPATH), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIBPATH


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)
