"""The C-ABI library loads (no GPU needed) and exports every symbol that
include/fiber3d_b200.h declares; host-side argument checks run without a
device (they return before any launch)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from fiber3d_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(f3d_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def dll():
    if not _lib.LIBPATH.exists():
        from fiber3d_b200 import build
        build.build()
    return _lib.load_library()


def test_every_declared_symbol_is_exported(dll):
    names = declared_symbols()
    assert len(names) >= 14
    for n in names:
        assert hasattr(dll, n), f"{n} declared in include/ but not exported"


def test_python_binding_covers_header(dll):
    missing = set(declared_symbols()) - set(_lib.SIGNATURES)
    assert not missing, f"no ctypes prototype for {sorted(missing)}"


def test_version_and_status_strings(dll):
    assert b"sm_100a" in dll.f3d_version()
    assert dll.f3d_status_string(0) == b"ok"
    assert dll.f3d_status_string(3).startswith(b"a pointer")


def test_workspace_query_and_argument_checks(dll):
    nbytes = ctypes.c_size_t(123)
    # FP64, large target count: one split, no workspace
    assert dll.f3d_pair_workspace_bytes(0, 0, 1 << 20, 1 << 20, None, ctypes.byref(nbytes)) == 0
    # small target count: source splits need partial sums
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 100, None, ctypes.byref(nbytes)) == 0
    assert nbytes.value > 0
    # FP32C packs sources in the workspace
    assert dll.f3d_pair_workspace_bytes(0, 1, 1000, 1 << 20, None, ctypes.byref(nbytes)) == 0
    assert nbytes.value >= 1000 * 48
    # bad enums / shapes are rejected on the host
    assert dll.f3d_pair_workspace_bytes(7, 0, 10, 10, None, ctypes.byref(nbytes)) == 5
    assert dll.f3d_pair_workspace_bytes(0, 0, -1, 10, None, ctypes.byref(nbytes)) == 2
    bad = _lib.PairShape(3, 1, 0, 0)
    assert dll.f3d_pair_workspace_bytes(0, 0, 10, 10, ctypes.byref(bad), ctypes.byref(nbytes)) == 5
    # null output pointer with work to do
    assert dll.f3d_oseen_source_target(None, None, None, None, 10, 10, 1.0, 5e-3, 1e-5, 0,
                                       None, 0, None) == 1
    # nothing to do: OK without touching the device
    assert dll.f3d_oseen_source_target(None, None, None, None, 10, 0, 1.0, 5e-3, 1e-5, 0,
                                       None, 0, None) == 0
    # every workspace keeps the split-counter region (256 KiB) at its start,
    # also an FP32C single-split one whose packed sources follow it
    one = _lib.PairShape(1, 8, 1, 0)
    assert dll.f3d_pair_workspace_bytes(1, 1, 1000, 100, ctypes.byref(one), ctypes.byref(nbytes)) == 0
    assert nbytes.value >= (256 << 10) + 1000 * 12 * 4
    # skip-index needs the sources as the first targets (nt >= ns)
    assert dll.f3d_pair_sum(0, 0, 1, 8, 8, 8, None, None, None, 8, 11, 10, 1.0, 5e-3, 1e-5, 0,
                            None, None, 0, None) == 2


def test_argument_checks_of_newer_entries(dll):
    """Shape, null-pointer and size checks of the body advance, batched
    GEMV and grid-velocity entries return before any launch."""
    NULL, SHAPE, TOO_LARGE = 1, 2, 10
    # nothing to do: OK without a device
    assert dll.f3d_body_advance(None, None, 0, 1e-3, None, None, None, None) == 0
    assert dll.f3d_gemv_batched(None, None, None, None, None, 0, 10, 0, None, None, None) == 0
    assert dll.f3d_grid_near_fiber(None, 0, None, None, 5, None, 0.2, None, None) == 0
    assert dll.f3d_grid_rigid_override(None, 0, None, None, 0.5, None, None) == 0
    assert dll.f3d_fiber_self_flow_up(None, None, None, 0, 32, None, None, None, None, 2, 1.0, 5e-3, 1e-5,
                                      None, None) == 0
    # negative sizes and null pointers with work to do
    assert dll.f3d_body_advance(None, None, -1, 1e-3, None, None, None, None) == SHAPE
    assert dll.f3d_body_advance(None, None, 2, 1e-3, None, None, None, None) == NULL
    assert dll.f3d_gemv_batched(None, None, None, None, None, -1, 10, 0, None, None, None) == SHAPE
    assert dll.f3d_gemv_batched(None, None, None, None, None, 2, 10, 0, None, None, None) == NULL
    assert dll.f3d_grid_near_fiber(None, -1, None, None, 5, None, 0.2, None, None) == SHAPE
    assert dll.f3d_grid_near_fiber(None, 10, None, None, 5, None, 0.2, None, None) == NULL
    assert dll.f3d_grid_rigid_override(None, 10, None, None, 0.5, None, None) == NULL
    assert dll.f3d_fiber_self_flow_up(None, None, None, 3, 32, None, None, None, None, 0, 1.0, 5e-3, 1e-5,
                                      None, None) == SHAPE
    assert dll.f3d_fiber_self_flow_up(None, None, None, 3, 32, None, None, None, None, 2, 1.0, 5e-3, 1e-5,
                                      None, None) == NULL
    # shared-memory limit of the self-flow kernel: rejected before any launch
    # (the pointers are placeholders that the check never dereferences)
    p = ctypes.c_void_p(256)
    assert dll.f3d_fiber_self_flow_up(p, p, p, 3, 1024, p, p, p, p, 2, 1.0, 5e-3, 1e-5, p, None) == TOO_LARGE


def test_argument_checks_of_surface_quadrature(dll):
    SHAPE, NULL, ALIGN, WORKSPACE = 2, 1, 3, 4
    nbytes = ctypes.c_size_t(0)
    assert dll.f3d_surface_quadrature_workspace_bytes(12000, 23996, ctypes.byref(nbytes)) == 0
    # triangles x 80 neighbours and weights dominate the workspace
    assert nbytes.value >= 23996 * 80 * (4 + 8 + 4)
    assert dll.f3d_surface_quadrature_workspace_bytes(-1, 10, ctypes.byref(nbytes)) == SHAPE
    assert dll.f3d_surface_quadrature_workspace_bytes(100, 10, None) == NULL
    # fewer nodes than the 80 neighbours, no triangles: shape errors before any launch
    assert dll.f3d_surface_quadrature(None, 79, None, 10, None, None, None, None, 0, None) == SHAPE
    assert dll.f3d_surface_quadrature(None, 400, None, 0, None, None, None, None, 0, None) == SHAPE
    assert dll.f3d_surface_quadrature(None, 400, None, 796, None, None, None, None, 0, None) == NULL
    # placeholder pointers the checks never dereference: misaligned, then a short workspace
    p8, p_odd = ctypes.c_void_p(4096), ctypes.c_void_p(4100)
    assert dll.f3d_surface_quadrature(p8, 400, p8, 796, p8, p8, None, p_odd, 1 << 30, None) == ALIGN
    assert dll.f3d_surface_quadrature(p8, 400, p8, 796, p8, p8, None, p8, 16, None) == WORKSPACE


def test_wait_limit_setting_and_selftest_checks(dll):
    """The bounded-wait limit is a host-side setting (no device needed); the
    self-test rejects a zero or over-long limit before any launch."""
    try:
        assert dll.f3d_set_wait_limit_ns(123456) == 0
        assert dll.f3d_wait_limit_ns() == 123456
    finally:
        assert dll.f3d_set_wait_limit_ns(0) == 0
    assert dll.f3d_wait_limit_ns() == 2_000_000_000
    assert dll.f3d_selftest_bounded_wait(0, None) == 5
    assert dll.f3d_selftest_bounded_wait(3_000_000_000, None) == 5


def test_pair_occupancy_argument_checks(dll):
    n = ctypes.c_int(0)
    assert dll.f3d_pair_occupancy(0, 0, 0, 0, None, None) == 1          # F3D_ERR_NULL
    assert dll.f3d_pair_occupancy(7, 0, 0, 0, None, ctypes.byref(n)) == 5  # unknown kernel
    assert dll.f3d_pair_occupancy(1, 0, 0, 1, None, ctypes.byref(n)) == 5  # dual is FP64 Oseen only


def test_autotune_candidates_fill_whole_waves():
    from fiber3d_b200 import autotune
    cands = autotune.candidates(16096, 148, occ=lambda tpt, sl: 10 if tpt == 1 else 6)
    # (tpt 2, sl 1): 256 targets per CTA, 63 target blocks, 6 x 148 = 888 slots
    splits = {c[2] for c in cands if c[:2] == (2, 1)}
    for waves in (1, 2, 3, 4):
        assert (waves * 888) // 63 in splits
    assert all(c[3] in (0, -1) for c in cands)


def test_host_entry_argument_checks(dll):
    nb = ctypes.c_size_t(0)
    assert dll.f3d_pair_host_bytes(1, 100, 50, 0, ctypes.byref(nb)) == 0 and nb.value > 0
    assert dll.f3d_pair_host_bytes(9, 100, 50, 0, ctypes.byref(nb)) == 5
    # group ids are not accepted on the host path; nothing is launched
    assert dll.f3d_pair_sum_host(0, 0, 2, None, None, None, None, None, 10, 10, 1.0, 5e-3, 1e-5,
                                 None, None, 0, None, 0, None) == 5


def test_symmetric_shape_plan_checks(dll):
    shp = _lib.PairShape(1, -1, 0, -1)
    nb = ctypes.c_size_t(0)
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 12000, ctypes.byref(shp), ctypes.byref(nb)) == 0
    assert nb.value >= 94 * 94 * 128 * 3 * 8          # T^2 partial tiles
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 4096, ctypes.byref(shp), ctypes.byref(nb)) == 2  # nt < ns
    # further targets after the sources: (T + T2) x T partial tiles
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 16096, ctypes.byref(shp), ctypes.byref(nb)) == 0
    assert nb.value >= (94 + 32) * 94 * 128 * 3 * 8
    # partial storage above 2 GiB: too large
    assert dll.f3d_pair_workspace_bytes(1, 0, 1024 * 128, 1024 * 128 + 128 * 100, ctypes.byref(shp),
                                        ctypes.byref(nb)) == 10
    assert dll.f3d_pair_workspace_bytes(1, 1, 1000, 1000, ctypes.byref(shp), ctypes.byref(nb)) == 5   # FP32C
    assert dll.f3d_pair_workspace_bytes(2, 0, 1000, 1000, ctypes.byref(shp), ctypes.byref(nb)) == 5   # rotlet
    assert dll.f3d_pair_workspace_bytes(0, 0, 1024 * 128 + 1, 1024 * 128 + 1, ctypes.byref(shp),
                                        ctypes.byref(nb)) == 10
    # 64000 fiber points onto 85600 targets (the largest time step): 1 GB of partials
    assert dll.f3d_pair_workspace_bytes(0, 0, 64000, 85600, ctypes.byref(shp), ctypes.byref(nb)) == 0
    assert nb.value >= 500 * (500 + 169) * 3072


def test_tile_shape_plan_checks(dll):
    """The tile form (sl = -2) of a source -> target sum: T x T2 partial
    tiles of 3 KB, FP64 Oseen / stresslet only, close pairs regularised
    only (checked before any memory is touched)."""
    shp = _lib.PairShape(1, -2, 0, -1)
    nb = ctypes.c_size_t(0)
    # 12000 sphere nodes onto the 4096 ball points: 94 x 32 tiles
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 4096, ctypes.byref(shp), ctypes.byref(nb)) == 0
    assert nb.value >= 94 * 32 * 128 * 3 * 8
    assert dll.f3d_pair_workspace_bytes(0, 0, 100, 100000, ctypes.byref(shp), ctypes.byref(nb)) == 0
    assert dll.f3d_pair_workspace_bytes(1, 1, 1000, 1000, ctypes.byref(shp), ctypes.byref(nb)) == 5   # FP32C
    assert dll.f3d_pair_workspace_bytes(2, 0, 1000, 1000, ctypes.byref(shp), ctypes.byref(nb)) == 5   # rotlet
    assert dll.f3d_pair_workspace_bytes(0, 0, 1024 * 128 + 1, 10, ctypes.byref(shp), ctypes.byref(nb)) == 10
    assert dll.f3d_pair_workspace_bytes(0, 0, 1024 * 128, 1024 * 128, ctypes.byref(shp),
                                        ctypes.byref(nb)) == 10                                      # > 2 GiB
    for mode in (1, 2, 3):
        assert dll.f3d_pair_sum(0, 0, mode, None, None, None, None, None, None, None, 10, 10, 1.0, 5e-3, 1e-5, 0,
                                ctypes.byref(shp), None, 0, None) == 5
    # nsplit picks 128- or 64-point source tiles: the half tiles keep twice the partials
    b1, b2 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 40960, ctypes.byref(_lib.PairShape(1, -2, 1, -1)),
                                        ctypes.byref(b1)) == 0
    assert dll.f3d_pair_workspace_bytes(1, 0, 12000, 40960, ctypes.byref(_lib.PairShape(1, -2, 2, -1)),
                                        ctypes.byref(b2)) == 0
    assert b2.value - 256 * 1024 == 2 * (b1.value - 256 * 1024) == 2 * 94 * 320 * 3072
    assert dll.f3d_pair_workspace_bytes(1, 0, 100, 100, ctypes.byref(_lib.PairShape(1, -2, 3, -1)),
                                        ctypes.byref(b1)) == 5


def test_block3_gemv_argument_checks(dll):
    """The block-Jacobi periphery preconditioner's entry checks its sizes,
    pointers and aliasing before any launch."""
    NULL, SHAPE, ARG = 1, 2, 5
    p, q = ctypes.c_void_p(256), ctypes.c_void_p(512)
    assert dll.f3d_block3_gemv(None, None, None, 0, None) == 0
    assert dll.f3d_block3_gemv(p, p, q, -1, None) == SHAPE
    assert dll.f3d_block3_gemv(None, p, q, 4, None) == NULL
    assert dll.f3d_block3_gemv(p, q, q, 4, None) == ARG


def test_shell_block_inverse_argument_checks(dll):
    NULL, SHAPE = 1, 2
    p = ctypes.c_void_p(256)
    assert dll.f3d_shell_block_inverse(None, None, None, None, 0, None, None) == 0
    assert dll.f3d_shell_block_inverse(p, p, p, p, -1, None, None) == SHAPE
    assert dll.f3d_shell_block_inverse(p, None, p, p, 4, None, None) == NULL


def test_dense_inverse_sizes_and_checks(dll):
    """Workspace of the dense inverse: a 128 x 128 pivot block, the saved
    block row (128 x ld) and one info word per 128-row step; the entry
    checks sizes, pointers, the leading dimension, alignment and the
    workspace before any CUDA call."""
    NULL, SHAPE, ALIGN, WORKSPACE = 1, 2, 3, 4
    nb = ctypes.c_size_t(0)
    assert dll.f3d_dense_inverse_workspace_bytes(300, 384, ctypes.byref(nb)) == 0
    need = nb.value
    assert need >= 128 * 128 * 8 + 128 * 384 * 8 + 3 * 4
    assert dll.f3d_dense_inverse_workspace_bytes(-1, 0, ctypes.byref(nb)) == SHAPE
    assert dll.f3d_dense_inverse_workspace_bytes(3, 128, None) == NULL
    A, ws = ctypes.c_void_p(4096), ctypes.c_void_p(8192)
    assert dll.f3d_dense_inverse(None, 0, 0, None, 0, None) == 0
    assert dll.f3d_dense_inverse(A, -3, 384, ws, need, None) == SHAPE
    assert dll.f3d_dense_inverse(None, 300, 384, ws, need, None) == NULL
    assert dll.f3d_dense_inverse(A, 300, 300, ws, need, None) == SHAPE      # ld below 384
    assert dll.f3d_dense_inverse(A, 300, 385, ws, need, None) == SHAPE      # odd ld
    assert dll.f3d_dense_inverse(ctypes.c_void_p(4104), 300, 384, ws, need, None) == ALIGN
    assert dll.f3d_dense_inverse(A, 300, 384, ws, need - 1, None) == WORKSPACE
