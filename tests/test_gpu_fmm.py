"""The GPU FMM (fiber3d_b200/fmm.py, csrc/f3d_fmm.cu) against direct sums,
the measure fiber3d's own STKFMM test uses (kernels/test_stkfmm.py:
relative L2 and L-infinity errors of the FMM against the numba direct sums
on random single- and double-layer sources and targets in a cube).

References: the C oracle (oracle/pairs_c.py) on a small case, and the
library's direct pair sums with coincident pairs excluded (exact FP64,
themselves pinned to the oracle in test_gpu_pairs.py) at larger sizes.
Tolerances per expansion order are those of kernel-independent FMMs of the
same surface grid (order 6: 1e-4 class, 8: 1e-5 to 1e-6, 10: 1e-7).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import pairs_c

pytestmark = pytest.mark.gpu

TOL = {6: 3e-4, 8: 2e-5, 10: 3e-6}


def direct(sl=None, f=None, dl=None, nrm=None, dens=None, trg=None):
    from fiber3d_b200 import kernels as K
    trg = torch.as_tensor(trg, dtype=torch.float64, device="cuda")
    u = torch.zeros(trg.numel(), dtype=torch.float64, device="cuda")
    kw = dict(self_mode="skip_close", epsilon_distance=1e-150, reg=0.0, out=u, accumulate=True)
    if sl is not None:
        K.pair_sum("oseen", torch.as_tensor(sl, device="cuda"), trg, f, **kw)
    if dl is not None:
        K.pair_sum("stresslet", torch.as_tensor(dl, device="cuda"), trg, dens, nrm, **kw)
    return u.cpu().numpy()


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def cube():
    rng = np.random.default_rng(11)
    n = 20000
    return dict(sl=rng.random((n, 3)) * 10, dl=rng.random((n, 3)) * 10, trg=rng.random((n, 3)) * 10,
                f=rng.normal(size=(n, 3)), nrm=rng.normal(size=(n, 3)), dens=rng.normal(size=(n, 3)))


@pytest.mark.parametrize("order", [6, 8, 10])
def test_cube_single_and_double_layer(cube, order):
    from fiber3d_b200 import fmm as F
    c = cube
    m = F.FMM(order=order, max_pts=200)
    m.set_points(c["sl"], c["dl"], c["trg"])
    info = m.tree_info()
    assert info["depth"] >= 3
    u = m.evaluate(sl_density=c["f"], dl_normal=c["nrm"], dl_density=c["dens"]).cpu().numpy()
    ref = direct(c["sl"], c["f"], c["dl"], c["nrm"], c["dens"], c["trg"])
    assert rel(u, ref) < TOL[order]
    # each layer alone, on their own trees
    m.set_points(c["sl"], None, c["trg"])
    u = m.evaluate(sl_density=c["f"]).cpu().numpy()
    assert rel(u, direct(c["sl"], c["f"], trg=c["trg"])) < TOL[order]
    m.set_points(None, c["dl"], c["trg"])
    u = m.evaluate(dl_normal=c["nrm"], dl_density=c["dens"]).cpu().numpy()
    assert rel(u, direct(dl=c["dl"], nrm=c["nrm"], dens=c["dens"], trg=c["trg"])) < TOL[order]


def test_deep_tree_is_deterministic(cube):
    """Small leaves (depth 4-5: several M2M and L2L levels); two evaluations
    agree bit for bit; eta divides the result."""
    from fiber3d_b200 import fmm as F
    c = cube
    m = F.FMM(order=8, max_pts=24)
    m.set_points(c["sl"], c["dl"], c["trg"])
    assert m.tree_info()["depth"] >= 4
    a = m.evaluate(sl_density=c["f"], dl_normal=c["nrm"], dl_density=c["dens"])
    b = m.evaluate(sl_density=c["f"], dl_normal=c["nrm"], dl_density=c["dens"])
    assert torch.equal(a, b)
    ref = direct(c["sl"], c["f"], c["dl"], c["nrm"], c["dens"], c["trg"])
    assert rel(a.cpu().numpy(), ref) < TOL[8]
    e = m.evaluate(sl_density=c["f"], dl_normal=c["nrm"], dl_density=c["dens"], eta=2.5)
    assert torch.allclose(e, a / 2.5, rtol=1e-15, atol=0)


def test_clustered_points_reach_the_deepest_tree():
    """Two tight clusters far apart and leaves of ~2 sources: the depth
    reaches 8 (dense slot tables of 2^24 boxes), most boxes are empty, and
    the far field passes through six levels of translations."""
    from fiber3d_b200 import fmm as F
    rng = np.random.default_rng(12)
    a = rng.normal(size=(1500, 3)) * 1e-3
    b = rng.normal(size=(1500, 3)) * 1e-3 + np.array([1.0, 0.5, -0.25])
    src = np.concatenate([a, b])
    trg = np.concatenate([a[:700] + 2e-4, b[:700] - 2e-4])
    f, nrm, dens = rng.normal(size=src.shape), rng.normal(size=src.shape), rng.normal(size=src.shape)
    m = F.FMM(order=8, max_pts=2)
    m.set_points(src, src, trg)
    assert m.tree_info()["depth"] == 8
    u = m.evaluate(sl_density=f, dl_normal=nrm, dl_density=dens).cpu().numpy()
    ref = direct(src, f, src, nrm, dens, trg)
    assert rel(u, ref) < TOL[8]


def test_against_c_oracle():
    """A small case against the C oracle directly (no pair regularised:
    epsilon 0; no coincident points)."""
    from fiber3d_b200 import fmm as F
    rng = np.random.default_rng(5)
    sl, dl, trg = rng.random((3000, 3)), rng.random((2500, 3)), rng.random((2000, 3))
    f, nrm, dens = rng.normal(size=(3000, 3)), rng.normal(size=(2500, 3)), rng.normal(size=(2500, 3))
    ref = pairs_c.pair_sum("oseen", sl, trg, f, epsilon_distance=0.0, reg=0.0)
    ref = ref + pairs_c.pair_sum("stresslet", dl, trg, dens, nrm, epsilon_distance=0.0, reg=0.0)
    m = F.FMM(order=8, max_pts=64)
    m.set_points(sl, dl, trg)
    u = m.evaluate(sl_density=f, dl_normal=nrm, dl_density=dens).cpu().numpy()
    assert rel(u, ref) < TOL[8]
    assert np.abs(u - ref).max() < 20 * TOL[8] * np.abs(ref).max()


def test_surfaces_and_fibers_targets_on_sources():
    """fiber3d's geometry: a periphery (Fibonacci sphere) of double-layer
    sources and fibers of single-layer sources, evaluated on all the points
    (targets coincide with sources: those pairs are left out, as STKFMM's
    kernels leave them out)."""
    from fiber3d_b200 import fmm as F, geometry
    rng = np.random.default_rng(2)
    shell, normals = geometry.fibonacci_sphere(12000, 10.0)
    fib = np.concatenate(geometry.perturbed_fibers(rng, 200, 32, 2.0, 5.0))
    trg = np.concatenate([fib, shell])
    f, dens = rng.normal(size=fib.shape), rng.normal(size=shell.shape)
    m = F.FMM(order=8, max_pts=300)
    m.set_points(fib, shell, trg)
    u = m.evaluate(sl_density=f, dl_normal=normals, dl_density=dens).cpu().numpy()
    ref = direct(fib, f, shell, normals, dens, trg)
    assert rel(u, ref) < TOL[8]


def test_stkfmm_module_in_the_reference_call_pattern(cube):
    """fiber3d's *_stkfmm functions with an fmm_PVel handle from the
    stkfmm-compatible module (tstep.py:120-137, kernels.py:1298-1485): numpy in
    and out, the second call on the same points reuses the tree and agrees
    bit for bit, and the combined single + double layer call equals the sum."""
    from fiber3d_b200 import kernels as K, stkfmm
    c = {k: v[:8000] for k, v in cube.items()}
    kernel = stkfmm.KERNEL.PVel
    h = stkfmm.STKFMM(8, 1000, stkfmm.PAXIS.NONE, stkfmm.KERNEL(kernel))
    assert stkfmm.getKernelDimension(h, kernel) == (4, 9, 4)
    u1 = K.oseen_kernel_source_target_stkfmm(c["sl"], c["trg"], c["f"], fmm_PVel=h)
    u2 = K.oseen_kernel_source_target_stkfmm(c["sl"], c["trg"], c["f"], fmm_PVel=h)
    assert isinstance(u1, np.ndarray) and np.array_equal(u1, u2)
    ref_sl = direct(c["sl"], c["f"], trg=c["trg"])
    assert rel(u1, ref_sl) < TOL[8]
    h2 = stkfmm.STKFMM(8, 1000, stkfmm.PAXIS.NONE, stkfmm.KERNEL(kernel))
    v = K.stresslet_kernel_source_target_stkfmm(c["dl"], c["trg"], c["nrm"], c["dens"], eta=2.0, fmm_PVel=h2)
    ref_dl = direct(dl=c["dl"], nrm=c["nrm"], dens=c["dens"], trg=c["trg"])
    assert rel(v, ref_dl / 2.0) < TOL[8]
    h3 = stkfmm.STKFMM(8, 1000, stkfmm.PAXIS.NONE, stkfmm.KERNEL(kernel))
    w = K.single_double_layer_kernel_source_target_stkfmm(c["sl"], c["dl"], c["trg"], c["nrm"], c["f"], c["dens"],
                                                          fmm_PVel=h3)
    assert rel(w, ref_sl + ref_dl) < TOL[8]
    # the module's own calls, as kernels.py makes them
    tv = np.zeros((len(c["trg"]), 4))
    lo, hi = c["trg"].min(0) - 1.0, c["trg"].max(0) + 1.0
    stkfmm.setBox(h3, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])
    stkfmm.setPoints(h3, len(c["sl"]), c["sl"], 0, np.zeros(0), len(c["trg"]), c["trg"])
    stkfmm.setupTree(h3, kernel)
    stkfmm.clearFMM(h3, kernel)
    sv = np.zeros((len(c["sl"]), 4))
    sv[:, :3] = c["f"]
    stkfmm.evaluateFMM(h3, len(c["sl"]), sv, 0, np.zeros(0), len(c["trg"]), tv, kernel)
    assert np.all(tv[:, 0] == 0.0)
    assert rel(tv[:, 1:].reshape(-1), ref_sl) < TOL[8]
    sv[0, 3] = 1.0
    with pytest.raises(NotImplementedError):
        stkfmm.evaluateFMM(h3, len(c["sl"]), sv, 0, np.zeros(0), len(c["trg"]), tv, kernel)


def test_without_handle_the_stkfmm_functions_sum_directly(cube):
    from fiber3d_b200 import kernels as K
    c = {k: v[:3000] for k, v in cube.items()}
    u = K.oseen_kernel_source_target_stkfmm(c["sl"], c["trg"], c["f"])
    assert rel(u, direct(c["sl"], c["f"], trg=c["trg"])) < 1e-13


def test_empty_sources_and_targets():
    from fiber3d_b200 import fmm as F
    rng = np.random.default_rng(0)
    m = F.FMM(order=6, max_pts=100)
    m.set_points(rng.random((100, 3)), None, rng.random((50, 3)))
    assert m.evaluate(sl_density=np.zeros((100, 3))).abs().max().item() == 0.0
    m.set_points(None, None, rng.random((50, 3)))
    assert m.evaluate().abs().max().item() == 0.0
    with pytest.raises(ValueError):
        m.set_points(rng.random((10, 3)), None, None)
