"""The rest of fiber3d's kernels.kernels module on the GPU, against
tests/golden/dropin.npz (fiber3d's own functions; make_golden_dropin.py):
traction, the 3-index stresslet, the numpy stresslet times normal, and the
PyCUDA / STKFMM entry points (direct sums with their pair semantics)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def K():
    torch.cuda.set_device(0)
    from fiber3d_b200 import kernels
    return kernels


@pytest.fixture(scope="module")
def g():
    return load_golden("dropin.npz")


def test_traction(K, g):
    v = K.traction_kernel_times_normal_times_density_numba(g["traction_r"], g["traction_n"], g["traction_d"])
    assert rel_err(v, g["traction_v"]) < TOL
    v = K.traction_kernel_times_normal_times_density_numba(g["traction_r"], g["traction_n"], g["traction_d"],
                                                           2.5, 1e-2, 1e-4)
    assert rel_err(v, g["traction_v_eta"]) < TOL


def test_traction_fp32c(K, g):
    v = K.traction_kernel_times_normal_times_density_numba(g["traction_r"], g["traction_n"], g["traction_d"],
                                                           precision="fp32c")
    assert rel_err(v, g["traction_v"]) < 2e-6


def test_traction_large_against_oracle(K):
    """Several tiles and splits; device tensors in, device tensor out."""
    from fiber3d_b200 import geometry
    from oracle import kernels_np as O
    rng = np.random.default_rng(8)
    x = rng.random((2100, 3)) * 4
    n = geometry.uniform_directions(rng, 2100)
    d = rng.normal(size=(2100, 3))
    ref = O.traction_kernel_times_normal_times_density(x, n, d)
    t = lambda a: torch.as_tensor(a, device="cuda")
    v = K.traction_kernel_times_normal_times_density_numba(t(x), t(n), t(d))
    assert v.is_cuda
    assert rel_err(v.cpu().numpy(), ref) < TOL


def test_stresslet_tensor(K, g):
    assert rel_err(K.stresslet_kernel(g["stk_r"]), g["stk_S"]) < TOL
    assert rel_err(K.stresslet_kernel(g["stk_r"].T.flatten(), input_format='xyz'), g["stk_S_xyz"]) < TOL
    assert rel_err(K.stresslet_kernel(g["stk_r"], 3.0, 1e-2, 1e-4), g["stk_S_eta"]) < TOL
    assert K.stresslet_kernel(g["stk_r"]).shape == g["stk_S"].shape


def test_stresslet_times_normal_numpy_form(K, g):
    assert rel_err(K.stresslet_kernel_times_normal(g["stkn_r"], g["stkn_n"]), g["stkn_M"]) < TOL


def test_pycuda_oseen(K, g):
    u = K.oseen_kernel_source_target_pycuda(g["pyc_rs"], g["pyc_rt"], g["pyc_f"])
    assert rel_err(u, g["pyc_u"]) < TOL


def test_stkfmm_stand_ins(K, g):
    u = K.oseen_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rt"], g["fmm_f"], fmm_PVel=object())
    assert rel_err(u, g["fmm_oseen_u"]) < TOL
    u = K.oseen_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rt"], g["fmm_f"], 2.0, fmm_PVel=None)
    assert rel_err(u, g["fmm_eta_u"]) < TOL
    v = K.stresslet_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rt"], g["fmm_n"], g["fmm_d"], fmm_PVel=None)
    assert rel_err(v, g["fmm_stresslet_v"]) < TOL
    w = K.single_double_layer_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rdl"], g["fmm_rt"], g["fmm_ndl"],
                                                          g["fmm_f"], g["fmm_ddl"], fmm_PVel=None)
    assert rel_err(w, g["fmm_sdl_u"]) < TOL


def test_stkfmm_functions_on_the_gpu_fmm(K, g):
    """With this package's stkfmm handle the same functions run the GPU FMM:
    against fiber3d's own direct sums (the values STKFMM is checked
    against), to the FMM's order-10 accuracy."""
    from fiber3d_b200 import stkfmm
    mk = lambda: stkfmm.STKFMM(10, 64, stkfmm.PAXIS.NONE, stkfmm.KERNEL(stkfmm.KERNEL.PVel))
    u = K.oseen_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rt"], g["fmm_f"], fmm_PVel=mk())
    assert rel_err(u, g["fmm_oseen_u"]) < 1e-6
    u = K.oseen_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rt"], g["fmm_f"], 2.0, fmm_PVel=mk())
    assert rel_err(u, g["fmm_eta_u"]) < 1e-6
    v = K.stresslet_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rt"], g["fmm_n"], g["fmm_d"], fmm_PVel=mk())
    assert rel_err(v, g["fmm_stresslet_v"]) < 1e-6
    w = K.single_double_layer_kernel_source_target_stkfmm(g["fmm_rs"], g["fmm_rdl"], g["fmm_rt"], g["fmm_ndl"],
                                                          g["fmm_f"], g["fmm_ddl"], fmm_PVel=mk())
    assert rel_err(w, g["fmm_sdl_u"]) < 1e-6


def test_skip_close_fp32c_drops_coincident_pairs(K, g):
    from fiber3d_b200 import kernels
    u = kernels.pair_sum("oseen", torch.as_tensor(g["fmm_rs"], device="cuda"),
                         torch.as_tensor(g["fmm_rt"], device="cuda"), torch.as_tensor(g["fmm_f"], device="cuda"),
                         self_mode="skip_close", epsilon_distance=kernels.COINCIDENT, precision="fp32c")
    u = u.cpu().numpy()
    assert np.isfinite(u).all()
    assert rel_err(u, g["fmm_oseen_u"]) < 2e-6
