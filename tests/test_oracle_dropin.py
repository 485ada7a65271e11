"""Pin the oracle's restatements of the remaining kernels.kernels functions
(traction, the 3-index stresslet, the numpy stresslet times normal, the
PyCUDA and STKFMM semantics) to tests/golden/dropin.npz, which fiber3d's own
functions produced (make_golden_dropin.py).  No GPU needed."""
from __future__ import annotations

from conftest import load_golden, rel_err
from oracle import kernels_np as O

TOL = 1e-12


def test_traction():
    g = load_golden("dropin.npz")
    assert rel_err(O.traction_kernel_times_normal_times_density(g["traction_r"], g["traction_n"],
                                                                g["traction_d"]), g["traction_v"]) < TOL
    assert rel_err(O.traction_kernel_times_normal_times_density(g["traction_r"], g["traction_n"], g["traction_d"],
                                                                2.5, 1e-2, 1e-4), g["traction_v_eta"]) < TOL


def test_stresslet_tensor():
    g = load_golden("dropin.npz")
    assert rel_err(O.stresslet_kernel(g["stk_r"]), g["stk_S"]) < TOL
    assert rel_err(O.stresslet_kernel(g["stk_r"].T.flatten(), input_format='xyz'), g["stk_S_xyz"]) < TOL
    assert rel_err(O.stresslet_kernel(g["stk_r"], 3.0, 1e-2, 1e-4), g["stk_S_eta"]) < TOL


def test_stresslet_times_normal_numpy_form():
    g = load_golden("dropin.npz")
    assert rel_err(O.stresslet_kernel_times_normal_dense(g["stkn_r"], g["stkn_n"]), g["stkn_M"]) < TOL


def test_pycuda_and_stkfmm_semantics():
    g = load_golden("dropin.npz")
    assert rel_err(O.oseen_kernel_source_target_skip_close(g["pyc_rs"], g["pyc_rt"], g["pyc_f"]), g["pyc_u"]) < TOL
    u = O.oseen_kernel_source_target_skip_close(g["fmm_rs"], g["fmm_rt"], g["fmm_f"], epsilon_distance=1e-150)
    assert rel_err(u, g["fmm_oseen_u"]) < TOL
    v = O.stresslet_kernel_source_target_skip_close(g["fmm_rs"], g["fmm_rt"], g["fmm_n"], g["fmm_d"])
    assert rel_err(v, g["fmm_stresslet_v"]) < TOL
    w = O.stresslet_kernel_source_target_skip_close(g["fmm_rdl"], g["fmm_rt"], g["fmm_ndl"], g["fmm_ddl"])
    assert rel_err(u + w, g["fmm_sdl_u"]) < TOL
    u2 = O.oseen_kernel_source_target_skip_close(g["fmm_rs"], g["fmm_rt"], g["fmm_f"], eta=2.0,
                                                 epsilon_distance=1e-150)
    assert rel_err(u2, g["fmm_eta_u"]) < TOL
