"""Pin the CPU oracle to golden vectors produced by fiber3d's own code.

These run without a GPU.  Tolerance 1e-12 norm-wise relative (the reference
numba kernels use fastmath, which allows reassociation).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import kernels_np as O
from oracle import pairs_c
from fiber3d_b200 import geometry
from conftest import rel_err

TOL = 1e-12


@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
def test_oseen_source_target(golden_kernels, tag):
    g = golden_kernels
    u = O.oseen_kernel_source_target(g[f"ost_{tag}_rs"], g[f"ost_{tag}_rt"], g[f"ost_{tag}_f"])
    assert rel_err(u, g[f"ost_{tag}_u"]) < TOL


def test_oseen_params(golden_kernels):
    g = golden_kernels
    u = O.oseen_kernel_source_target(g["ostp_rs"], g["ostp_rt"], g["ostp_f"], 2.5, 1e-2, 1e-4)
    assert rel_err(u, g["ostp_u"]) < TOL


def test_oseen_times_density(golden_kernels):
    g = golden_kernels
    assert rel_err(O.oseen_kernel_times_density(g["otd_r"], g["otd_f"]), g["otd_u"]) < TOL


def test_rotlet(golden_kernels):
    g = golden_kernels
    assert rel_err(O.rotlet_kernel_source_target(g["rot_rs"], g["rot_rt"], g["rot_t"]), g["rot_u"]) < TOL


def test_stresslet_source_target(golden_kernels):
    g = golden_kernels
    v = O.stresslet_kernel_source_target(g["sst_rs"], g["sst_rt"], g["sst_n"], g["sst_d"])
    assert rel_err(v, g["sst_v"]) < TOL


def test_stresslet_times_density(golden_kernels):
    g = golden_kernels
    assert rel_err(O.stresslet_kernel_times_normal_times_density(g["stnd_r"], g["stnd_n"], g["stnd_d"]),
                   g["stnd_v"]) < TOL
    assert rel_err(O.stresslet_kernel_times_normal_times_density(g["stnd_r"], g["stnd_n"], g["stnd_d"], 3.0),
                   g["stnd_v_eta"]) < TOL


def test_dense_operators(golden_kernels):
    g = golden_kernels
    assert rel_err(O.stresslet_kernel_times_normal_dense(g["stn_r"], g["stn_n"]), g["stn_M"]) < TOL
    assert rel_err(O.oseen_tensor(g["ot_r"]), g["ot_G"]) < TOL
    assert rel_err(O.oseen_tensor(g["ot_r"].T.flatten(), input_format='xyz'), g["ot_Gxyz"]) < TOL
    assert rel_err(O.oseen_tensor_source_target(g["otst_rs"], g["otst_rt"]), g["otst_G"]) < TOL
    assert rel_err(O.complementary_kernel(None, g["comp_n"]), g["comp_C"]) < TOL
    assert rel_err(O.complementary_kernel_times_density(None, g["comp_n"], g["compd_d"]), g["compd_u"]) < TOL


def test_config1(golden_config1):
    g = golden_config1
    x, f = geometry.oseen_fiber_workload(seed=1)
    np.testing.assert_array_equal(x, g["x"])
    np.testing.assert_array_equal(f, g["f"])
    assert rel_err(O.oseen_kernel_times_density(x, f), g["u"]) < TOL


@pytest.mark.parametrize("n", [100, 101, 600])
def test_fibonacci_sphere_matches_shape_gallery(golden_sphere, n):
    nodes, normals = geometry.fibonacci_sphere(n, 10.0)
    np.testing.assert_allclose(nodes, golden_sphere[f"nodes_{n}"], rtol=0, atol=1e-13)
    ok = np.isfinite(golden_sphere[f"normals_{n}"]).all(axis=1)
    np.testing.assert_allclose(normals[ok], golden_sphere[f"normals_{n}"][ok], rtol=0, atol=1e-15)


# ---- C/OpenMP restatement (the timed CPU baseline) -------------------------
def test_c_oracle_matches_golden(golden_kernels, golden_config1):
    g = golden_kernels
    for tag in "abcd":
        u = pairs_c.pair_sum("oseen", g[f"ost_{tag}_rs"], g[f"ost_{tag}_rt"], g[f"ost_{tag}_f"])
        assert rel_err(u, g[f"ost_{tag}_u"]) < TOL
    u = pairs_c.pair_sum("oseen", g["otd_r"], g["otd_r"], g["otd_f"], self_mode="skip_index")
    assert rel_err(u, g["otd_u"]) < TOL
    u = pairs_c.pair_sum("rotlet", g["rot_rs"], g["rot_rt"], g["rot_t"])
    assert rel_err(u, g["rot_u"]) < TOL
    v = pairs_c.pair_sum("stresslet", g["sst_rs"], g["sst_rt"], g["sst_d"], g["sst_n"])
    assert rel_err(v, g["sst_v"]) < TOL
    v = pairs_c.pair_sum("stresslet", g["stnd_r"], g["stnd_r"], g["stnd_d"], g["stnd_n"],
                         self_mode="skip_index")
    assert rel_err(v, g["stnd_v"]) < TOL
    c = golden_config1
    u = pairs_c.pair_sum("oseen", c["x"], c["x"], c["f"], self_mode="skip_index")
    assert rel_err(u, c["u"]) < TOL


def test_group_skip_equals_reference_order():
    """Skipping same-fiber pairs equals the reference's add-all-then-subtract
    order (flow_fibers then self_flow_fibers with dense per-fiber Oseen
    blocks, tstep_utils.py:653-727, 812-851) up to cancellation rounding."""
    rng = np.random.default_rng(5)
    fibs = geometry.perturbed_fibers(rng, 6, 16, 1.0, 2.0)
    x = np.concatenate(fibs)
    grp = np.repeat(np.arange(6), 16)
    f = rng.normal(size=x.shape)
    fused = O.oseen_kernel_source_target(x, x, f, src_group=grp, trg_group=grp)
    full = O.oseen_kernel_source_target(x, x, f)
    for k in range(6):
        sl = slice(16 * k, 16 * (k + 1))
        full[3 * sl.start:3 * sl.stop] -= O.oseen_tensor(x[sl]) @ f[sl].reshape(-1)
    assert rel_err(fused, full) < 1e-12
    c = pairs_c.pair_sum("oseen", x, x, f, self_mode="skip_group", src_group=grp, trg_group=grp)
    assert rel_err(c, fused) < 1e-13
