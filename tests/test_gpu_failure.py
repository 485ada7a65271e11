"""Failure detection without a GPU fault: a kernel's bounded wait runs out
(an mbarrier that nothing arrives on, no copy in flight), the kernel records
F3D_ERR_TIMEOUT in the device error word and returns; the host reads the
status, the Python layers raise, and the next sums are correct."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu

LIMIT_NS = 5000  # 5 us: the self-test wait runs out at once


def _expire(_lib):
    _lib.call("f3d_selftest_bounded_wait", LIMIT_NS, _lib.stream_handle())


def test_wait_runs_out_and_is_reported():
    from fiber3d_b200 import _lib
    torch.cuda.set_device(0)
    assert _lib.device_error() == _lib.F3D_OK
    _expire(_lib)
    torch.cuda.synchronize()  # the context is still usable
    assert _lib.device_error() == _lib.F3D_ERR_TIMEOUT
    assert _lib.device_error() == _lib.F3D_OK  # read clears it
    _expire(_lib)
    with pytest.raises(_lib.F3DError) as e:
        _lib.check_device_error("selftest")
    assert e.value.status == _lib.F3D_ERR_TIMEOUT


def test_drop_in_raises_then_next_sum_correct():
    from fiber3d_b200 import _lib, geometry, kernels
    from oracle import kernels_np as O
    torch.cuda.set_device(0)
    x, f = geometry.oseen_fiber_workload(seed=1)
    ref = O.oseen_kernel_times_density(x, f)
    _expire(_lib)
    with pytest.raises(_lib.F3DError) as e:
        kernels.oseen_kernel_times_density_numba(x, f)
    assert e.value.status == _lib.F3D_ERR_TIMEOUT
    u = kernels.oseen_kernel_times_density_numba(x, f)
    assert rel_err(u, ref) < 1e-12


def test_wait_limit_is_a_runtime_argument():
    from fiber3d_b200 import _lib, geometry, kernels
    from oracle import kernels_np as O
    torch.cuda.set_device(0)
    assert _lib.wait_limit_ns() == 2_000_000_000
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=2, n=3000, n_vol=500)
    ref = O.stresslet_kernel_source_target(nodes, vol, normals, mu)
    try:
        _lib.set_wait_limit_ns(500_000_000)  # 0.5 s: ample for every copy
        assert _lib.wait_limit_ns() == 500_000_000
        v = kernels.stresslet_kernel_source_target_numba(nodes, vol, normals, mu)
    finally:
        _lib.set_wait_limit_ns(0)
    assert _lib.wait_limit_ns() == 2_000_000_000
    assert rel_err(v, ref) < 1e-12


def test_solve_raises_then_recovers():
    from fiber3d_b200 import _lib
    from fiber3d_b200.hydro import HydroSystem
    from test_gpu_hydro import problem_from_golden
    torch.cuda.set_device(0)
    g = load_golden("step_small.npz")
    s = HydroSystem(problem_from_golden(g))
    _expire(_lib)
    with pytest.raises(_lib.F3DError):
        s.solve(tol=1e-10)
    x = s.solve(tol=1e-10)["x"].cpu().numpy()
    assert np.linalg.norm(x - g["sol"]) / np.linalg.norm(g["sol"]) < 1e-7
