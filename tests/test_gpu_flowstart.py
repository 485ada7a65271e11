"""The (positions, background velocity) -> (tensions, force densities)
warm start on a small marched system: training pairs from the solver's
own steps, the network's kernels train on them, and GMRES converges to
the same tolerance from its guess."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _system(seed):
    from fiber3d_b200 import geometry, hydro as H
    P = geometry.hydro_step_problem(seed=seed, nfib=24, nbody=1, body_nodes=100, nshell=400, shell_radius=6.0,
                                    fiber_ball=3.0, body_shell=4.5)
    return H.HydroSystem(P)


def test_flow_warm_start_trains_and_converges():
    from fiber3d_b200 import flowstart as FS
    torch.cuda.set_device(0)
    stats, X, Y = FS.march(_system(21), 10, guess="extrapolate", record=True, tol=1e-10, record_from=2)
    assert X.shape == (8 * 24, 192) and Y.shape == (8 * 24, 128)
    assert torch.isfinite(X).all() and torch.isfinite(Y).all()
    net = FS.FlowWarmStart(seed=0)
    hist, val = net.fit(X, Y, epochs=3, batch=64)
    assert np.isfinite(hist).all() and np.isfinite(val["tension"]) and np.isfinite(val["force"])
    st = FS.march(_system(22), 6, guess="flow", net=net, tol=1e-8, oracle_steps=2, record_from=2)
    assert len(st) == 6 and all(np.isfinite(s["initial_rel_residual"]) for s in st)
    assert all(s["iterations"] < 100 for s in st)
    maps = [s["oracle_map_rel_residual"] for s in st if "oracle_map_rel_residual" in s]
    assert len(maps) == 2 and all(np.isfinite(maps))


def test_background_velocity_is_the_matvec_flow():
    """u_bg at the fiber points equals the flow the FP64 matvec sums there
    (plus the external forces' flow), to FP32C accuracy."""
    from fiber3d_b200 import flowstart as FS
    s = _system(23)
    x = s.solve(tol=1e-10)["x"]
    u32 = FS.background_velocity(s, x, precision="fp32c")
    u64 = FS.background_velocity(s, x, precision="fp64")
    assert float((u32 - u64).abs().max() / u64.abs().max()) < 1e-5
