"""The solver-level drop-in (fiber3d_b200.tstep_bridge): given a time
stepper's state and fiber3d's own right-hand side b, the GPU solve returns
fiber3d's solution of the step (tests/golden/step_small.npz: 6 fibers,
2 rigid spheres, a 240-node periphery).  The time stepper is a stand-in with
the attributes the bridge reads from fiber3d's ``tstep`` object."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu


def fake_tstep(g):
    from fiber3d_b200 import hydro as H
    npts = [int(n) for n in g["npts"]]
    fibers = [SimpleNamespace(x=g[f"fib{k}_x"], length=float(g["L"]), E=float(g["E"]), epsilon=1e-3,
                              penalty_param=500.0) for k in range(len(npts))]
    bodies = []
    k = 0
    while f"body{k}_loc" in g:
        R = H.quaternion_rotation(g[f"body{k}_quat"])
        bodies.append(SimpleNamespace(location=g[f"body{k}_loc"],
                                      orientation=SimpleNamespace(rotation_matrix=lambda R=R: R),
                                      reference_configuration=g[f"body{k}_ref_nodes"],
                                      reference_normals=g[f"body{k}_ref_normals"],
                                      quadrature_weights=g[f"body{k}_w"]))
        k += 1
    return SimpleNamespace(fibers=fibers, bodies=bodies, shell=SimpleNamespace(quadrature_weights=g["shell_w"]),
                           trg_shell_surf=g["shell_nodes"], normals_shell=g["shell_normals"],
                           dt=float(g["dt"]), eta=float(g["eta"]))


@pytest.mark.parametrize("mixed", [False, True])
def test_bridge_solves_fibers3d_step(mixed):
    from fiber3d_b200.tstep_bridge import GpuGmres
    g = load_golden("step_small.npz")
    solver = GpuGmres(fake_tstep(g), mixed=mixed)
    tol = float(g["tol"])
    x, info = solver(None, g["rhs"], tol=tol)
    assert info == 0
    assert x.shape == g["sol"].shape
    assert rel_err(x, g["sol"]) < 1e-7
    # the periphery preconditioner is built once and reused by later calls
    shell = solver._shell
    x2, info2 = solver(None, g["rhs"], tol=tol)
    assert solver._shell is shell and info2 == 0
    assert np.array_equal(x, x2)


@pytest.mark.parametrize("mixed", [False, True])
def test_bridge_warm_start(mixed):
    """With warm_start="extrapolate" a repeated call on the same system starts
    from the previous solution: no more iterations than the first call, and
    the same answer to the tolerance."""
    from fiber3d_b200.tstep_bridge import GpuGmres
    g = load_golden("step_small.npz")
    solver = GpuGmres(fake_tstep(g), mixed=mixed, warm_start="extrapolate")
    tol = float(g["tol"])
    x1, info1 = solver(None, g["rhs"], tol=tol)
    its1 = solver.last["iterations"]
    x2, info2 = solver(None, g["rhs"], tol=tol)
    assert info1 == 0 and info2 == 0
    assert solver.last["iterations"] <= its1
    assert rel_err(x2, g["sol"]) < 1e-7
    with pytest.raises(ValueError):
        GpuGmres(fake_tstep(g), warm_start="learned")


def test_bridge_learned_warm_start():
    """warm_start="learned" takes a LearnedWarmStart; on systems it does not
    apply to (fibers of other resolutions) it is the extrapolation, and the
    answer meets fiber3d's tolerance either way."""
    from fiber3d_b200.tstep_bridge import GpuGmres
    from fiber3d_b200.warmstart import LearnedWarmStart
    g = load_golden("step_small.npz")
    solver = GpuGmres(fake_tstep(g), mixed=True, warm_start="learned", model=LearnedWarmStart(seed=0))
    tol = float(g["tol"])
    for _ in range(5):
        x, info = solver(None, g["rhs"], tol=tol)
        assert info == 0 and rel_err(x, g["sol"]) < 1e-7
    assert len(solver._history) == 4
