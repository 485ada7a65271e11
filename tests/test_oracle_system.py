"""Pin the oracle's linear system of one hydrodynamic step to fiber3d's own
time step (tests/golden/make_golden_step.py: 6 fibers of 16/24/32 points,
2 rigid spheres of 80 nodes, a 240-node periphery).  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden, rel_err
from oracle import system as S


def build_from_golden(g) -> S.HydroSystem:
    npts = [int(n) for n in g["npts"]]
    fibers = [g[f"fib{k}_x"] for k in range(len(npts))]
    ff = np.concatenate([np.tile(g["fext"][k], (npts[k], 1)) for k in range(len(npts))])
    bodies = []
    k = 0
    while f"body{k}_loc" in g:
        bodies.append(S.Body(g[f"body{k}_loc"], S.quaternion_rotation(g[f"body{k}_quat"]),
                             g[f"body{k}_ref_nodes"], g[f"body{k}_ref_normals"], g[f"body{k}_w"]))
        k += 1
    shell = S.Shell(g["shell_nodes"].reshape(-1, 3), g["shell_normals"].reshape(-1, 3), g["shell_w"])
    return S.HydroSystem(fibers, [float(g["L"])] * len(npts), float(g["E"]), float(g["dt"]),
                         float(g["eta"]), bodies, shell, ff)


@pytest.fixture(scope="module")
def step():
    g = load_golden("step_small.npz")
    return g, build_from_golden(g)


def test_layout_and_rhs(step):
    g, sys_ = step
    assert sys_.size == g["rhs"].size
    assert rel_err(sys_.rhs, g["rhs"]) < 1e-12


def test_matvec(step):
    g, sys_ = step
    for x, ax in zip(g["probe_x"], g["probe_Ax"]):
        assert rel_err(sys_.matvec(x), ax) < 1e-12


def test_preconditioner(step):
    g, sys_ = step
    for x, px in zip(g["probe_x"], g["probe_Px"]):
        assert rel_err(sys_.pc(x), px) < 1e-10


def test_solve(step):
    g, sys_ = step
    sol, info, its = sys_.solve(tol=float(g["tol"]))
    assert info == 0
    res = np.linalg.norm(sys_.matvec(sol) - sys_.rhs) / np.linalg.norm(sys_.rhs)
    assert res < 1e-9
    assert rel_err(sol, g["sol"]) < 1e-7


def test_grid_velocity_against_fiber3d():
    """The oracle's grid velocity against the field fiber3d's own time step
    writes (tests/golden/make_golden_grid.py): every kept grid point, the
    near-fiber and inside-body ones included."""
    g = load_golden("step_small.npz")
    gg = load_golden("grid_small.npz")
    sys_ = build_from_golden(g)
    v = sys_.grid_velocity(gg["sol"], gg["grid_points"], body0_radius=float(gg["body0_radius"]))
    assert rel_err(v, gg["grid_velocity"]) < 1e-12


def test_reference_grid():
    """geometry.ellipsoid_grid is fiber3d's grid (tstep.py:1240-1270): the
    fixture's kept points at their indices."""
    from fiber3d_b200 import geometry
    gg = load_golden("grid_small.npz")
    g = geometry.ellipsoid_grid()
    assert g.shape[0] == int(gg["grid_count"])
    assert np.array_equal(g[gg["grid_index"]], gg["grid_points"])


def test_shell_block_pc_is_the_dense_operators_diagonal(step):
    """The block-Jacobi periphery preconditioner inverts exactly the 3 x 3
    diagonal blocks of the dense shell operator (pinned above through the
    preconditioner probes)."""
    _, sys_ = step
    M = sys_.M_shell
    n = sys_.nshell
    x = np.random.default_rng(0).normal(size=3 * n)
    ref = np.concatenate([np.linalg.solve(M[3 * i:3 * i + 3, 3 * i:3 * i + 3], x[3 * i:3 * i + 3])
                          for i in range(n)])
    assert rel_err(sys_.shell_block_pc(x), ref) < 1e-13
