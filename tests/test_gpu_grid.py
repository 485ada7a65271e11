"""Velocity field at grid points (HydroSystem.grid_velocity) against the
field fiber3d's own time step writes (tests/golden/grid_small.npz, made by
make_golden_grid.py on the step fixture's system) and against the CPU oracle
on a larger seeded system."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err
from test_gpu_hydro import problem_from_golden

pytestmark = pytest.mark.gpu


def test_grid_velocity_against_fiber3d():
    from fiber3d_b200.hydro import HydroSystem
    g = load_golden("step_small.npz")
    gg = load_golden("grid_small.npz")
    s = HydroSystem(problem_from_golden(g))
    v = s.grid_velocity(torch.tensor(gg["sol"], device="cuda"), gg["grid_points"],
                        body0_radius=float(gg["body0_radius"]))
    assert v.shape == (gg["grid_points"].shape[0], 3)
    assert rel_err(v.cpu().numpy(), gg["grid_velocity"]) < 1e-12


def test_grid_velocity_against_oracle_larger():
    """24 fibers of 32 points, one body, a 600-node periphery; grid points
    drawn near the fibers, inside the body and through the domain."""
    from fiber3d_b200 import geometry, hydro as H
    from oracle import system as S
    P = geometry.hydro_step_problem(seed=5, nfib=24, nshell=600, shell_radius=6.0, nbody=1, body_nodes=120,
                                    fiber_ball=3.0, body_shell=4.0)
    s = H.HydroSystem(P)
    rng = np.random.default_rng(11)
    sol = rng.normal(size=s.size) * 0.1
    X = np.concatenate(P.fibers)
    grid = np.concatenate([X[rng.integers(0, X.shape[0], 400)] + rng.normal(scale=0.08, size=(400, 3)),
                           np.asarray(P.bodies[0].location) + rng.normal(scale=0.25, size=(100, 3)),
                           geometry.uniform_ball(rng, 500, 5.0)])
    v = s.grid_velocity(torch.tensor(sol, device="cuda"), grid, body0_radius=0.5).cpu().numpy()
    bodies = [S.Body(np.asarray(b.location, dtype=np.float64), np.asarray(b.rotation, dtype=np.float64),
                     np.asarray(b.ref_nodes, dtype=np.float64), np.asarray(b.ref_normals, dtype=np.float64),
                     np.asarray(b.weights, dtype=np.float64)) for b in P.bodies]
    shell = S.Shell(np.asarray(P.shell.nodes), np.asarray(P.shell.normals), np.asarray(P.shell.weights))
    o = S.HydroSystem([np.asarray(f) for f in P.fibers], list(P.lengths), P.E, P.dt, P.eta, bodies, shell,
                      np.asarray(P.force_fibers).reshape(-1, 3))
    ref = o.grid_velocity(sol, grid, body0_radius=0.5)
    assert rel_err(v, ref) < 1e-12

