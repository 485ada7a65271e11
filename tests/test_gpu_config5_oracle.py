"""The largest time-step configuration (2000 fibers x 32 points in a ball of
radius 8, 4 rigid spheres x 400 nodes at distance 9.5, a 20000-node
periphery of radius 12: 320 824 unknowns) against the CPU oracle's
matrix-free restatement of fiber3d's step (oracle/system.py: tstep.py:
1003-1178 matvec, :745-846 right-hand side), at full size.  The periphery
takes the block-Jacobi preconditioner (ShellOperator(pc="block")), so no
dense 60000 x 60000 inverse is formed; the preconditioner changes the
iterations, not the system or its solution.

* right-hand side: 1e-12 norm-wise relative;
* A x: 1e-12 on the step's own solution (a smooth vector), 1e-10 on an
  N(0, 1) probe (the bending operator differentiates the probe's point noise
  four times, so any two FP64 evaluation orders differ there by ~1e-11);
* the mixed-precision solve to 1e-8 meets its tolerance as a true residual
  of the ORACLE's operator and right-hand side.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    from fiber3d_b200 import geometry, hydro as H
    from oracle import system as S
    torch.cuda.set_device(0)
    P = geometry.hydro_step_problem(seed=3, nfib=2000, nshell=20000, shell_radius=12.0, fiber_ball=8.0,
                                    body_shell=9.5)
    dev = H.HydroSystem(P, shell_pc="block")
    op = S.system_at(P, P.fibers)
    return dev, op


def test_sizes_and_rhs(systems):
    dev, op = systems
    assert dev.size == op.size == 320824
    assert rel_err(dev.rhs.cpu().numpy(), op.rhs) < 1e-12


def test_matvec_random_probe(systems):
    dev, op = systems
    x = np.random.default_rng(5).normal(size=op.size)
    y = torch.empty(op.size, dtype=torch.float64, device="cuda")
    dev.matvec(torch.tensor(x, device="cuda"), y)
    assert rel_err(y.cpu().numpy(), op.matvec(x)) < 1e-10


def test_solve_against_oracle_operator(systems):
    dev, op = systems
    res = dev.solve(tol=1e-8, restart=100, maxiter=600, mixed=True)
    assert res["info"] == 0
    x = res["x"]
    assert op.true_residual(x.cpu().numpy()) < 1e-8
    y = torch.empty_like(x)
    dev.matvec(x, y)
    assert rel_err(y.cpu().numpy(), op.matvec(x.cpu().numpy())) < 1e-12
