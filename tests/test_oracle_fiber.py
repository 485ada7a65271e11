"""Pin the oracle's fiber discretisation to fiber3d's own matrices
(fixtures from tests/golden/make_golden.py).  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_err
from oracle import fiber_ops as F

TOL = 1e-12


@pytest.mark.parametrize("N", [16, 24, 32, 48, 64])
def test_fiber_matrices(golden_fiber, N):
    g = golden_fiber
    fm = F.FiberMatrices(N)
    for k in range(4):
        assert rel_err(fm.D0[k], g[f"fm{N}_D{k + 1}"]) < TOL, f"D{k + 1}"
    assert rel_err(fm.PX, g[f"fm{N}_PX"]) < TOL
    assert rel_err(fm.PT, g[f"fm{N}_PT"]) < TOL
    assert rel_err(fm.Pcheb, g[f"fm{N}_Pcheb"]) < TOL
    assert rel_err(fm.weights0, g[f"fm{N}_w"]) < TOL


@pytest.mark.parametrize("c", [0, 1])
def test_fiber_operator_rhs_bc(golden_fiber, c):
    g = golden_fiber
    N, L, E, dt = int(g[f"fib{c}_N"]), float(g[f"fib{c}_L"]), float(g[f"fib{c}_E"]), float(g[f"fib{c}_dt"])
    bc = tuple(str(s) for s in g[f"fib{c}_bc"])
    x, flow, force = g[f"fib{c}_x"], g[f"fib{c}_flow"], g[f"fib{c}_force"]
    fm = F.FiberMatrices(N)
    c0, c1 = F.mobility_constants(1e-3, 1.0)
    assert abs(c0 - g[f"fib{c}_c0"]) < 1e-15 and abs(c1 - g[f"fib{c}_c1"]) < 1e-15
    A = F.linear_operator(fm, x, L, E, dt, c0, c1)
    assert rel_err(A, g[f"fib{c}_A"]) < TOL
    R = F.rhs(fm, x, L, dt, c0, c1, force=force, flow=flow)
    assert rel_err(R, g[f"fib{c}_RHS"]) < TOL
    B, r = F.bc_rows(fm, x, L, E, dt, c0, bc, end_vec0=force[-1] if bc[2] == "force" else None,
                     v_on_fiber=flow, force_on_fiber=force)
    AA, RR = F.apply_bc_rectangular(fm, A, R, B, r)
    assert rel_err(AA, g[f"fib{c}_Abc"]) < TOL
    assert rel_err(RR, g[f"fib{c}_RHSbc"]) < TOL
    assert rel_err(F.force_operator(fm, x, L, E), g[f"fib{c}_Fop"]) < TOL
