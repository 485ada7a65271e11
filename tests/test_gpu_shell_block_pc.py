"""The block-Jacobi periphery preconditioner (ShellOperator(pc="block")):
the inverses of the 3 x 3 diagonal blocks of fiber3d's dense shell operator
(tstep.py:327-347) instead of its LU (tstep.py:348).

* f3d_block3_gemv applied to N(0, 1) vectors: 1e-13 against the oracle's
  block solves (oracle/system.py shell_block_pc), itself pinned to the dense
  operator's diagonal blocks on CPU;
* a step solved with it meets its tolerance as the oracle's true residual
  (FP64 and mixed), and solved to 1e-12 it gives the dense inverse's
  solution to 1e-8;
* its GMRES needs more iterations than the dense inverse (the periphery's
  nonlocal coupling is left to GMRES) but no O(N^2) memory.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from fiber3d_b200 import geometry, hydro as H
    from oracle import system as S
    torch.cuda.set_device(0)
    P = geometry.hydro_step_problem(seed=5, nfib=64, nshell=3000, shell_radius=10.0)
    blk = H.HydroSystem(P, shell_pc="block")
    dense = H.HydroSystem(P)
    op = S.system_at(P, P.fibers)
    return P, blk, dense, op


def test_block_inverse_has_no_dense_copy(setup):
    _, blk, _, _ = setup
    sh = blk.shell
    assert sh.pc == "block" and sh.inv64 is None and sh.inv32 is None and sh.inv16 is None
    assert tuple(sh.block_inv.shape) == (sh.n, 9)


@pytest.mark.parametrize("seed", [0, 1])
def test_apply_against_oracle(setup, seed):
    _, blk, _, op = setup
    ns = 3 * op.nshell
    x = np.random.default_rng(seed).normal(size=ns)
    y = torch.empty(ns, dtype=torch.float64, device="cuda")
    for storage in ("fp64", "fp32", "fp16"):
        blk.shell.apply(torch.tensor(x, device="cuda"), y, storage)
        assert rel_err(y.cpu().numpy(), op.shell_block_pc(x)) < 1e-13


def test_pc_keeps_the_other_blocks(setup):
    _, blk, dense, op = setup
    x = torch.tensor(np.random.default_rng(7).normal(size=op.size), device="cuda")
    yb, yd = torch.empty_like(x), torch.empty_like(x)
    blk.pc(x, yb)
    dense.pc(x, yd)
    ns = 3 * op.nshell
    assert torch.equal(yb[ns:], yd[ns:])


@pytest.mark.parametrize("mixed,tol", [(False, 1e-8), (True, 1e-9)])
def test_solve_meets_the_oracle_residual(setup, mixed, tol):
    _, blk, dense, op = setup
    rb = blk.solve(tol=tol, restart=100, maxiter=400, mixed=mixed)
    assert rb["info"] == 0
    assert op.true_residual(rb["x"].cpu().numpy()) < tol
    rd = dense.solve(tol=tol, restart=100, mixed=mixed)
    assert rb["iterations"] >= rd["iterations"]


def test_tight_solutions_agree(setup):
    """Both preconditioners solve the same system: to 1e-12 their solutions
    agree to the operator's conditioning times that residual.  (At 1e-8 each
    solution is only within ~kappa * 1e-8 ~ 1e-6 of the exact one, in
    directions that depend on the preconditioner.)"""
    _, blk, dense, op = setup
    xb = blk.solve(tol=1e-12, restart=100, maxiter=600)["x"].cpu().numpy()
    xr = dense.solve(tol=1e-12, restart=100)["x"].cpu().numpy()
    assert np.linalg.norm(xb - xr) / np.linalg.norm(xr) < 1e-8


def test_bad_option():
    from fiber3d_b200 import geometry, hydro as H
    P = geometry.hydro_step_problem(seed=5, nfib=4, nshell=200, shell_radius=10.0, nbody=0)
    with pytest.raises(ValueError):
        H.ShellOperator(P.shell, pc="lu")


def test_singular_blocks_are_counted():
    """A block made exactly singular (E_i = -I and n_i = e_z give
    B_i = diag(0, 0, 1) in any rounding) is counted in info; the others are
    the inverses numpy finds."""
    from fiber3d_b200 import _lib
    rng = np.random.default_rng(3)
    n = 5
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    w = rng.uniform(0.05, 0.2, n)
    E = rng.normal(size=(n, 3, 3)) * 0.1 - 0.5 * np.eye(3)
    E[2] = -np.eye(3)
    nrm[2] = [0.0, 0.0, 1.0]
    # device copies held for the call (a temporary freed right after its
    # pointer is taken could be handed to the next copy before the kernel runs)
    dE, dw, dn = (torch.as_tensor(np.ascontiguousarray(a), device="cuda") for a in (E.reshape(n, 9), w, nrm))
    out = torch.empty((n, 9), dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("f3d_shell_block_inverse", _lib.ptr(dE), _lib.ptr(dw), _lib.ptr(dn),
              _lib.ptr(out), n, _lib.ptr(info), _lib.stream_handle(torch.device("cuda")))
    assert int(info.item()) == 1
    B = -(E + np.eye(3)) / w[:, None, None] + nrm[:, :, None] * nrm[:, None, :]
    got = out.cpu().numpy().reshape(n, 3, 3)
    for i in (0, 1, 3, 4):
        ref = np.linalg.inv(B[i])
        assert np.abs(got[i] - ref).max() < 1e-13 * np.abs(ref).max()
