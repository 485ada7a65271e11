"""GPU batched LU (uneven block sizes, one persistent launch) against
scipy.linalg.lu_factor / lu_solve — the calls fiber3d's block
preconditioner makes per block (tstep_utils.py:1341-1419, tstep.py:950-994)."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg as sla
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu


def random_blocks(rng, sizes):
    out = []
    for n in sizes:
        A = rng.normal(size=(n, n))
        A += np.diag(rng.uniform(0.5, 2.0, n) * np.sign(rng.normal(size=n)))  # mildly conditioned
        out.append(A)
    return out


@pytest.mark.parametrize("sizes", [[64, 96, 128, 192, 256] * 3, [1, 2, 3, 31, 33, 65], [1206, 64, 1206]])
def test_factor_and_solve_match_scipy(sizes):
    from fiber3d_b200.blocklu import BlockLU
    rng = np.random.default_rng(len(sizes))
    blocks = random_blocks(rng, sizes)
    lu = BlockLU(sizes)
    lu.load(blocks)
    lu.factor()
    lu.check()
    rhs = rng.normal(size=sum(sizes))
    x = lu.solve(torch.tensor(rhs, device="cuda")).cpu().numpy()
    off = 0
    for A, n in zip(blocks, sizes):
        xr = sla.lu_solve(sla.lu_factor(A), rhs[off:off + n])
        assert rel_err(x[off:off + n], xr) < 1e-10
        off += n
    # factors and pivots equal LAPACK's up to rounding
    for b, (A, n) in enumerate(zip(blocks, sizes)):
        ref_lu, ref_piv = sla.lu_factor(A)
        assert np.array_equal(lu.piv[lu.voff_h[b]:lu.voff_h[b] + n].cpu().numpy(), ref_piv)
        assert rel_err(lu.block(b).cpu().numpy(), ref_lu) < 1e-11


def test_queue_counters_reset_between_calls():
    from fiber3d_b200.blocklu import BlockLU
    rng = np.random.default_rng(1)
    sizes = [96] * 50
    lu = BlockLU(sizes)
    blocks = random_blocks(rng, sizes)
    for _ in range(3):
        lu.load(blocks)
        lu.factor()
        x = lu.solve(torch.ones(sum(sizes), dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    assert int(lu.ws[:16].view(torch.int32).abs().sum()) == 0
    ref = np.concatenate([np.linalg.solve(A, np.ones(96)) for A in blocks])
    assert rel_err(x.cpu().numpy(), ref) < 1e-10


def test_zero_pivot_reported():
    from fiber3d_b200.blocklu import BlockLU
    A = np.eye(8)
    A[3, 3] = 0.0
    A[3, :] = 0.0
    lu = BlockLU([8, 8])
    lu.load([np.eye(8), A])
    lu.factor()
    with pytest.raises(ZeroDivisionError):
        lu.check()


def test_fiber_blocks_of_reference_step():
    """The fiber blocks of fiber3d's step (oracle-assembled) through the GPU
    LU give fiber3d's preconditioner output on those rows."""
    from fiber3d_b200.blocklu import BlockLU
    from test_oracle_system import build_from_golden
    g = load_golden("step_small.npz")
    sys_ = build_from_golden(g)
    sizes = [A.shape[0] for A in sys_.A_fib]
    lu = BlockLU(sizes)
    lu.load(sys_.A_fib)
    lu.factor()
    lu.check()
    o = sys_.o_fib
    for x, px in zip(g["probe_x"], g["probe_Px"]):
        y = lu.solve(torch.tensor(x[o:], device="cuda")).cpu().numpy()
        assert rel_err(y, px[o:]) < 1e-10


@pytest.mark.parametrize("sizes", [[128] * 40, [4, 16, 33, 64, 100, 128, 7], [32, 1, 32, 17], [128] * 512])
def test_inverse_and_block_gemv_match_numpy(sizes):
    """Blocks of at most 32 rows take the register-tiled kernel, 33-128 the
    blocked tensor-core one; 512 blocks of 128 are the 512-fiber step's."""
    from fiber3d_b200.blocklu import BlockLU
    rng = np.random.default_rng(sum(sizes))
    blocks = random_blocks(rng, sizes)
    lu = BlockLU(sizes)
    lu.load(blocks)
    lu.invert(fp32=True)
    lu.check()
    for b, A in enumerate(blocks):
        ref = np.linalg.inv(A)
        # forward error of an inverse: a few ulps times the condition number
        assert rel_err(lu.block(b).cpu().numpy(), ref) < max(1e-12, 1e-14 * np.linalg.cond(A))
    x = torch.tensor(rng.normal(size=sum(sizes)), device="cuda")
    y64 = lu.apply(x, torch.empty_like(x), "fp64").cpu().numpy()
    y32 = lu.apply(x, torch.empty_like(x), "fp32c").cpu().numpy()
    off = 0
    for A, n in zip(blocks, sizes):
        ref = np.linalg.solve(A, x[off:off + n].cpu().numpy())
        assert rel_err(y64[off:off + n], ref) < max(1e-12, 1e-14 * np.linalg.cond(A))
        assert rel_err(y32[off:off + n], ref) < 1e-5
        off += n


@pytest.mark.parametrize("n", [8, 64, 128])
def test_inverse_zero_pivot_reported(n):
    from fiber3d_b200.blocklu import BlockLU
    A = np.eye(n)
    A[3, :] = 0.0
    lu = BlockLU([n, n])
    lu.load([np.eye(n), A])
    lu.invert()
    with pytest.raises(ZeroDivisionError):
        lu.check()


def test_inverse_of_reference_fiber_blocks():
    """Applying the explicit inverses of the fiber blocks of fiber3d's step
    gives fiber3d's lu_solve-based preconditioner output on those rows."""
    from fiber3d_b200.blocklu import BlockLU
    from test_oracle_system import build_from_golden
    g = load_golden("step_small.npz")
    sys_ = build_from_golden(g)
    sizes = [A.shape[0] for A in sys_.A_fib]
    lu = BlockLU(sizes)
    lu.load(sys_.A_fib)
    lu.invert()
    lu.check()
    o = sys_.o_fib
    for x, px in zip(g["probe_x"], g["probe_Px"]):
        xd = torch.tensor(x[o:], device="cuda")
        y = lu.apply(xd, torch.empty_like(xd)).cpu().numpy()
        assert rel_err(y, px[o:]) < 1e-10
