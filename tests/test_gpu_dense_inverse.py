"""f3d_dense_inverse (blocked Gauss-Jordan on the device) against LAPACK
(numpy's LU inverse) and the residual M X - I: random matrices of ragged
sizes (one to many 128-row blocks, a padded last block), a leading dimension
beyond the padding, fiber3d's dense shell operator (the matrix its
tstep.py:327-348 factors), and a singular pivot block reported as an error."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def H():
    torch.cuda.set_device(0)
    from fiber3d_b200 import hydro
    return hydro


def invert(H, M: np.ndarray, extra_cols: int = 0) -> tuple[np.ndarray, torch.Tensor]:
    m = M.shape[0]
    ld = H.dense_inverse_ld(m) + extra_cols
    A = torch.full((H.dense_inverse_ld(m), ld), np.nan, dtype=torch.float64, device="cuda")
    A[:m, :m] = torch.as_tensor(M, device="cuda")
    H.dense_inverse(A, m)
    return A[:m, :m].cpu().numpy(), A


def second_kind(rng, m: int) -> np.ndarray:
    """A dense matrix like the operators inverted here: a dominant diagonal
    of mixed signs, O(1) random couplings and a rank-one term."""
    d = rng.uniform(8.0, 12.0, m) * rng.choice([-1.0, 1.0], m)
    v = rng.normal(size=m)
    return np.diag(d) + rng.normal(size=(m, m)) * (3.0 / np.sqrt(m)) + np.outer(v, v) * 0.5


@pytest.mark.parametrize("m", [1, 5, 127, 128, 129, 300, 1000])
def test_random_against_lapack(H, m):
    rng = np.random.default_rng(m)
    M = second_kind(rng, m)
    X, A = invert(H, M)
    ref = np.linalg.inv(M)
    assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-13
    assert np.abs(M @ X - np.eye(m)).max() < 1e-12
    # the padding is the identity
    np_ = A.shape[0]
    if np_ > m:
        pad = A[m:, :np_].cpu().numpy()
        assert np.array_equal(pad, np.eye(np_)[m:, :np_])
        assert torch.count_nonzero(A[:m, m:np_]).item() == 0


def test_leading_dimension_beyond_padding(H):
    """Columns past the padded square are neither read nor written."""
    rng = np.random.default_rng(7)
    M = second_kind(rng, 260)
    X, A = invert(H, M, extra_cols=6)
    assert np.linalg.norm(X - np.linalg.inv(M)) / np.linalg.norm(X) < 1e-13
    assert torch.isnan(A[:, A.shape[0]:]).all()


def test_shell_operator_against_lapack(H):
    """fiber3d's dense periphery operator on a 1500-node sphere (4500 x 4500,
    36 blocks with a padded last one): the library's inverse against LAPACK's
    LU inverse of the same matrix, and the preconditioner applied through the
    FP64 and FP32 copies."""
    from fiber3d_b200 import geometry
    from fiber3d_b200.hydro import Shell, ShellOperator
    nodes, normals = geometry.fibonacci_sphere(1500, 10.0)
    w = np.full(1500, 4.0 * np.pi * 100.0 / 1500)  # equal-area weights of the Fibonacci sphere
    sh = ShellOperator(Shell(nodes, normals, w), 1.0, 5e-3, 1e-5, torch.device("cuda"))
    M = sh.dense().cpu().numpy()
    ref = np.linalg.inv(M)
    X = sh.inv64.cpu().numpy()
    assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-12
    x = torch.as_tensor(np.random.default_rng(1).normal(size=M.shape[0]), device="cuda")
    y = torch.empty_like(x)
    sh.apply(x, y, "fp64")
    assert np.linalg.norm(y.cpu().numpy() - ref @ x.cpu().numpy()) / np.linalg.norm(ref @ x.cpu().numpy()) < 1e-12
    sh.apply(x, y, "fp32")
    assert np.linalg.norm(y.cpu().numpy() - ref @ x.cpu().numpy()) / np.linalg.norm(ref @ x.cpu().numpy()) < 1e-5


def test_singular_pivot_block_is_reported(H):
    from fiber3d_b200 import _lib
    rng = np.random.default_rng(3)
    M = second_kind(rng, 200)
    M[:128, 3] = 0.0  # a zero column inside the first pivot block: an exactly zero pivot
    with pytest.raises(_lib.F3DError) as e:
        invert(H, M)
    assert e.value.status == _lib.F3D_ERR_SINGULAR
