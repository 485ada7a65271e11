"""The periphery (shell) operator on the GPU against fiber3d's own Periphery
and dense shell operator (tests/golden/sphere.npz, make_golden.py: a
300-node sphere of radius 10, inward normals, equal weights):

* f3d_singularity_vectors against Periphery.get_singularity_subtraction_vectors
  (periphery/periphery.py:75-98): ex, ey, ez;
* the matrix-free shell rows, f3d_shell_residual after the double-layer sum
  (tstep.py:1097-1104 with the matrices of tstep.py:327-347), against
  shell_stresslet @ q and (shell_stresslet + shell_complementary) @ q;
* the dense operator f3d_surface_dense and the preconditioner apply (its
  explicit inverse) against fiber3d's LU solve of the same matrix.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shell(golden_sphere):
    from fiber3d_b200 import hydro as H
    torch.cuda.set_device(0)
    g = golden_sphere
    sh = H.Shell(g["shell_nodes"], g["shell_normals"], g["shell_w"])
    return H.ShellOperator(sh, eta=1.0)


def test_singularity_vectors(shell, golden_sphere):
    g = golden_sphere
    E = shell.E.cpu().numpy().reshape(-1, 3, 3)  # E[i, a, c] = e_c(i)_a
    for c, key in enumerate(("shell_ex", "shell_ey", "shell_ez")):
        assert rel_err(E[:, :, c].reshape(-1), g[key]) < 1e-12


def _shell_rows(shell, q):
    from fiber3d_b200 import _lib, kernels
    n = shell.n
    qd = torch.as_tensor(q.reshape(n, 3), device="cuda").contiguous()
    v = kernels.pair_sum("stresslet", shell.nodes, shell.nodes, qd, shell.normals, self_mode="skip_index")
    res = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    scratch = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.call("f3d_shell_residual", _lib.ptr(v), _lib.ptr(shell.E), _lib.ptr(shell.weights),
              _lib.ptr(shell.normals), _lib.ptr(qd), _lib.ptr(res), n, _lib.ptr(scratch), _lib.stream_handle())
    return res.cpu().numpy()


def test_matrix_free_shell_rows(shell, golden_sphere):
    g = golden_sphere
    nrm = g["shell_normals"]
    for k in range(g["shell_q"].shape[0]):
        q = g["shell_q"][k]
        res = _shell_rows(shell, q)
        assert rel_err(res, g["shell_full_q"][k]) < 1e-12
        # without the complementary (rank-one) term
        comp = (nrm * np.sum(nrm.reshape(-1) * q)).reshape(-1)
        assert rel_err(res - comp, g["shell_stresslet_q"][k]) < 1e-12


def test_dense_operator_and_preconditioner(shell, golden_sphere):
    g = golden_sphere
    M = shell.dense().cpu().numpy()
    q = g["shell_q"]
    assert rel_err(q @ M.T, g["shell_full_q"]) < 1e-12
    for k in range(q.shape[0]):
        x = torch.as_tensor(q[k], device="cuda")
        y = torch.empty_like(x)
        shell.apply(x, y, storage="fp64")
        assert rel_err(y.cpu().numpy(), g["shell_pc_q"][k]) < 1e-10
