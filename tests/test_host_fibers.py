"""The product's host-side fiber matrices (fiber3d_b200.fibers) equal
fiber3d's own (golden fixtures).  CPU only."""
from __future__ import annotations

import pytest

from conftest import rel_err
from fiber3d_b200 import fibers as F


@pytest.mark.parametrize("N", [16, 24, 32, 48, 64])
def test_resolution_matrices(golden_fiber, N):
    g = golden_fiber
    r = F.Resolution(N)
    for k in range(4):
        assert rel_err(r.D0[k], g[f"fm{N}_D{k + 1}"]) < 1e-12
    assert rel_err(r.PX, g[f"fm{N}_PX"]) < 1e-12
    assert rel_err(r.PT, g[f"fm{N}_PT"]) < 1e-12
    assert rel_err(r.w0, g[f"fm{N}_w"]) < 1e-14
    assert r.packed().size == 4 * N * N + (N - 4) * N + (N - 2) * N + N


def test_stencil_band():
    """Every D_k row is non-zero only within n_fd + 3 of the diagonal (the
    window the device kernels loop over)."""
    import numpy as np
    for N in (16, 33, 64):
        r = F.Resolution(N)
        for D in r.D0:
            i, j = np.nonzero(D)
            assert np.max(np.abs(i - j)) <= F.N_FD + 3
