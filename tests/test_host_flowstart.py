"""The local-mobility map of the (positions, background velocity) warm
start against the oracle's restatement of fiber.self_mobility
(fiber/fiber.py:964-993), on the CPU (torch CPU tensors, no GPU)."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import torch

from fiber3d_b200 import flowstart as FS
from fiber3d_b200.fibers import Resolution
from oracle import fiber_ops as OF


def test_map_to_guess_matches_self_mobility():
    rng = np.random.default_rng(3)
    nfib, n, L, dt = 3, 32, 2.0, 1e-3
    c0, c1 = OF.mobility_constants(1e-3, 1.0)
    res = Resolution(n)
    X = np.stack([np.cumsum(np.full((n, 3), L / (n - 1) / np.sqrt(3)), axis=0)
                  + 0.01 * rng.normal(size=(n, 3)) for _ in range(nfib)])
    U = rng.normal(size=(nfib, n, 3))
    f = rng.normal(size=(nfib, n, 3))
    T = rng.normal(size=(nfib, n))
    system = SimpleNamespace(o_fib=0, fs=SimpleNamespace(nfib=nfib, resolutions={n: res},
                                                         length=torch.full((nfib,), L, dtype=torch.float64)),
                             device=torch.device("cpu"), c0=c0, c1=c1, p=SimpleNamespace(dt=dt))
    x_base = torch.zeros(4 * n * nfib, dtype=torch.float64)
    tX, tU, tf, tT = (torch.as_tensor(a) for a in (X, U, f, T))
    x0 = FS.map_to_guess(system, x_base, tX, tU, tT, tf, FS._Tangent(system)).numpy().reshape(nfib, 4, n)
    D1 = res.D0[0] * (2.0 / L)
    for k in range(nfib):
        xs = D1 @ X[k]
        M = OF.self_mobility(xs, c0, c1)
        Mf = (M @ f[k].T.reshape(-1)).reshape(3, n)
        want = X[k].T + dt * (Mf + U[k].T)
        assert np.max(np.abs(x0[k, :3] - want)) < 1e-14 * np.max(np.abs(want))
        assert np.array_equal(x0[k, 3], T[k])


def test_features_and_targets_shapes():
    X = torch.randn(5, 32, 3, dtype=torch.float64)
    F = FS.features(X, torch.randn(5, 32, 3, dtype=torch.float64))
    assert F.shape == (5, 192) and F.dtype == torch.float32
    assert torch.allclose(F[:, :96].view(5, 32, 3).double().mean(1), torch.zeros(5, 3, dtype=torch.float64),
                          atol=1e-6)
    Y = FS.targets(torch.randn(5, 32, dtype=torch.float64), torch.randn(5, 32, 3, dtype=torch.float64))
    assert Y.shape == (5, 128)
