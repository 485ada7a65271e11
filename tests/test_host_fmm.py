"""The FMM's host-side operators (fiber3d_b200/fmm.py), checked in numpy on
the CPU: the surface grid, and that the two pseudo-inverses turn check
potentials into equivalent densities that reproduce the Stokeslet and
stresslet fields of sources in a box outside it (upward) and of sources far
from a box inside it (downward), with the unit-scaled density convention
the device passes rely on.  References: direct sums in numpy."""
from __future__ import annotations

import numpy as np
import pytest

from fiber3d_b200 import fmm as F


def oseen(x, y, f):
    r = x[:, None, :] - y[None, :, :]
    d = np.linalg.norm(r, axis=-1)
    rf = np.einsum("ijk,jk->ij", r, f)
    return (f[None] / d[..., None] + r * (rf / d**3)[..., None]).sum(1) / (8 * np.pi)


def stresslet(x, y, n, d):
    r = x[:, None, :] - y[None, :, :]
    dist = np.linalg.norm(r, axis=-1)
    q = np.einsum("ijk,jk->ij", r, n) * np.einsum("ijk,jk->ij", r, d) / dist**5
    return -3 / (4 * np.pi) * (r * q[..., None]).sum(1)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("order", [4, 6, 8, 10])
def test_surface_grid(order):
    s = F.surface(order)
    assert s.shape == (6 * (order - 1) ** 2 + 2, 3)
    assert np.allclose(np.abs(s).max(axis=1), 1.0)
    assert len({tuple(p) for p in s.round(12)}) == s.shape[0]
    assert s.shape[0] % 8 == 0  # the device tiles take equivalent points 8 at a time


def test_orders_are_even():
    for bad in (3, 5, 18, 2):
        with pytest.raises(ValueError):
            F.operators(bad)


@pytest.fixture(scope="module")
def sources():
    rng = np.random.default_rng(7)
    y = rng.uniform(-1, 1, (150, 3))
    return y, rng.normal(size=(150, 3)), rng.normal(size=(150, 3)), rng.normal(size=(150, 3))


@pytest.mark.parametrize("order,tol_sl,tol_dl", [(6, 5e-5, 1e-3), (8, 1e-6, 2e-5), (10, 2e-7, 3e-6)])
@pytest.mark.parametrize("h", [1.0, 0.125])
def test_upward_equivalent_density(sources, order, tol_sl, tol_dl, h):
    """Sources in a box of half-width h: their velocity on the upward check
    surface, times h * uc2ue, is the unit-scaled density (f, q / h) whose K4
    field equals the sources' field outside the box."""
    y, f, n, d = sources
    s, uc2ue, _ = F.operators(order)
    rng = np.random.default_rng(3)
    far = rng.normal(size=(200, 3))
    far = far / np.linalg.norm(far, axis=1)[:, None] * rng.uniform(3.0, 6.0, (200, 1)) * h
    for field, tol in ((lambda x: oseen(x, h * y, f), tol_sl), (lambda x: stresslet(x, h * y, n, d), tol_dl)):
        chk = field(F.R_OUT * h * s).reshape(-1)
        phi = (h * uc2ue @ chk).reshape(-1, 4)
        phi[:, 3] *= h  # the unit-scaled source component back to q
        u = (F.k4(far, F.R_IN * h * s) @ phi.reshape(-1)).reshape(-1, 3)
        assert rel(u, field(far)) < tol


@pytest.mark.parametrize("order,tol", [(6, 1e-3), (8, 3e-5), (10, 1e-6)])
def test_downward_equivalent_density(sources, order, tol):
    """Sources well outside a unit box: their velocity on the downward check
    surface, times dc2de, is a density on the downward equivalent surface
    whose K4 field equals theirs inside the box (both layers)."""
    y, f, n, d = sources
    s, _, dc2de = F.operators(order)
    y_far = y + np.array([5.0, -1.0, 0.5])
    rng = np.random.default_rng(4)
    inside = rng.uniform(-1, 1, (200, 3))
    for field in (lambda x: oseen(x, y_far, f), lambda x: stresslet(x, y_far, n, d)):
        psi = dc2de @ field(F.R_IN * s).reshape(-1)
        u = (F.k4(inside, F.R_OUT * s) @ psi).reshape(-1, 3)
        assert rel(u, field(inside)) < tol


def test_stokeslet_only_equivalents_miss_the_double_layer_flux(sources):
    """Why the densities carry a source component: a double layer whose
    tensor has a trace has a net flux, which a Stokeslet-only equivalent
    density cannot reproduce."""
    y, f, n, d = sources
    s = F.surface(8)
    k3 = lambda x, z: F.k4(x, z).reshape(3 * len(x), len(z), 4)[:, :, :3].reshape(3 * len(x), 3 * len(z))
    p3 = F.pinv(k3(F.R_OUT * s, F.R_IN * s))
    far = np.array([[4.0, 1.0, -2.0], [-3.0, 3.5, 1.0], [0.5, -4.5, 2.5]])
    chk = stresslet(F.R_OUT * s, y, n, d).reshape(-1)
    u3 = (k3(far, F.R_IN * s) @ (p3 @ chk)).reshape(-1, 3)
    assert rel(u3, stresslet(far, y, n, d)) > 1e-2
