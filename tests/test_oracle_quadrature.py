"""The CPU oracle of the RBF surface quadrature against fiber3d's own outputs
(tests/golden/quadrature.npz, written by make_golden_quadrature.py)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from oracle import quadrature as OQ

# The weights carry the rounding noise of the method itself: moving every
# node coordinate by one ulp moves fiber3d's weights (relative to the
# largest) by 1.5e-11 (sphere R = 10), 2.6e-11 (ellipsoid) and 5.9e-9 (the
# R = 0.5 body sphere, whose local systems mix r^7 ~ 1e-7 with constants).
# The oracle differs from fiber3d only in rounding order and agrees to
# 1.2e-11, 2.1e-11 and 1.1e-9.  Tolerances: about five times the one-ulp
# movement.
W_TOL = {"sphere": 1e-10, "ellipsoid": 1.5e-10, "body": 3e-8}


@pytest.fixture(scope="module")
def gq():
    return load_golden("quadrature.npz")


def test_polynomial_moments_match_reference(gq):
    for v, ref in zip(gq["poly_vertices"], gq["poly_moments"]):
        got = OQ.polynomial_moments(v)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-13 * scale


def test_neighbours_match_scikit_learn(gq):
    nodes, tri = gq["sphere_nodes"], np.sort(gq["sphere_tri"], axis=1)
    mids = (nodes[tri[:, 0]] + nodes[tri[:, 1]] + nodes[tri[:, 2]]) / 3
    assert np.array_equal(OQ.nearest_neighbors(nodes, mids), gq["sphere_nni"].astype(np.int64))


@pytest.mark.parametrize("name", ["sphere", "ellipsoid", "body"])
def test_weights_match_reference(gq, name):
    w = OQ.quadrature_weights(gq[f"{name}_nodes"], gq[f"{name}_tri"], gq[f"{name}_grad"])
    ref = gq[f"{name}_w"]
    assert np.abs(w - ref).max() <= W_TOL[name] * np.abs(ref).max()


def test_vertex_order_does_not_matter(gq):
    tri = gq["body_tri"][:, ::-1].copy()
    w = OQ.quadrature_weights(gq["body_nodes"], tri, gq["body_grad"])
    assert np.abs(w - gq["body_w"]).max() <= W_TOL["body"] * np.abs(gq["body_w"]).max()


def test_open_surface_is_rejected(gq):
    with pytest.raises(ValueError):
        OQ.quadrature_weights(gq["body_nodes"], gq["body_tri"][1:], gq["body_grad"])


def test_sphere_moments(gq):
    """Size-independent property: the weights integrate 1 and x^2 on the
    sphere (4 pi R^2 and 4 pi R^4 / 3) to the method's accuracy."""
    x, w = gq["sphere_nodes"], gq["sphere_w"]
    R = 10.0
    assert abs(w.sum() / (4 * np.pi * R ** 2) - 1) < 5e-6
    assert abs((w * x[:, 0] ** 2).sum() / (4 * np.pi * R ** 4 / 3) - 1) < 5e-5


def test_periphery_reference_weights_integrate(gq):
    """fiber3d's own weights of the 12000-node periphery integrate 1 and x^2
    over the sphere to 1e-10 (the GPU tests compare against them)."""
    from fiber3d_b200 import geometry
    x, _ = geometry.fibonacci_sphere(12000, 10.0)
    w = gq["periphery12000_w"]
    assert abs(w.sum() / (4 * np.pi * 100.0) - 1) < 1e-10
    assert abs((w * x[:, 0] ** 2).sum() / (4 * np.pi * 1e4 / 3) - 1) < 2e-10
