"""Golden vectors of fiber3d's RBF surface quadrature (needs the fiber3d
sources; see refshim.py).

    python tests/golden/make_golden_quadrature.py

Runs fiber3d's own ``Smooth_Closed_Surface_Quadrature_RBF`` (quadratures/
Smooth_Closed_Surface_Quadrature_RBF.py) with the exact gradient, as
tstep/tstep.py:285-300 does: nodes and gradient from ``shape_gallery``, the
triangles from ``scipy.spatial.ConvexHull``.  Three surfaces: a 400-node
sphere of radius 10 (a periphery), a 500-node ellipsoid (6, 5, 4) and a
200-node sphere of radius 0.5 (a body); and the weights and triangles of
the 12000-node sphere of radius 10 (the time-step workload's periphery,
about two minutes in fiber3d).  Also stores the 80 nearest
neighbours of each triangle midpoint from scikit-learn (the reference's
search, :114-115) for the 400-node sphere, and the reference's polynomial
moments (``Polynomial_Term_Right_Triangle_Double_Integrals``, :473-622) of 24
random triangles.  Writes ``quadrature.npz``.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import refshim  # noqa: E402

sys.path.insert(0, refshim.install())

from quadratures import Smooth_Closed_Surface_Quadrature_RBF as Q  # noqa: E402
from shape_gallery import shape_gallery as SG  # noqa: E402
from scipy.spatial import ConvexHull  # noqa: E402
from sklearn.neighbors import NearestNeighbors  # noqa: E402


def case(shape, n, **kw):
    nodes, normals, h, gradh = SG.shape_gallery(shape, n, **kw)
    tri = ConvexHull(nodes).simplices.astype(np.int32)
    w = Q.Smooth_Closed_Surface_Quadrature_RBF(nodes, tri, h, gradh)[:, 0]
    return nodes, tri, np.asarray(gradh(nodes), dtype=np.float64), w


def main():
    out = {}
    for name, args, kw in (("sphere", ("sphere", 400), dict(radius=10.0)),
                           ("ellipsoid", ("ellipsoid", 500), dict(a=6.0, b=5.0, c=4.0)),
                           ("body", ("sphere", 200), dict(radius=0.5))):
        nodes, tri, grad, w = case(*args, **kw)
        out[f"{name}_nodes"] = nodes
        out[f"{name}_tri"] = tri
        out[f"{name}_grad"] = grad
        out[f"{name}_w"] = w
        if name == "sphere":
            ts = np.sort(tri, axis=1)
            mids = (nodes[ts[:, 0]] + nodes[ts[:, 1]] + nodes[ts[:, 2]]) / 3
            _, nni = NearestNeighbors(n_neighbors=80).fit(nodes).kneighbors(mids)
            out["sphere_nni"] = nni.astype(np.int16)
        print(name, len(nodes), len(tri), w.sum())
    # the 12000-node periphery of radius 10 (the time-step workload's shell):
    # weights and triangles only (the nodes are shape_gallery's, regenerated)
    nodes, tri, grad, w = case("sphere", 12000, radius=10.0)
    out["periphery12000_tri"] = tri.astype(np.int16)
    out["periphery12000_w"] = w
    print("periphery12000", len(nodes), len(tri), w.sum())
    rng = np.random.default_rng(7)
    verts = rng.normal(size=(24, 3, 2))
    moms = np.stack([Q.Polynomial_Term_Right_Triangle_Double_Integrals(np.vstack([v, v[:2]]), 7) for v in verts])
    out["poly_vertices"] = verts
    out["poly_moments"] = moms
    np.savez_compressed(HERE / "quadrature.npz", **out)


if __name__ == "__main__":
    main()
