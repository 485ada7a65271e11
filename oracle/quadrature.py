"""CPU oracle (test infrastructure only) for fiber3d's RBF surface quadrature.

Restates ``Smooth_Closed_Surface_Quadrature_RBF`` with an exact surface
gradient (python/quadratures/Smooth_Closed_Surface_Quadrature_RBF.py:3-470,
the branch every fiber3d caller takes: tstep/tstep.py:297-300,
body/body.py:104-107), the method of Reeger, Fornberg and Watts, "Numerical
quadrature over smooth, closed surfaces" (Proc. R. Soc. A 472, 2016):

* every triangle of the surface triangulation is paired with its 80 nearest
  nodes (nearest to the triangle's midpoint, scikit-learn's
  ``NearestNeighbors``, :114-115);
* those nodes are projected, through a projection point built from the
  edge normals (the average of the two adjacent triangles' normals,
  :118-127, 175-201), onto the plane of the triangle (:225-236);
* in that plane the weights of the phs RBF r^7 plus bivariate polynomials
  up to degree 7 are the solution of the saddle-point system
  [Phi P; P^T 0] [w; lambda] = [I_RBF; I_poly] (:334-336), with I_RBF the
  exact integrals of r^7 over the triangle (sums of right triangles,
  :262-309) and I_poly the polynomial moments of the triangle (Green's
  theorem, :473-622);
* the plane weights are scaled by the area-element distortion of the
  projection (:431-447) and summed per node over triangles (:460-468).

Differences from the reference that change nothing in exact arithmetic:
the polynomial moments are computed by Gauss-Legendre quadrature of the
Green's-theorem line integrals (exact for these degrees) instead of the
reference's expanded closed forms, and the loop over triangles is batched.
The solve is LAPACK ``gesv`` (numpy's batched ``solve``), as in the
reference.
"""
from __future__ import annotations

import numpy as np

POLY_ORDER = 7
N_NEIGHBORS = 80
N_POLY = (POLY_ORDER + 1) * (POLY_ORDER + 2) // 2
EPSMULT = 1e-4


def triangle_normals(nodes: np.ndarray, tri: np.ndarray) -> np.ndarray:
    """Unit normals of the triangles (rows of ``tri`` sorted), :109-112."""
    v1 = nodes[tri[:, 1]] - nodes[tri[:, 0]]
    v2 = nodes[tri[:, 2]] - nodes[tri[:, 0]]
    n = np.stack([v1[:, 1] * v2[:, 2] - v2[:, 1] * v1[:, 2],
                  v2[:, 0] * v1[:, 2] - v1[:, 0] * v2[:, 2],
                  v1[:, 0] * v2[:, 1] - v2[:, 0] * v1[:, 1]], axis=1)
    return n / np.sqrt(n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1] + n[:, 2] * n[:, 2])[:, None]


def edge_normals(tri: np.ndarray, tnorm: np.ndarray) -> np.ndarray:
    """(T, 3, 3): per triangle, the unit normals of its edges (i0,i1),
    (i0,i2), (i1,i2) (vertices sorted), each the average of the two
    adjacent triangles' normals (:97-127).  The edge's first copy in the
    stacked edge list [(i0,i1) of all triangles; (i0,i2); (i1,i2)] gives the
    first normal of the average, the second copy's normal is flipped when
    the two disagree in sign."""
    T = len(tri)
    edges = np.vstack([tri[:, [0, 1]], tri[:, [0, 2]], tri[:, [1, 2]]])
    owner = np.tile(np.arange(T), 3)
    order = np.lexsort((edges[:, 1], edges[:, 0]))
    se = edges[order]
    if len(se) % 2 or np.any(se[0::2] != se[1::2]):
        raise ValueError("triangulation is not a closed surface (every edge must be shared "
                         "by exactly two triangles)")
    na = tnorm[owner[order[0::2]]]
    nb = tnorm[owner[order[1::2]]]
    s = np.sign(na[:, 0] * nb[:, 0] + na[:, 1] * nb[:, 1] + na[:, 2] * nb[:, 2])
    e = (na + s[:, None] * nb) / 2
    e = e / np.sqrt(e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1] + e[:, 2] * e[:, 2])[:, None]
    en = np.empty((3 * T, 3))
    en[order[0::2]] = e
    en[order[1::2]] = e
    return en.reshape(3, T, 3).transpose(1, 0, 2)


def nearest_neighbors(nodes: np.ndarray, queries: np.ndarray, k: int = N_NEIGHBORS) -> np.ndarray:
    """Indices of the k nodes nearest each query point, nearest first, ties
    by index (brute force on squared distances)."""
    out = np.empty((len(queries), k), dtype=np.int64)
    for s in range(0, len(queries), 512):
        q = queries[s:s + 512]
        d = ((q[:, None, :] - nodes[None, :, :]) ** 2).sum(-1)
        part = np.argpartition(d, k, axis=1)[:, :k + 1]
        for r in range(len(q)):
            cand = part[r]
            o = np.lexsort((cand, d[r, cand]))[:k]
            # a tie at the k-th distance may leave a lower index outside the
            # partition: take every node at or below the k-th distance
            kth = d[r, cand[o[-1]]]
            full = np.nonzero(d[r] <= kth)[0]
            out[s + r] = full[np.lexsort((full, d[r, full]))][:k]
    return out


def rotation_matrix(n: np.ndarray) -> np.ndarray:
    """Rotation taking the unit normal n to +z (:210-220)."""
    rxy = np.sqrt(n[0] ** 2 + n[1] ** 2)
    if rxy < np.spacing(1):
        return np.eye(3)
    nn = np.sqrt(n[0] ** 2 + n[1] ** 2 + n[2] ** 2)
    r1 = np.array([[n[2] / nn, 0, -rxy / nn], [0, 1, 0], [rxy / nn, 0, n[2] / nn]])
    r2 = np.array([[n[0] / rxy, n[1] / rxy, 0], [-n[1] / rxy, n[0] / rxy, 0], [0, 0, 1]])
    return r1 @ r2


_GL_X, _GL_W = np.polynomial.legendre.leggauss(6)


def polynomial_moments(v: np.ndarray, order: int = POLY_ORDER) -> np.ndarray:
    """Integrals of x^(d-t) y^t (d = 0..order, t = 0..d, in that order) over
    the triangle with vertices v[0:3] (counter-clockwise positive), by
    Green's theorem: the integral of x^a y^b over the area equals the line
    integral of x^(a+1) y^b / (a+1) dy around it, computed edge by edge with
    6-point Gauss-Legendre (exact up to degree 11).  Same moments as
    Polynomial_Term_Right_Triangle_Double_Integrals (:473-622)."""
    t = 0.5 * (_GL_X + 1.0)
    wt = 0.5 * _GL_W
    out = np.zeros((order + 1) * (order + 2) // 2)
    for s in range(3):
        x1, y1 = v[s]
        x2, y2 = v[(s + 1) % 3]
        x = x1 + t * (x2 - x1)
        y = y1 + t * (y2 - y1)
        dy = y2 - y1
        i = 0
        for d in range(order + 1):
            for k in range(d + 1):
                a = d - k
                out[i] += dy * np.sum(wt * x ** (a + 1) * y ** k) / (a + 1)
                i += 1
    return out


def rbf_right_triangle(alpha: np.ndarray, beta: np.ndarray) -> np.ndarray:
    """Integral of r^7 over the right triangle with legs alpha (from the RBF
    centre to the foot on the side) and beta (along the side), :302."""
    a2 = alpha * alpha
    b2 = beta * beta
    with np.errstate(divide="ignore", invalid="ignore"):
        return alpha * (beta * np.sqrt(a2 + b2) * (279 * a2 ** 3 + 326 * a2 * a2 * b2 + 200 * a2 * b2 * b2
                                                    + 48 * b2 ** 3)
                        + 105 * a2 ** 4 * np.arcsinh(beta / alpha)) / 3456


def monomials(c: np.ndarray, order: int = POLY_ORDER) -> np.ndarray:
    """Rows [1, x, y, x^2, xy, y^2, ...] built by the reference's recursion
    (:324-329): column (d, t) is x * (d-1, t) below the middle and
    y * (d-1, t-1) from the middle on."""
    n = len(c)
    P = np.ones((n, (order + 1) * (order + 2) // 2))
    for d in range(1, order + 1):
        for t in range(d + 1):
            if t >= (d + 1) // 2:
                P[:, d * (d + 1) // 2 + t] = c[:, 1] * P[:, (d - 1) * d // 2 + t - 1]
            else:
                P[:, d * (d + 1) // 2 + t] = c[:, 0] * P[:, (d - 1) * d // 2 + t]
    return P


def triangle_system(nodes, grad, tri_t, tnorm_t, enorm_t, nni):
    """Saddle-point matrix, right-hand side and distortion factors of one
    triangle (vertices sorted)."""
    X = nodes
    A, B, C = X[tri_t[0]], X[tri_t[1]], X[tri_t[2]]
    AB, BC, CA = B - A, C - B, A - C
    nAB, nCA, nBC = enorm_t[0], enorm_t[1], enorm_t[2]
    nOAB = np.cross(nAB, AB)
    nOBC = np.cross(nBC, BC)
    nOCA = np.cross(nCA, CA)
    vOA = np.cross(nOAB, nOCA)
    tA = (nOBC @ AB) / (nOBC @ vOA)
    XP = A + tA * vOA
    n = tnorm_t
    R = rotation_matrix(n)
    Q = X[nni]
    mult = (n[0] * (A[0] - Q[:, 0]) + n[1] * (A[1] - Q[:, 1]) + n[2] * (A[2] - Q[:, 2])) / \
        (n[0] * (Q[:, 0] - XP[0]) + n[1] * (Q[:, 1] - XP[1]) + n[2] * (Q[:, 2] - XP[2]))
    Pc = Q + mult[:, None] * (Q - XP)
    Pc = (R @ (Pc - XP).T).T
    height = Pc[0, 2]
    c = Pc[:, :2].copy()
    V = (R @ (np.stack([A, B, C]) - XP).T).T[:, :2]
    mid = (A + B + C) / 3
    shift = (R @ (mid - XP))[:2]
    c = c - shift
    V = V - shift
    Vc = np.vstack([V, V[:2]])
    s_abc = np.sign((Vc[0, 1] - Vc[1, 1]) * (Vc[2, 0] - Vc[0, 0]) + (Vc[1, 0] - Vc[0, 0]) * (Vc[2, 1] - Vc[0, 1]))
    i_poly = s_abc * polynomial_moments(V)
    eps = np.spacing(1)
    i_rbf = np.zeros(len(nni))
    for s in range(3):
        e = Vc[s + 1] - Vc[s]
        m = ((c[:, 0] - Vc[s, 0]) * e[0] + (c[:, 1] - Vc[s, 1]) * e[1]) / (e[0] ** 2 + e[1] ** 2)
        fx = m * e[0] + Vc[s, 0]
        fy = m * e[1] + Vc[s, 1]
        sg1 = s_abc * np.sign((c[:, 1] - Vc[s, 1]) * (fx - c[:, 0]) + (Vc[s, 0] - c[:, 0]) * (fy - c[:, 1]))
        sg2 = s_abc * np.sign((c[:, 1] - fy) * (Vc[s + 1, 0] - c[:, 0]) + (fx - c[:, 0]) * (Vc[s + 1, 1] - c[:, 1]))
        alpha = np.sqrt((c[:, 0] - fx) ** 2 + (c[:, 1] - fy) ** 2)
        b1 = np.sqrt((fx - Vc[s, 0]) ** 2 + (fy - Vc[s, 1]) ** 2)
        b2 = np.sqrt((fx - Vc[s + 1, 0]) ** 2 + (fy - Vc[s + 1, 1]) ** 2)
        for sg, b in ((sg1, b1), (sg2, b2)):
            ok = (np.abs(alpha) > EPSMULT * eps) & (np.abs(b) > EPSMULT * eps)
            i_rbf[ok] += (sg * rbf_right_triangle(alpha, b))[ok]
    ip = c @ c.T
    d = np.diag(ip)
    r2 = d[None, :] + d[:, None] - 2 * ip
    P = monomials(c)
    k = len(nni)
    M = np.zeros((k + N_POLY, k + N_POLY))
    M[:k, :k] = np.sqrt(r2 ** 7)
    M[:k, k:] = P
    M[k:, :k] = P.T
    rhs = np.concatenate([i_rbf, i_poly])
    # area-element distortion of the projection (:431-442)
    g = grad[nni]
    nS = g / np.sqrt((g * g).sum(1))[:, None]
    Vv = Q - XP
    nv = np.sqrt((Vv * Vv).sum(1))
    Rr = np.sqrt(((c + shift) ** 2).sum(1) + height ** 2)
    Pn = n / np.sqrt((n * n).sum())
    Vh = Vv / nv[:, None]
    dist = np.abs((Vh @ Pn) / (nS * Vh).sum(1) * (nv / Rr) ** 2)
    return M, rhs, dist


def quadrature_weights(nodes: np.ndarray, triangles: np.ndarray, grad: np.ndarray,
                       nni: np.ndarray | None = None, return_parts: bool = False):
    """Node weights (N,) of the RBF surface quadrature with the exact surface
    gradient ``grad`` (N, 3) at the nodes (gradh(nodes) in the reference)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    grad = np.asarray(grad, dtype=np.float64)
    tri = np.sort(np.asarray(triangles, dtype=np.int64), axis=1)
    tn = triangle_normals(nodes, tri)
    en = edge_normals(tri, tn)
    mids = (nodes[tri[:, 0]] + nodes[tri[:, 1]] + nodes[tri[:, 2]]) / 3
    if nni is None:
        nni = nearest_neighbors(nodes, mids)
    T = len(tri)
    wt = np.zeros((T, nni.shape[1]))
    for s in range(0, T, 256):
        Ms, rs, ds = [], [], []
        for t in range(s, min(T, s + 256)):
            M, r, d = triangle_system(nodes, grad, tri[t], tn[t], en[t], nni[t])
            Ms.append(M)
            rs.append(r)
            ds.append(d)
        sol = np.linalg.solve(np.stack(Ms), np.stack(rs)[..., None])[..., 0]
        wt[s:s + len(Ms)] = sol[:, :nni.shape[1]] * np.stack(ds)
    w = np.zeros(len(nodes))
    for t in range(T):
        w[nni[t]] += wt[t]
    if return_parts:
        return w, {"nni": nni, "triangle_weights": wt}
    return w
