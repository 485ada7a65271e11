"""Seeded synthetic geometry for the fiber3d hot-path workloads.

* :func:`fibonacci_sphere` restates fiber3d's ``shape_gallery('sphere', N,
  radius=R)`` (python/shape_gallery/shape_gallery.py:7-32): a latitude/longitude
  Fibonacci lattice with outward unit normals.
* Fiber generators: straight fibers on Chebyshev-Lobatto nodes (the Oseen
  kernel workload), and fibers on the solver's equispaced parameter nodes
  alpha = linspace(-1, 1, N) (python/fiber/fiber.py:128) with random transverse
  Fourier modes (the time-step workloads).

All generators take a ``numpy.random.Generator`` or an integer seed.
"""
from __future__ import annotations

import numpy as np


def _rng(seed) -> np.random.Generator:
    return seed if isinstance(seed, np.random.Generator) else np.random.default_rng(seed)


def fibonacci_sphere(n: int, radius: float):
    """Nodes and outward unit normals of shape_gallery('sphere', n, radius).

    Node k = i + n//2 for i in [-n//2, n//2): latitude asin(2i/(2(n//2)+1)),
    longitude (i mod phi) * 2 pi / phi wrapped into [-pi, pi], phi the golden
    ratio (shape_gallery.py:9-22).  For odd n the last node stays at the
    origin, as in the reference.
    """
    phi = (1.0 + np.sqrt(5.0)) / 2.0
    half = n // 2
    nodes = np.zeros((n, 3))
    i = np.arange(-half, half)
    lat = np.arcsin((2.0 * i) / (2 * half + 1))
    lon = np.mod(i, phi) * 2.0 * np.pi / phi
    lon = np.where(lon < -np.pi, 2.0 * np.pi + lon, lon)
    lon = np.where(lon > np.pi, lon - 2.0 * np.pi, lon)
    nodes[: 2 * half] = np.stack([np.cos(lon) * np.cos(lat), np.sin(lon) * np.cos(lat),
                                  np.sin(lat)], axis=1)
    nodes *= radius
    normals = 2.0 * nodes
    with np.errstate(invalid="ignore", divide="ignore"):
        normals /= np.linalg.norm(normals, axis=1, keepdims=True)
    return nodes, normals


def uniform_ball(rng, n: int, radius: float) -> np.ndarray:
    rng = _rng(rng)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = radius * rng.random(n) ** (1.0 / 3.0)
    return v * r[:, None]


def uniform_directions(rng, n: int) -> np.ndarray:
    rng = _rng(rng)
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def chebyshev_lobatto(n: int) -> np.ndarray:
    """-cos(pi k/(n-1)), k = 0..n-1 (ascending in [-1, 1])."""
    return -np.cos(np.pi * np.arange(n) / (n - 1))


def straight_fibers_cheb(rng, nfib: int, npts: int, length: float, ball_radius: float):
    """Straight fibers on Chebyshev-Lobatto nodes: x = c + (L/2) s d."""
    rng = _rng(rng)
    c = uniform_ball(rng, nfib, ball_radius)
    d = uniform_directions(rng, nfib)
    s = chebyshev_lobatto(npts)
    x = c[:, None, :] + (length / 2.0) * s[None, :, None] * d[:, None, :]
    return x.reshape(nfib * npts, 3)


def _segment_distances(p0, d0, P, D):
    """Distances between segment p0 + t d0 and segments P_k + s D_k, t, s in [0, 1]."""
    r = p0[None, :] - P
    a = np.dot(d0, d0)
    e = np.einsum("ij,ij->i", D, D)
    b = D @ d0
    c = r @ d0
    f = np.einsum("ij,ij->i", D, r)
    den = a * e - b * b
    t = np.where(den > 1e-12, (b * f - c * e) / np.where(den > 1e-12, den, 1.0), 0.0)
    t = np.clip(t, 0.0, 1.0)
    s = np.clip((b * t + f) / e, 0.0, 1.0)
    t = np.clip((b * s - c) / a, 0.0, 1.0)
    q = r + t[:, None] * d0[None, :] - s[:, None] * D
    return np.sqrt(np.einsum("ij,ij->i", q, q))


def separated_fibers(rng, nfib: int, length: float, ball_radius: float, min_sep: float,
                     max_tries: int = 200000):
    """Centres and directions of `nfib` straight fibers (uniform in a ball,
    uniform directions) whose centre lines stay at least `min_sep` apart
    (rejection sampling)."""
    rng = _rng(rng)
    C, Dd = [], []
    tries = 0
    while len(C) < nfib:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could only place {len(C)} of {nfib} fibers {min_sep} apart")
        c = uniform_ball(rng, 1, ball_radius)[0]
        d = uniform_directions(rng, 1)[0]
        p0 = c - 0.5 * length * d
        if C:
            Pa = np.array(C) - 0.5 * length * np.array(Dd)
            if np.min(_segment_distances(p0, length * d, Pa, length * np.array(Dd))) < min_sep:
                continue
        C.append(c)
        Dd.append(d)
    return np.array(C), np.array(Dd)


def perturbed_fibers(rng, nfib: int, npts, length: float, ball_radius: float,
                     amplitude: float = 0.05, modes: int = 3, min_sep: float | None = None):
    """Fibers on the solver's equispaced nodes alpha = linspace(-1, 1, N):
    straight line through a centre uniform in a ball, plus ``modes`` random
    transverse Fourier modes sin(k pi (alpha+1)/2) of amplitude ``amplitude``.

    ``npts`` is an int or a per-fiber sequence.  Returns a list of (N_k, 3)
    arrays.
    """
    rng = _rng(rng)
    if np.isscalar(npts):
        npts = [int(npts)] * nfib
    if min_sep:
        c, d = separated_fibers(rng, nfib, length, ball_radius, min_sep + 2 * amplitude)
    else:
        c = uniform_ball(rng, nfib, ball_radius)
        d = uniform_directions(rng, nfib)
    out = []
    for k in range(nfib):
        n = int(npts[k])
        alpha = np.linspace(-1.0, 1.0, n)
        # two unit vectors orthogonal to d
        a = np.array([1.0, 0.0, 0.0]) if abs(d[k, 0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        e1 = np.cross(d[k], a)
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(d[k], e1)
        x = c[k] + (length / 2.0) * alpha[:, None] * d[k]
        for m in range(1, modes + 1):
            w = rng.normal(size=2)
            w /= np.linalg.norm(w)
            x = x + amplitude * np.sin(m * np.pi * (alpha + 1.0) / 2.0)[:, None] * (w[0] * e1 + w[1] * e2)
        out.append(x)
    return out


# --------------------------------------------------------------- workloads --
def oseen_fiber_workload(seed: int = 1, nfib: int = 32, npts: int = 32):
    """32 straight fibers of length 2 x 32 Chebyshev-Lobatto nodes, centres
    uniform in a ball of radius 5, directions uniform; forces N(0,1)."""
    rng = _rng(seed)
    x = straight_fibers_cheb(rng, nfib, npts, 2.0, 5.0)
    f = rng.normal(size=x.shape)
    return x, f


def stresslet_sphere_workload(seed: int = 2, n: int = 12000, radius: float = 10.0,
                              n_vol: int = 4096, vol_radius: float = 9.0):
    """Spherical periphery (Fibonacci nodes, outward normals, equal weights
    4 pi R^2 / N), double-layer density N(0,1), plus volume targets uniform
    in a ball of radius 9."""
    rng = _rng(seed)
    nodes, normals = fibonacci_sphere(n, radius)
    w = np.full(n, 4.0 * np.pi * radius**2 / n)
    mu = rng.normal(size=(n, 3))
    vol = uniform_ball(rng, n_vol, vol_radius)
    return nodes, normals, w, mu, vol


def hydro_step_problem(seed: int = 3, nfib: int = 512, npts=32, nbody: int = 4,
                       body_nodes: int = 400, nshell: int = 12000, shell_radius: float = 10.0,
                       length: float = 2.0, E: float = 0.0025, dt: float = 1e-3, eta: float = 1.0,
                       force_std: float = 0.1, fiber_ball: float = 5.0, body_shell: float = 7.5,
                       min_sep: float | None = 0.1):
    """Full-step workload: `nfib` fibers (equispaced nodes, straight + 3
    transverse modes of amplitude 0.05, centres uniform in a ball of radius
    5), `nbody` rigid spheres of radius 0.5 (Fibonacci nodes, equal weights,
    random orientation, centres at radius `body_shell`), a spherical periphery
    of `nshell` nodes (inward normals as fiber3d uses them, equal weights
    4 pi R^2 / N), and a constant external force N(0, force_std) per fiber.
    Fiber centre lines are kept `min_sep` apart (plus the mode amplitudes)."""
    from .hydro import Body, Problem, Shell, quaternion_rotation
    rng = _rng(seed)
    fibers = perturbed_fibers(rng, nfib, npts, length, fiber_ball, min_sep=min_sep)
    counts = [f.shape[0] for f in fibers]
    ff = np.concatenate([np.tile(rng.normal(scale=force_std, size=3), (n, 1)) for n in counts])
    bn, bnn = fibonacci_sphere(body_nodes, 0.5)
    bw = np.full(body_nodes, 4.0 * np.pi * 0.25 / body_nodes)
    bodies = []
    dirs = uniform_directions(rng, nbody)
    for k in range(nbody):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        bodies.append(Body(body_shell * dirs[k], quaternion_rotation(q), bn, bnn, bw))
    sn, snn = fibonacci_sphere(nshell, shell_radius)
    sw = np.full(nshell, 4.0 * np.pi * shell_radius**2 / nshell)
    return Problem(fibers, [length] * nfib, E, dt, eta, bodies, Shell(sn, -snn, sw), ff)


def ellipsoid_grid(b: float = 5.5, c: float = 5.5, dx: float = 0.25) -> np.ndarray:
    """Grid points at which fiber3d evaluates the velocity field
    (tstep.py:1240-1270): the ij-meshgrid of arange(-b, b + dx, dx) (x, y)
    and arange(-c, c + dx, dx) (z), kept where
    sqrt(x^2/c^2 + y^2/b^2 + z^2/c^2) <= 0.99, in meshgrid order."""
    xs = np.arange(-b, b + dx, dx)
    ys = np.arange(-b, b + dx, dx)
    zs = np.arange(-c, c + dx, dx)
    xv, yv, zv = np.meshgrid(xs, ys, zs, sparse=False, indexing="ij")
    xv, yv, zv = xv.ravel(), yv.ravel(), zv.ravel()
    keep = np.sqrt(xv ** 2 / c ** 2 + yv ** 2 / b ** 2 + zv ** 2 / c ** 2) <= 0.99
    return np.stack([xv[keep], yv[keep], zv[keep]], axis=1)
