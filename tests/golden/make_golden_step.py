"""Golden vectors of one fiber3d hydrodynamic time step (needs the fiber3d
sources; see refshim.py).

    python tests/golden/make_golden_step.py

Runs fiber3d's own ``tstep.time_step_hydro`` (tstep/tstep.py:628-1458) on a
small seeded system — fibers of uneven resolution, rigid spheres and a
spherical periphery — and records, by wrapping the GMRES call
(tstep.py:1209-1216), the right-hand side, the matvec closure
A_body_fiber_hyd (tstep.py:1003-1178) and the preconditioner closure P_inv
(tstep.py:950-994) applied to seeded vectors, and the GMRES solution.
Writes ``step_small.npz``.

External forces: fiber3d injects them through
forces.compute_hydro_repulsion_force (tstep.py:726-730); here that function
is replaced by one returning a seeded constant force per fiber.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

import refshim  # noqa: E402

refshim.install()

from tstep import tstep as ts, initialize  # noqa: E402
from fiber import fiber as fiber_mod  # noqa: E402
from body import body as body_mod  # noqa: E402
from quaternion import quaternion  # noqa: E402
from bpm_utilities import gmres as gmres_mod  # noqa: E402
from shape_gallery import shape_gallery  # noqa: E402

from fiber3d_b200 import geometry  # noqa: E402


def build_system(rng, npts, nbody, nb_nodes, nper, R_per, L, E, dt, tol):
    nfib = len(npts)
    xs = geometry.perturbed_fibers(rng, nfib, npts, L, 0.45 * R_per)
    fibers = []
    for k in range(nfib):
        f = fiber_mod.fiber(num_points=npts[k], length=L, dt=dt, E=E, adaptive_num_points=0,
                            num_points_finite_diff=4, epsilon=1e-3, viscosity=1.0)
        f.x = xs[k].copy()
        f.length_previous = L
        fibers.append(f)
    bodies = []
    ref_nodes, ref_normals, _, _ = shape_gallery.shape_gallery('sphere', nb_nodes, radius=0.5)
    w = np.full(nb_nodes, 4.0 * np.pi * 0.5**2 / nb_nodes)
    for k in range(nbody):
        loc = geometry.uniform_ball(rng, 1, 0.4 * R_per)[0]
        qv = rng.normal(size=4)
        qv /= np.linalg.norm(qv)
        b = body_mod.Body(loc, quaternion.Quaternion(qv), ref_nodes.copy(), ref_normals.copy(), w.copy())
        b.radius = 0.5
        b.quadrature_radius = 0.5
        bodies.append(b)
    options = initialize.set_options(num_points=npts[0], time_step_scheme='time_step_hydro', dt=dt,
                                     tol_gmres=tol, Nperiphery=nper, output_name='/tmp/f3d_golden_step',
                                     dynInstability=False, adaptive_num_points=False, iupsample=False,
                                     repulsion=True)
    prams = initialize.set_parameters(eta=1.0, final_time=dt, periphery='sphere', periphery_radius=R_per,
                                      Efib=E, fiber_body_attached=False, growing=0)
    return fibers, bodies, options, prams


def main():
    rng = np.random.default_rng(424242)
    npts = [16, 16, 24, 16, 24, 32]
    fibers, bodies, options, prams = build_system(rng, npts, nbody=2, nb_nodes=80, nper=240,
                                                  R_per=6.0, L=2.0, E=0.0025, dt=1e-3, tol=1e-10)
    fext = rng.normal(scale=0.1, size=(len(npts), 3))
    x0_fib = [f.x.copy() for f in fibers]

    def fake_repulsion(bodies_, x0, offset_fibers, *a, **k):
        ff = np.zeros((offset_fibers[-1], 3))
        for i in range(len(offset_fibers) - 1):
            ff[offset_fibers[i]:offset_fibers[i + 1]] = fext[i]
        return np.zeros((len(bodies_), 6)), ff

    ts.forces.compute_hydro_repulsion_force = fake_repulsion

    rec = {}
    real_gmres = gmres_mod.gmres

    def wrapped(A, b, **kw):
        rec["A"], rec["b"], rec["M"], rec["kw"] = A, b.copy(), kw.get("M"), kw
        sol, info = real_gmres(A, b, **kw)
        rec["sol"], rec["info"] = sol.copy(), info
        return sol, info

    gmres_mod.gmres = wrapped
    T = ts.tstep(prams, options, None, fibers, bodies, None)
    T.time_step_hydro(1e-3)

    out = {}
    out["npts"] = np.array(npts)
    out["fext"] = fext
    out["L"], out["E"], out["dt"], out["eta"], out["tol"] = 2.0, 0.0025, 1e-3, 1.0, 1e-10
    for k, x in enumerate(x0_fib):
        out[f"fib{k}_x"] = x
    for k, b in enumerate(bodies):
        out[f"body{k}_loc"] = b.location          # time_step_hydro only sets location_new
        out[f"body{k}_quat"] = np.array([b.orientation.s, *b.orientation.p])
        out[f"body{k}_ref_nodes"] = b.reference_configuration
        out[f"body{k}_ref_normals"] = b.reference_normals
        out[f"body{k}_w"] = b.quadrature_weights
    out["shell_nodes"] = T.trg_shell_surf
    out["shell_normals"] = T.normals_shell
    out["shell_w"] = T.shell.quadrature_weights
    A, M = rec["A"], rec["M"]
    n = rec["b"].size
    out["rhs"] = rec["b"]
    out["sol"] = rec["sol"]
    out["gmres_info"] = rec["info"]
    X = rng.normal(size=(3, n))
    out["probe_x"] = X
    out["probe_Ax"] = np.stack([A.matvec(x) for x in X])
    out["probe_Px"] = np.stack([M.matvec(x) for x in X])
    np.savez_compressed(HERE / "step_small.npz", **out)
    print("system size", n, "gmres info", rec["info"], "bytes", (HERE / "step_small.npz").stat().st_size)


if __name__ == "__main__":
    main()
