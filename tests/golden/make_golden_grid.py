"""Golden vectors of fiber3d's grid-velocity evaluation (needs the fiber3d
sources; see refshim.py).

    python tests/golden/make_golden_grid.py

Runs fiber3d's own ``tstep.time_step_hydro`` with ``iComputeVelocity`` on
(tstep/tstep.py:1238-1456) for the system of ``make_golden_step.py`` (same
seed, same fibers, bodies and periphery), and reads back the grid points and
velocities the reference writes (``<output_name>_grid_points.txt`` and
``_velocity_at_grid.txt``, tstep.py:177-181, 1454-1456).  The velocity is
the periphery and body double layers, the fibers' Oseen flow with the
near-fiber replacement, the external-force flow, and the rigid motion
inside the first body.  Writes ``grid_small.npz`` with the GMRES solution
and a subset of the grid: every point within 0.25 of a fiber node or inside
the first body, and every 16th other point.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

import make_golden_step as mgs  # noqa: E402  (installs the shims)

from tstep import tstep as ts  # noqa: E402
from bpm_utilities import gmres as gmres_mod  # noqa: E402

OUT = "/tmp/f3d_golden_grid"


def main():
    rng = np.random.default_rng(424242)
    npts = [16, 16, 24, 16, 24, 32]
    fibers, bodies, options, prams = mgs.build_system(rng, npts, nbody=2, nb_nodes=80, nper=240,
                                                      R_per=6.0, L=2.0, E=0.0025, dt=1e-3, tol=1e-10)
    fext = rng.normal(scale=0.1, size=(len(npts), 3))
    options.iComputeVelocity = True
    options.output_name = OUT
    x_fib = [f.x.copy() for f in fibers]

    def fake_repulsion(bodies_, x0, offset_fibers, *a, **k):
        ff = np.zeros((offset_fibers[-1], 3))
        for i in range(len(offset_fibers) - 1):
            ff[offset_fibers[i]:offset_fibers[i + 1]] = fext[i]
        return np.zeros((len(bodies_), 6)), ff

    ts.forces.compute_hydro_repulsion_force = fake_repulsion
    rec = {}
    real_gmres = gmres_mod.gmres

    def wrapped(A, b, **kw):
        sol, info = real_gmres(A, b, **kw)
        rec["sol"], rec["info"] = sol.copy(), info
        return sol, info

    gmres_mod.gmres = wrapped
    T = ts.tstep(prams, options, None, fibers, bodies, None)
    T.time_step_hydro(1e-3)
    T.f_grid_velocity.close()
    T.f_grid_points.close()
    grid = np.loadtxt(OUT + "_grid_points.txt").reshape(-1, 3)
    vel = np.loadtxt(OUT + "_velocity_at_grid.txt").reshape(-1, 3)
    allx = np.concatenate(x_fib)
    near = np.zeros(grid.shape[0], dtype=bool)
    for i in range(0, grid.shape[0], 4096):
        d = np.linalg.norm(grid[i:i + 4096, None, :] - allx[None, :, :], axis=2)
        near[i:i + 4096] = (d <= 0.25).any(axis=1)
    b0 = bodies[0]
    inside = np.linalg.norm(grid - b0.location_new, axis=1) <= 0.5 + 1e-9
    keep = near | inside | (np.arange(grid.shape[0]) % 16 == 0)
    out = {"sol": rec["sol"], "grid_index": np.nonzero(keep)[0], "grid_points": grid[keep],
           "grid_velocity": vel[keep], "grid_count": np.array(grid.shape[0]),
           "body0_radius": np.array(0.5)}
    np.savez_compressed(HERE / "grid_small.npz", **out)
    print("grid points", grid.shape[0], "kept", int(keep.sum()), "near fibers", int(near.sum()),
          "inside body 0", int(inside.sum()), "bytes", (HERE / "grid_small.npz").stat().st_size)


if __name__ == "__main__":
    main()
