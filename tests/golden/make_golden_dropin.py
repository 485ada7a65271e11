"""Golden vectors for the rest of fiber3d's ``kernels.kernels`` module, made
by running fiber3d's own functions (needs the fiber3d sources; set
FIBER3D_REFERENCE to their ``python/`` folder).

    python tests/golden/make_golden_dropin.py

Writes dropin.npz next to this file:
  traction_*     traction_kernel_times_normal_times_density_numba
                 (kernels.py:1221-1264), default and non-default eta
  stk_*          stresslet_kernel (kernels.py:911-992), 'r' and 'xyz' input
  stkn_*         stresslet_kernel_times_normal (kernels.py:995-1060)
  pyc_*          oseen_kernel_source_target_pycuda (kernels.py:849): PyCUDA is
                 absent here, so its result is formed from fiber3d's numba
                 Oseen sum (kernels.py:794-846) per target over the sources at
                 distance >= epsilon_distance -- the pairs the PyCUDA kernel
                 keeps (kernels_pycuda.py:52-53)
  fmm_*          the three *_stkfmm functions (kernels.py:1298-1485): STKFMM is
                 absent here, so the reference value is the direct sum fiber3d
                 checks its FMM against (kernels/test_stkfmm.py: numba Oseen
                 and stresslet source -> target sums), per target over the
                 sources that do not coincide with it (an FMM kernel leaves a
                 coincident pair out)
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

from kernels import kernels as K  # noqa: E402  (fiber3d)

from fiber3d_b200 import geometry  # noqa: E402


def filtered_sum(fn, xs, xt, keep, *dens):
    """fn(xs[keep_t], xt[t], *dens[keep_t]) target by target."""
    out = np.zeros((xt.shape[0], 3))
    for t in range(xt.shape[0]):
        m = keep(np.linalg.norm(xt[t] - xs, axis=1))
        if m.any():
            out[t] = fn(xs[m], xt[t:t + 1], *[d[m] for d in dens])
    return out.reshape(-1)


def main():
    rng = np.random.default_rng(20261204)
    out = {}
    # traction: duplicated point (regularised), a sub-epsilon pair, tile tails
    x = rng.random((150, 3)); x[5] = x[6]; x[40] = x[41] + 3e-6
    n = geometry.uniform_directions(rng, 150); d = rng.normal(size=(150, 3))
    out["traction_r"], out["traction_n"], out["traction_d"] = x, n, d
    out["traction_v"] = K.traction_kernel_times_normal_times_density_numba(x, n, d)
    out["traction_v_eta"] = K.traction_kernel_times_normal_times_density_numba(x, n, d, 2.5, 1e-2, 1e-4)
    # 3-index stresslet tensor
    x = rng.random((24, 3)); x[3] = x[4]; x[7] = x[8] + 2e-6
    out["stk_r"] = x
    out["stk_S"] = K.stresslet_kernel(x)
    out["stk_S_xyz"] = K.stresslet_kernel(x.T.flatten(), input_format='xyz')
    out["stk_S_eta"] = K.stresslet_kernel(x, 3.0, 1e-2, 1e-4)
    # numpy stresslet times normal
    x = rng.random((40, 3)); x[2] = x[9] + 1e-6
    n = geometry.uniform_directions(rng, 40)
    out["stkn_r"], out["stkn_n"] = x, n
    out["stkn_M"] = K.stresslet_kernel_times_normal(x, n)
    # PyCUDA Oseen: pairs closer than eps skipped (coincident and sub-eps targets)
    xs = rng.random((140, 3)); xt = rng.random((130, 3))
    xt[:3] = xs[:3]
    xt[3:5] = xs[3:5] + 3e-6 * rng.normal(size=(2, 3))
    f = rng.normal(size=(140, 3))
    out["pyc_rs"], out["pyc_rt"], out["pyc_f"] = xs, xt, f
    out["pyc_u"] = filtered_sum(K.oseen_kernel_source_target_numba, xs, xt, lambda r: r >= 1e-5, f)
    # STKFMM stand-ins: coincident points left out (no sub-eps pairs here)
    xs = rng.random((150, 3)); xt = rng.random((120, 3)); xt[:4] = xs[10:14]
    f = rng.normal(size=(150, 3))
    nd = geometry.uniform_directions(rng, 150); dd = rng.normal(size=(150, 3))
    out["fmm_rs"], out["fmm_rt"], out["fmm_f"], out["fmm_n"], out["fmm_d"] = xs, xt, f, nd, dd
    out["fmm_oseen_u"] = filtered_sum(K.oseen_kernel_source_target_numba, xs, xt, lambda r: r > 0, f)
    out["fmm_stresslet_v"] = filtered_sum(
        lambda s, t, nn, dn: K.stresslet_kernel_source_target_numba(s, t, nn, dn), xs, xt, lambda r: r > 0, nd, dd)
    xdl = rng.random((90, 3)); xdl[0] = xt[20]
    ndl = geometry.uniform_directions(rng, 90); ddl = rng.normal(size=(90, 3))
    out["fmm_rdl"], out["fmm_ndl"], out["fmm_ddl"] = xdl, ndl, ddl
    out["fmm_sdl_u"] = (filtered_sum(K.oseen_kernel_source_target_numba, xs, xt, lambda r: r > 0, f)
                        + filtered_sum(lambda s, t, nn, dn: K.stresslet_kernel_source_target_numba(s, t, nn, dn),
                                       xdl, xt, lambda r: r > 0, ndl, ddl))
    out["fmm_eta_u"] = filtered_sum(lambda s, t, ff: K.oseen_kernel_source_target_numba(s, t, ff, 2.0),
                                    xs, xt, lambda r: r > 0, f)
    np.savez_compressed(HERE / "dropin.npz", **out)
    print("dropin.npz", (HERE / "dropin.npz").stat().st_size)


if __name__ == "__main__":
    main()
