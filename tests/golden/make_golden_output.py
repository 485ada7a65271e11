"""Golden output files of fiber3d's writer (needs the fiber3d sources; see
refshim.py).

    python tests/golden/make_golden_output.py

Calls fiber3d's own ``tstep.write_to_file`` (tstep/tstep.py:2027-2200) on a
stand-in holding exactly the attributes it reads: 3 fibers (4, 5 and 4
points), 2 rigid bodies of radius 0.5, a periphery of radius 6, dt 1e-3,
n_save 1, with the files opened under the names ``initialize_from_file``
gives them (tstep/initialize.py:612-647).  Two saves (step 0 and step 1
with moved fibers and bodies), in the txt form and in the ``.fibers`` /
``.clones`` form.  Writes every file's bytes to ``output.npz`` (keys
``<form>/<file name>``) and the state to ``output_state.npz``.
"""
from __future__ import annotations

import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import refshim  # noqa: E402

sys.path.insert(0, refshim.install())

from tstep import tstep as ts  # noqa: E402


def state(rng):
    npts = [4, 5, 4]
    x = [rng.normal(size=(n, 3)) for n in npts]
    t = [rng.normal(size=n) for n in npts]
    loc = rng.normal(size=(2, 3))
    q = rng.normal(size=(2, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    vel = rng.normal(size=(2, 3))
    ang = rng.normal(size=(2, 3))
    return x, t, loc, q, vel, ang


def stand_in(out, txt, st, handles=None):
    x, t, loc, q, vel, ang = st
    S = types.SimpleNamespace()
    S.output_name, S.output_txt_files = out, txt
    S.dt, S.n_save = 1e-3, 1
    S.cortex_radius, S.periphery_radius, S.periphery_a = None, 6.0, None
    S.iPeripheralNucleation = False
    S.fibers_names, S.fibers_types = ["one"], [3]
    S.body_names, S.body_types = ["one"], [2]
    S.bodies_names_mm_attached, S.bodies_types_mm_attached = [], []
    S.f_bodies_mm_attached_ID, S.f_mm_on_moving_surf_ID, S.f_molecular_motors_ID = [], [], []
    S.fibers = [types.SimpleNamespace(x=x[k], tension=t[k], num_points=len(x[k]), E=0.0025,
                                      length=[1.0, 2.0, 1.5][k], growing=0, attached_to_body=-1,
                                      nuc_site_idx=-1, length_before_die=None) for k in range(3)]
    S.bodies = [types.SimpleNamespace(location=loc[k], orientation=types.SimpleNamespace(entries=q[k]),
                                      velocity=vel[k], angular_velocity=ang[k], radius=0.5,
                                      active_sites_idcs=None, passive_sites_idcs=None) for k in range(2)]
    if handles is None:  # the files stay open across saves, as in fiber3d
        handles = ([open(out + ("_one_fibers.txt" if txt else "_one.fibers"), "wb", buffering=100)],
                   [open(out + ("_one_clones.txt" if txt else "_one.clones"), "wb", buffering=100)],
                   [open(out + "_onevelocity_clones.txt", "wb", buffering=100)],
                   open(out + "_time_system_size.txt", "wb", buffering=100))
    S.f_fibers_ID, S.f_bodies_ID, S.f_body_vels_ID, S.f_time_system = handles
    return S


def main():
    rng = np.random.default_rng(99)
    s0, s1 = state(rng), state(rng)
    files = {}
    for form, txt in (("txt", True), ("bin", False)):
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "run")
            S = stand_in(out, txt, s0)
            ts.tstep.write_to_file(S, 0.0, 0, 0)
            S1 = stand_in(out, txt, s1, (S.f_fibers_ID, S.f_bodies_ID, S.f_body_vels_ID, S.f_time_system))
            ts.tstep.write_to_file(S1, 1e-3, 1, 0)
            for fh in (*S.f_fibers_ID, *S.f_bodies_ID, *S.f_body_vels_ID, S.f_time_system):
                fh.close()
            for f in sorted(os.listdir(d)):
                files[f"{form}/{f}"] = np.frombuffer(Path(d, f).read_bytes(), dtype=np.uint8)
    np.savez_compressed(HERE / "output.npz", **files)
    st = {}
    for i, s in enumerate((s0, s1)):
        x, t, loc, q, vel, ang = s
        for k in range(3):
            st[f"s{i}_x{k}"], st[f"s{i}_t{k}"] = x[k], t[k]
        st[f"s{i}_loc"], st[f"s{i}_q"], st[f"s{i}_vel"], st[f"s{i}_ang"] = loc, q, vel, ang
    np.savez_compressed(HERE / "output_state.npz", **st)
    print(sorted(files))


if __name__ == "__main__":
    main()
