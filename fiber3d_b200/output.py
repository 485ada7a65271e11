"""fiber3d's output and restart files for runs marched on the device.

fiber3d writes its state every ``n_save`` steps with
``tstep.write_to_file`` (python/tstep/tstep.py:2027-2200) into the files
``initialize_from_file`` opens (python/tstep/initialize.py:612-660); its
MATLAB post-processing and its restart path read them.  A run that goes
through ``tstep_bridge`` keeps fiber3d's own writer.  A run marched with
:class:`fiber3d_b200.hydro.HydroSystem` alone writes the same files here, byte
for byte (same names, number formats and line layouts):

* ``<out>_<ID>_fibers.txt`` (``<out>_<ID>.fibers`` without ``txt``): per
  save, the fiber count, then per fiber ``num_points E length growing`` and
  its ``x y z tension`` rows;
* ``<out>_<ID>_clones.txt`` (``.clones``): per save, per body its location
  and quaternion (with the count and radius rows in the txt form);
* ``<out>_<ID>velocity_clones.txt``: per save, per body U and Omega;
* ``<out>_time_system_size.txt``: per save, ``dt, time, accepted steps,
  rejected steps[, periphery radius | a b c | cortex radius], n_save``;
* the restart files, rewritten at every save: ``<out>_<ID>_resume.fibers``,
  ``_resume.clones``, ``_attached_to_body.fibers``, ``_nuc_site_idx.fibers``,
  ``_length_before_die.fibers`` and each body type's (empty unless the
  bodies carry nucleation sites) ``<out>-<ID>_active_site_idcs.clones`` /
  ``_passive_site_idcs.clones``.

Molecular motors, peripheral nucleation and motor-driven bodies are outside
the hydrodynamic solve and have no files here.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class FiberRecord:
    """What fiber3d writes of one fiber (python/fiber/fiber.py attributes)."""
    x: np.ndarray                 # (N, 3)
    tension: np.ndarray           # (N,)
    E: float
    length: float
    growing: int = 0
    attached_to_body: int = -1
    nuc_site_idx: int = -1
    length_before_die: float = float("nan")

    @property
    def num_points(self) -> int:
        return int(np.asarray(self.x).shape[0])


@dataclass
class BodyRecord:
    """What fiber3d writes of one rigid body (python/body/body.py attributes)."""
    location: np.ndarray          # (3,)
    orientation: np.ndarray       # quaternion (4,), scalar first
    velocity: np.ndarray = field(default_factory=lambda: np.zeros(3))
    angular_velocity: np.ndarray = field(default_factory=lambda: np.zeros(3))
    radius: float | None = None
    active_sites_idcs: np.ndarray | None = None
    passive_sites_idcs: np.ndarray | None = None


def _row(a) -> np.ndarray:
    return np.asarray(a)[None, :]


class OutputWriter:
    """Writes fiber3d's files for one fiber type and one body type (the
    names fiber3d gives them when read from an input file are the type
    IDs, ``fibers_id`` and ``bodies_id``)."""

    def __init__(self, output_name: str, txt: bool, dt: float, n_save: int, *, fibers_id: str | None = "one",
                 bodies_id: str | None = "one", periphery_radius: float | None = None,
                 periphery_abc: tuple | None = None, cortex_radius: float | None = None):
        self.out = output_name
        self.txt = bool(txt)
        self.dt, self.n_save = dt, n_save
        self.fibers_id, self.bodies_id = fibers_id, bodies_id
        self.periphery_radius, self.periphery_abc, self.cortex_radius = periphery_radius, periphery_abc, cortex_radius
        buf = 100  # fiber3d's buffering (initialize.py:612)
        self.f_fibers = self.f_bodies = self.f_vels = None
        if fibers_id is not None:
            name = f"{self.out}_{fibers_id}_fibers.txt" if self.txt else f"{self.out}_{fibers_id}.fibers"
            self.f_fibers = open(name, "wb", buffering=buf)
        if bodies_id is not None:
            name = f"{self.out}_{bodies_id}_clones.txt" if self.txt else f"{self.out}_{bodies_id}.clones"
            self.f_bodies = open(name, "wb", buffering=buf)
            self.f_vels = open(f"{self.out}_{bodies_id}velocity_clones.txt", "wb", buffering=buf)
        self.f_time = open(f"{self.out}_time_system_size.txt", "wb", buffering=buf)

    # ------------------------------------------------------------------
    def _time_row(self, current_time, step, steps_rejected) -> np.ndarray:
        head = [self.dt, current_time, step - steps_rejected, steps_rejected]
        if self.periphery_abc is not None:
            return np.array(head + list(self.periphery_abc) + [self.n_save])
        if self.periphery_radius is not None:
            return np.array(head + [self.periphery_radius, self.n_save])
        if self.cortex_radius is not None:
            return np.array(head + [self.cortex_radius, self.n_save])
        return np.array(head + [self.n_save])

    @staticmethod
    def _pose_line(b: BodyRecord) -> bytes:
        v = [b.location[0], b.location[1], b.location[2], *[b.orientation[i] for i in range(4)]]
        return (" ".join("%s" % e for e in v) + " \n").encode("utf-8")

    def write(self, current_time: float, step: int, steps_rejected: int, fibers: list, bodies: list) -> None:
        """One save: ``fibers`` a list of :class:`FiberRecord`, ``bodies`` a
        list of :class:`BodyRecord` (fiber3d's ``write_to_file``)."""
        np.savetxt(self.f_time, _row(self._time_row(current_time, step, steps_rejected)))
        if self.bodies_id is not None:
            self._write_bodies(bodies)
        if self.fibers_id is not None:
            self._write_fibers(fibers)

    def _write_bodies(self, bodies):
        ID, n = self.bodies_id, len(bodies)
        with open(f"{self.out}_{ID}_resume.clones", "wb") as resume, \
                open(f"{self.out}-{ID}_passive_site_idcs.clones", "wb") as passive, \
                open(f"{self.out}-{ID}_active_site_idcs.clones", "wb") as active:
            resume.write(("%s \n" % n).encode("utf-8"))
            if self.txt:
                np.savetxt(self.f_bodies, np.ones((1, 7), dtype=int) * n)
                np.savetxt(self.f_vels, np.ones((1, 6), dtype=int) * n)
            for b in bodies:
                if self.txt:
                    np.savetxt(self.f_bodies, np.ones((1, 7), dtype=int) * b.radius)
                    np.savetxt(self.f_bodies, _row([*b.location[:3], *b.orientation[:4]]))
                else:
                    self.f_bodies.write(self._pose_line(b))
                np.savetxt(self.f_vels, _row([*b.velocity[:3], *b.angular_velocity[:3]]))
                if b.active_sites_idcs is not None:
                    np.savetxt(active, b.active_sites_idcs)
                    np.savetxt(passive, b.passive_sites_idcs)
                resume.write(self._pose_line(b))

    def _write_fibers(self, fibers):
        ID, n = self.fibers_id, len(fibers)
        attached = np.array([f.attached_to_body for f in fibers], dtype=np.int32)
        nuc = np.array([f.nuc_site_idx for f in fibers], dtype=np.int32)
        before_die = np.array([f.length_before_die for f in fibers], dtype=np.float64)
        for suffix, arr in (("attached_to_body", attached), ("nuc_site_idx", nuc),
                            ("length_before_die", before_die)):
            with open(f"{self.out}_{ID}_{suffix}.fibers", "wb") as fh:
                np.savetxt(fh, arr)
        with open(f"{self.out}_{ID}_resume.fibers", "wb") as resume:
            resume.write(("%s \n" % n).encode("utf-8"))
            if self.txt:
                np.savetxt(self.f_fibers, np.ones((1, 4), dtype=int) * n)
            else:
                self.f_fibers.write((str(n) + "\n").encode("utf-8"))
            for f in fibers:
                info = (f.num_points, f.E, f.length, f.growing)
                if self.txt:
                    np.savetxt(self.f_fibers, _row(np.array(info)))
                else:
                    self.f_fibers.write(("%s %s %s %s \n" % info).encode("utf-8"))
                np.savetxt(self.f_fibers, np.concatenate((np.asarray(f.x), np.asarray(f.tension)[:, None]), axis=1))
                resume.write(("%s %s %s %s \n" % info).encode("utf-8"))
                np.savetxt(resume, np.asarray(f.x))

    def close(self) -> None:
        for fh in (self.f_fibers, self.f_bodies, self.f_vels, self.f_time):
            if fh is not None:
                fh.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def records_from_solution(system, sol, E: float, lengths, body_radius=None):
    """FiberRecords and BodyRecords of a HydroSystem after ``advance(sol)``:
    fiber positions and tensions are the solution's fiber blocks (x_1..N,
    y_1..N, z_1..N, T_1..N per fiber, fiber3d's layout), body locations and
    orientations the advanced ones, body velocities the solution's U and
    Omega."""
    x = sol.detach().cpu().numpy() if hasattr(sol, "detach") else np.asarray(sol)
    fibers = []
    for k in range(system.fs.nfib):
        n, p0 = int(system.fs.npts[k]), int(system.fs.pt_off_h[k])
        blk = x[system.o_fib + 4 * p0:system.o_fib + 4 * (p0 + n)].reshape(4, n)
        fibers.append(FiberRecord(x=blk[:3].T.copy(), tension=blk[3].copy(), E=E, length=float(lengths[k])))
    locs, quats = system.body_state()
    bodies = []
    for k in range(system.nbody):
        o = system.o_body[k] + 3 * int(system.nb[k])
        bodies.append(BodyRecord(location=locs[k], orientation=quats[k], velocity=x[o:o + 3].copy(),
                                 angular_velocity=x[o + 3:o + 6].copy(),
                                 radius=None if body_radius is None else body_radius[k]))
    return fibers, bodies
