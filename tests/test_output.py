"""fiber3d's output and restart files written by fiber3d_b200.output,
byte for byte against fiber3d's own writer (tests/golden/output.npz, from
make_golden_output.py)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import load_golden
from fiber3d_b200.output import BodyRecord, FiberRecord, OutputWriter


def _records(st, i):
    fibers = [FiberRecord(x=st[f"s{i}_x{k}"], tension=st[f"s{i}_t{k}"], E=0.0025, length=[1.0, 2.0, 1.5][k])
              for k in range(3)]
    bodies = [BodyRecord(location=st[f"s{i}_loc"][k], orientation=st[f"s{i}_q"][k], velocity=st[f"s{i}_vel"][k],
                         angular_velocity=st[f"s{i}_ang"][k], radius=0.5) for k in range(2)]
    return fibers, bodies


@pytest.mark.parametrize("form", ["txt", "bin"])
def test_files_match_fiber3d(tmp_path, form):
    gold = load_golden("output.npz")
    st = load_golden("output_state.npz")
    out = str(tmp_path / "run")
    with OutputWriter(out, form == "txt", 1e-3, 1, periphery_radius=6.0) as w:
        w.write(0.0, 0, 0, *_records(st, 0))
        w.write(1e-3, 1, 0, *_records(st, 1))
    want = {k.split("/", 1)[1]: v.tobytes() for k, v in gold.items() if k.startswith(form + "/")}
    got = {f: (tmp_path / f).read_bytes() for f in os.listdir(tmp_path)}
    assert sorted(got) == sorted(want)
    for name in want:
        assert got[name] == want[name], name


def test_time_row_variants(tmp_path):
    out = str(tmp_path / "r")
    with OutputWriter(out, True, 0.5, 3, fibers_id=None, bodies_id=None, periphery_abc=(1.0, 2.0, 3.0)) as w:
        w.write(1.5, 4, 1, [], [])
    row = np.loadtxt(out + "_time_system_size.txt")
    assert list(row) == [0.5, 1.5, 3, 1, 1.0, 2.0, 3.0, 3]
    with OutputWriter(out, True, 0.5, 3, fibers_id=None, bodies_id=None, cortex_radius=4.0) as w:
        w.write(1.5, 4, 1, [], [])
    assert list(np.loadtxt(out + "_time_system_size.txt")) == [0.5, 1.5, 3, 1, 4.0, 3]
