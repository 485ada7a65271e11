"""bench.py's host-only paths run without a GPU: the reference arm of the
surface quadrature workload prints one JSON line of the contract's shape."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_quadrature_reference_arm_prints_one_line():
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "surface_quadrature",
           "--nshell", "400", "--steps", "1", "--warmup", "1", "--cpu-seconds", "0.2"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["config"]["workload"] == "surface_quadrature" and d["config"]["triangles"] == 796
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] == 1
