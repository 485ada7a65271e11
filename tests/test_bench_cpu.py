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


def test_default_reference_arm_prints_one_line():
    """bench.py's reference arm (`--impl reference`), timed beside the GPU
    one: the C restatement of fiber3d's pair loop on the default workload's
    metric and config."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3",
           "--cpu-seconds", "0.5"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "Stokes pair interactions per second (FP64)"
    assert d["unit"] == "pairs/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "stresslet_sphere"
    # the same config dict as the GPU arm's (bench.workload_config)
    assert set(d["config"]) == {"workload", "description", "pairs_per_step", "l2"}
    cb = d["cpu_baseline"]
    assert cb["cores"] == cb["threads"] and "physical_cores" in cb
    assert d["e2e"] == {"value": d["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 runs the reference arm; the others exit 0
    and print nothing."""
    import os
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=120, cwd=ROOT, env=env)
    assert res.returncode == 0, res.stderr
    assert not [ln for ln in res.stdout.splitlines() if ln.startswith("{")]


def test_fmm_reference_arm_prints_one_line():
    """The FMM workload's reference arm (fiber3d's direct sums, which its
    STKFMM path is checked against) on a small case: one line, the FMM
    arm's metric and config keys."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "fmm",
           "--fmm-n", "5000", "--steps", "1", "--warmup", "1"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "pairs/s" and d["higher_is_better"] is True
    assert d["metric"].startswith("FMM equivalent Stokes pair interactions per second")
    c = d["config"]
    assert c["workload"] == "fmm" and c["n_single_layer"] == c["n_double_layer"] == c["n_targets"] == 5000
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
