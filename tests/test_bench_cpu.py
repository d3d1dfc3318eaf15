"""bench.py on the CPU: the workload arithmetic the JSON line is built from,
the reference arm's line (the oracle on the host cores), and option checks."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_face_states_and_algorithmic_bytes():
    import bench
    # 200^3 x 8, buff 6: N = 212, NC = 206 -> 2 x 206 x 212^2 x 8 per direction
    assert bench.face_states_per_dir(order=5) == 148_135_424
    assert 3 * bench.face_states_per_dir(order=5) == 444_406_272
    # WENO3 writes every face of the sweep
    assert bench.face_states_per_dir(order=3) == 2 * 212 ** 3 * 8
    # (NC + 4) N^2 V + 2 NC N^2 V doubles for WENO5 + MP
    assert bench.alg_bytes_per_sweep(order=5) == 1_789_130_752
    assert bench.alg_bytes_per_sweep(order=7) == (206 + 6) * 212 ** 2 * 8 * 8 + 2 * 206 * 212 ** 2 * 8 * 8
    assert bench.alg_bytes_per_sweep(order=5, elem=4) * 2 == bench.alg_bytes_per_sweep(order=5)


def _run(*args, timeout=600):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          timeout=timeout, cwd=ROOT)


def test_reference_arm_line():
    # a 64^3 block keeps the CPU suite short; the arm runs at least warmup 5
    # and 10 timed steps whatever is asked
    r = _run("--impl", "reference", "--steps", "1", "--warmup", "0", "--m", "63")
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["unit"] == "face-states/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["steps_run"] >= 10 and line["warmup_run"] >= 5
    assert line["cpu"]["nproc"] >= 1 and line["cpu"]["model"]
    assert "8 of 8 variables" in line["cpu_baseline"]["sample"]


def test_weno3_teno_refused():
    r = _run("--order", "3", "--scheme", "teno", timeout=120)
    assert r.returncode != 0 and "TENO" in r.stderr
