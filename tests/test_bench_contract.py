"""The reference arm of bench.py runs on the host: its JSON line keeps the
contract (one line; impl, metric, value, unit, e2e with no copies, the CPU
baseline describing the run) at small sizes."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    env = dict(os.environ, REFERENCE_BUDGET_S="20")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                         capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def _check_reference_line(line):
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["host"]["nproc"] >= 1
    assert line["backward_error"] < 1e-10


def test_reference_arm_plane_stress_small():
    line = _run("--impl", "reference", "--nel", "12", "--steps", "2", "--warmup", "1")
    _check_reference_line(line)
    assert line["unit"] == "factor+solve/s"
    assert "12x12" in line["config"]["workload"]


def test_reference_arm_batched_small():
    line = _run("--impl", "reference", "--workload", "batched", "--systems", "8", "--steps", "2",
                "--warmup", "1")
    _check_reference_line(line)
    assert line["unit"] == "batch factor+solve/s"
    assert line["inertia_all_expected"] is True
