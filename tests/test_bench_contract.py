"""The reference arm of bench.py on the CPU: the JSON line a run prints, no GPU needed.

`bench.py --impl reference` times the restated CPU implementation of the
coupled step on the host's cores.  Its line carries the same metric, unit and
workload naming as the GPU arm, plus `impl`, `cpu_baseline` and an `e2e` with
no host-device bytes.  Under a multi-rank launch only rank 0 runs and prints.
Fewer than 3 warm-up steps are refused.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, capture_output=True, text=True,
                          env=env, timeout=300)


def test_reference_line_keys_and_values():
    r = _bench("--impl", "reference", "--workload", "mfim", "--steps", "2", "--warmup", "3")
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "coupled-step cell-updates/s"
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3 and d["dtype"] == "f64"
    # the reference arm names the same workload as the GPU arm (mixed precision
    # by default) and says that it computes in FP64
    assert d["config"]["workload"] == "mfim-64x64x36-mixed" and d["config"]["cells"] == 64 * 64 * 36
    assert d["reference_precision"].startswith("fp64")
    assert d["config"]["history_steps_at_timed_start"] == 3 and d["config"]["phi_extrapolate_order"] == 4
    assert d["value"] > 0 and abs(d["value"] - 64 * 64 * 36 / (d["ms_per_step"] * 1e-3)) <= 1e-6 * d["value"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    r = _bench("--impl", "reference", "--workload", "mfim", "--steps", "1", "--warmup", "3",
               env_extra={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_fewer_than_three_warmup_steps_are_refused():
    r = _bench("--impl", "reference", "--workload", "mfim", "--steps", "1", "--warmup", "2")
    assert r.returncode != 0 and "--warmup must be >= 3" in r.stderr
