"""The `ferrox_b200` executable without a GPU: usage, unreadable inputs, command-line
overrides (`key=value` after the inputs file, applied after it, as FerroX's own
command line does), and a refusal to run on the CPU when no device is present."""
from __future__ import annotations

import os
import subprocess

import pytest

from ferrox_b200 import decks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "ferrox_b200", "ferrox_b200")


def _run(*args):
    # the executable is a build output (not tracked): build it from the current sources
    from ferrox_b200 import build
    build.build()
    if not os.path.exists(EXE):
        pytest.fail("ferrox_b200 executable not built")
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=120)


def test_usage_and_missing_file():
    r = _run()
    assert r.returncode != 0 and "usage:" in r.stderr
    r = _run("/nonexistent/inputs")
    assert r.returncode != 0 and "cannot open" in r.stderr


def test_command_line_overrides_come_after_the_file(tmp_path):
    deck = tmp_path / "inputs"
    deck.write_text(decks.mfim(8, 8, 12, nsteps=2) + "prob_type = 9\n")
    r = _run(str(deck))
    assert r.returncode != 0 and "prob_type" in r.stderr
    good = _run(str(deck), "prob_type=2")          # the override replaces the bad value
    assert "prob_type" not in good.stderr
    bad = _run(str(tmp_path / "inputs"), "prob_type=2", "TimeIntegratorOrder=3")
    assert bad.returncode != 0 and "TimeIntegratorOrder" in bad.stderr


def test_no_cpu_fallback_without_a_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    deck = tmp_path / "inputs"
    deck.write_text(decks.mfim(8, 8, 12, nsteps=2))
    r = _run(str(deck))
    assert r.returncode != 0 and "no usable CUDA device" in r.stderr
    assert not any(p.startswith("plt") for p in os.listdir(tmp_path))
