"""Reader for the single-level AMReX plotfiles written by fx_write_plotfile
(the format of WriteSingleLevelPlotfile, Source/Plotfile.cpp:177)."""
from __future__ import annotations

import os
import re

import numpy as np


def read(path: str) -> dict:
    """Return {"names", "time", "step", "n", "prob_lo", "prob_hi", "dx", "fields"}
    where fields[name] has shape (nz, ny, nx)."""
    with open(os.path.join(path, "Header")) as f:
        lines = f.read().split("\n")
    assert lines[0] == "HyperCLaw-V1.1", lines[0]
    nvar = int(lines[1])
    names = lines[2:2 + nvar]
    p = 2 + nvar
    assert int(lines[p]) == 3
    time = float(lines[p + 1])
    assert int(lines[p + 2]) == 0            # finest level
    prob_lo = [float(v) for v in lines[p + 3].split()]
    prob_hi = [float(v) for v in lines[p + 4].split()]
    box = re.findall(r"-?\d+", lines[p + 6])
    hi = [int(v) for v in box[3:6]]
    n = [h + 1 for h in hi]
    step = int(lines[p + 7].split()[0])
    dx = [float(v) for v in lines[p + 8].split()]
    mf = [l for l in lines if l.startswith("Level_0/")][0]
    with open(os.path.join(path, mf + "_H")) as f:
        h = f.read().split("\n")
    fod = [l for l in h if l.startswith("FabOnDisk:")][0].split()
    fname, offset = fod[1], int(fod[2])
    with open(os.path.join(path, "Level_0", fname), "rb") as f:
        f.seek(offset)
        header = f.readline().decode()
        assert header.startswith("FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))"), header
        ncomp = int(header.split()[-1])
        npts = n[0] * n[1] * n[2]
        data = np.frombuffer(f.read(8 * npts * ncomp), dtype="<f8").reshape(ncomp, n[2], n[1], n[0])
    return dict(names=names, time=time, step=step, n=n, prob_lo=prob_lo, prob_hi=prob_hi, dx=dx,
                fields={nm: data[q] for q, nm in enumerate(names)})
