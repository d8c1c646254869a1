"""The C boundary as a C or C++ host sees it, no GPU needed.

include/ferrox_b200.h is what a C host, a cgo preamble or a JNI/N-API shim
includes.  A small program includes it, is built with gcc as strict C99 and with
g++ as C++17 (the header's extern "C" guards), links libferrox_b200.so, and runs
the create / query / step / destroy calls.  The deck is read from a file, its dims
and dt come back, and fx_step returns FX_ERR_CUDA (no usable device) when no GPU is present.
"""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from ferrox_b200 import decks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ferrox_b200")

PROGRAM = r"""
#include "ferrox_b200.h"
#include <stdio.h>
int main(int argc, char** argv) {
    fx_ctx* ctx = NULL;
    int n[3];
    double dx[3], dt = 0.0;
    int rc;
    if (argc < 2) return 2;
    if (fx_create(argv[1], 0, &ctx) != FX_OK) { fprintf(stderr, "create: %s\n", fx_create_error()); return 3; }
    if (fx_get_dims(ctx, n, dx) != FX_OK) return 4;
    if (fx_get_param(ctx, "dt", &dt) != FX_OK) return 5;
    rc = fx_step(ctx, 1, NULL);
    printf("%d %d %d %.17g %d\n", n[0], n[1], n[2], dt, rc);
    fx_destroy(ctx);
    return 0;
}
"""


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++17")])
def test_header_compiles_links_and_runs(tmp_path, compiler, std):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    src = tmp_path / ("main.c" if compiler == "gcc" else "main.cpp")
    src.write_text(PROGRAM)
    exe = tmp_path / "host"
    subprocess.run([compiler, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", LIBDIR, "-lferrox_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    deck = tmp_path / "inputs"
    deck.write_text(decks.mfim(8, 8, 12, nsteps=2))
    r = subprocess.run([str(exe), str(deck)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    nx, ny, nz, dt, rc = r.stdout.split()
    assert (int(nx), int(ny), int(nz)) == (8, 8, 12) and float(dt) == 1.0e-13
    import torch
    assert int(rc) == (0 if torch.cuda.is_available() else -4)   # FX_ERR_CUDA
