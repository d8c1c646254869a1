"""Host-side tests of the plotfile writer (csrc/plotfile.cpp), no GPU needed.

The writer produces the single-level AMReX plotfile that FerroX writes through
WriteSingleLevelPlotfile (Source/Plotfile.cpp:177).  It is plain C++ inside the
library, so these tests compile it with g++ next to a small C shim and read
its output back with ferrox_b200.plotfile: field order and x-fastest layout on a
ragged box, exact round trip of every double in the data and the geometry, the
VisMF header's box and min/max lines, the pltNNNNNNNN name and the error path.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from ferrox_b200 import plotfile

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "ferrox_b200", "csrc")

SHIM = r"""
#include "plotfile.h"
#include <cstring>
extern "C" int pf_write(const char* dir, const int* n, const double* lo, const double* hi,
                        const double* dx, double time, int step, int ncomp,
                        const char* const* names, const double* const* comps,
                        char* err, int errlen) {
    fx::PlotGeom g;
    for (int d = 0; d < 3; ++d) { g.n[d] = n[d]; g.prob_lo[d] = lo[d]; g.prob_hi[d] = hi[d]; g.dx[d] = dx[d]; }
    g.time = time; g.step = step;
    std::vector<std::string> nm(names, names + ncomp);
    std::vector<const double*> c(comps, comps + ncomp);
    std::string e;
    int rc = fx::write_plotfile(dir, g, nm, c, &e);
    std::strncpy(err, e.c_str(), errlen - 1); err[errlen - 1] = 0;
    return rc;
}
extern "C" void pf_name(int step, char* out, int len) {
    std::strncpy(out, fx::plotfile_name(step).c_str(), len - 1); out[len - 1] = 0;
}
"""


@pytest.fixture(scope="module")
def writer(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    d = tmp_path_factory.mktemp("pfshim")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    so = d / "libpfshim.so"
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-I", CSRC, str(src),
                    os.path.join(CSRC, "plotfile.cpp"), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.pf_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), dp, dp, dp, ctypes.c_double,
                             ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                             ctypes.POINTER(dp), ctypes.c_char_p, ctypes.c_int]
    lib.pf_write.restype = ctypes.c_int
    lib.pf_name.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    return lib


def _write(lib, path, n, lo, dx, time, step, fields):
    """fields: {name: float64 array of n[0]*n[1]*n[2], x fastest}."""
    arr3 = lambda v: (ctypes.c_double * 3)(*v)
    hi = [lo[d] + n[d] * dx[d] for d in range(3)]
    names = (ctypes.c_char_p * len(fields))(*[k.encode() for k in fields])
    bufs = [np.ascontiguousarray(v, dtype=np.float64) for v in fields.values()]
    dp = ctypes.POINTER(ctypes.c_double)
    comps = (dp * len(bufs))(*[b.ctypes.data_as(dp) for b in bufs])
    err = ctypes.create_string_buffer(256)
    rc = lib.pf_write(str(path).encode(), (ctypes.c_int * 3)(*n), arr3(lo), arr3(hi), arr3(dx), time, step,
                      len(bufs), names, comps, err, 256)
    return rc, err.value.decode(), hi


def test_roundtrip_ragged_box_is_bit_exact(writer, tmp_path):
    n = [5, 3, 7]                                   # every extent different: catches a transposed layout
    npts = n[0] * n[1] * n[2]
    rng = np.random.default_rng(7)
    idx = np.arange(npts, dtype=np.float64)
    fields = {
        "Pz": rng.standard_normal(npts) * 0.3,
        "Phi": idx * 1.0e-3 - 0.01,                 # value encodes the flat x-fastest index
        "rho": np.where(idx % 2 == 0, -0.0, 1.0 / 3.0) * 1.602176634e-19,
    }
    lo = [-2.0e-9, 0.0, 1.0e-10]
    dx = [0.1e-9, 2.0e-9 / 3.0, 0.7e-9]
    time, step = 1.2345678901234567e-12, 42
    path = tmp_path / "plt00000042"
    rc, err, hi = _write(writer, path, n, lo, dx, time, step, fields)
    assert rc == 0, err

    pf = plotfile.read(str(path))
    assert pf["names"] == list(fields)
    assert pf["n"] == n and pf["step"] == step
    assert pf["time"] == time                       # written with 17 digits: exact
    assert pf["prob_lo"] == lo and pf["prob_hi"] == hi and pf["dx"] == dx
    for name, v in fields.items():
        got = pf["fields"][name]
        assert got.shape == (n[2], n[1], n[0])
        assert np.array_equal(got.reshape(-1).view(np.uint64), v.view(np.uint64)), name
    k, j, i = 4, 2, 3                               # spot check of the x-fastest order
    assert pf["fields"]["Phi"][k, j, i] == (i + n[0] * (j + n[1] * k)) * 1.0e-3 - 0.01


def test_vismf_header_box_and_min_max(writer, tmp_path):
    n = [4, 2, 6]
    npts = n[0] * n[1] * n[2]
    a = np.linspace(-3.5, 9.25, npts)
    b = np.full(npts, 2.0)
    b[11] = -7.0
    path = tmp_path / "plt00000000"
    rc, err, _ = _write(writer, path, n, [0, 0, 0], [1, 1, 1], 0.0, 0, {"a": a, "b": b})
    assert rc == 0, err
    lines = (path / "Level_0" / "Cell_H").read_text().split("\n")
    assert lines[:4] == ["1", "0", "2", "0"]        # version, how, ncomp, ngrow
    assert lines[4] == "(1 0" and lines[5] == "((0,0,0) (3,1,5) (0,0,0))" and lines[6] == ")"
    assert lines[7] == "1" and lines[8] == "FabOnDisk: Cell_D_00000 0"
    mins = [float(v) for v in lines[11].rstrip(",").split(",")]
    maxs = [float(v) for v in lines[14].rstrip(",").split(",")]
    assert lines[10] == "1,2" and lines[13] == "1,2"
    np.testing.assert_allclose(mins, [a.min(), b.min()], rtol=1e-14)
    np.testing.assert_allclose(maxs, [a.max(), b.max()], rtol=1e-14)
    header = (path / "Header").read_text().split("\n")
    assert header[-2] == "Level_0/Cell"


def test_plotfile_name_is_eight_digits(writer):
    out = ctypes.create_string_buffer(32)
    for step, want in [(0, "plt00000000"), (7, "plt00000007"), (12345678, "plt12345678")]:
        writer.pf_name(step, out, 32)
        assert out.value.decode() == want


def test_unwritable_directory_is_an_error_with_a_message(writer, tmp_path):
    blocker = tmp_path / "file"
    blocker.write_text("not a directory")
    rc, err, _ = _write(writer, blocker / "plt00000001", [2, 2, 2], [0, 0, 0], [1, 1, 1], 0.0, 1,
                        {"a": np.zeros(8)})
    assert rc != 0 and "cannot create" in err
