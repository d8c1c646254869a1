"""The inputs keys fx.grain_file and fx.initial_P_file: a polycrystal and an
initial polarization given as files, so that the executable (which only takes
an inputs deck) can run them.

The formats are raw and little-endian (ferrox_b200.decks.write_grain_file /
write_P_file; include/ferrox_b200.h).  The library reads them in C++, the
oracle through the Python reader; both must give the setup that the API calls
fx_set_grains / fx_set_initial_P give, bit for bit.  The GPU test runs the
executable on a file-defined deck and compares its plotfile with an API run.
"""
import os
import subprocess

import numpy as np
import pytest

from ferrox_b200 import api, decks, plotfile
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SETUP_FIELDS = ["mask", "epsilon", "tphase", "alpha", "beta", "theta", "Px", "Py", "Pz"]


def _file_deck(tmp_path, nx=16, ny=16, nz=32, ngrains=8, vector=False, nsteps=4, plot_int=4):
    text, g = decks.polycrystal(nx, ny, nz, ngrains=ngrains, seed=5, nsteps=nsteps,
                                extra={"Phi_Bc_hi": 0.5, "plot_int": plot_int,
                                       "is_polarization_scalar": 0 if vector else 1})
    rng = np.random.Generator(np.random.PCG64(11))
    shape = (nz, ny, nx)
    P = [rng.uniform(-0.1, 0.1, shape) if vector else None, rng.uniform(-0.1, 0.1, shape) if vector else None,
         rng.uniform(-0.2, 0.2, shape)]
    gpath, ppath = str(tmp_path / "grains.bin"), str(tmp_path / "P0.bin")
    decks.write_grain_file(gpath, g)
    decks.write_P_file(ppath, P[2], P[0], P[1])
    ftext = text + f'fx.grain_file = "{gpath}"\nfx.initial_P_file = "{ppath}"\n'
    return text, ftext, g, P


def _api_run(text, g, P):
    f = api.FerroX(text)
    f.set_grains(g["id"], g["angles"], g["tphase"])
    f.set_initial_P(*P)
    return f


@pytest.mark.parametrize("vector", [False, True])
def test_files_give_the_api_setup_bit_for_bit(tmp_path, vector):
    text, ftext, g, P = _file_deck(tmp_path, vector=vector)
    a = api.FerroX(ftext)
    b = _api_run(text, g, P)
    o = O.Oracle.from_text(ftext)
    for n in SETUP_FIELDS:
        assert np.array_equal(a.field(n), b.field(n)), n
        assert np.array_equal(a.field(n), o.field(n)), n
    assert a.param("num_variants") == b.param("num_variants") > 0


def test_grain_file_round_trip(tmp_path):
    _, g = decks.polycrystal(8, 8, 24, ngrains=5, seed=2)
    p = str(tmp_path / "g.bin")
    decks.write_grain_file(p, g)
    h = decks.read_grain_file(p)
    assert np.array_equal(h["id"], g["id"]) and np.array_equal(h["angles"], g["angles"])
    assert np.array_equal(h["tphase"], np.asarray(g["tphase"], dtype=np.uint8))
    with open(p, "rb") as f:
        b = f.read()
    assert b[:8] == b"FXGRAIN1" and len(b) == 24 + 32 * 5 + 8 * 8 * 24


def test_bad_files_are_refused(tmp_path):
    text, ftext, g, P = _file_deck(tmp_path)
    # missing file: I/O error
    with pytest.raises(api.FxError) as e:
        api.FerroX(text + 'fx.initial_P_file = "/nonexistent/P0.bin"\n')
    assert e.value.code == -8 and "fx.initial_P_file" in str(e.value)
    # wrong size
    short = tmp_path / "short.bin"
    short.write_bytes(np.zeros(7).tobytes())
    with pytest.raises(api.FxError) as e:
        api.FerroX(text + f'fx.initial_P_file = "{short}"\n')
    assert e.value.code == -2 and "expected" in str(e.value)
    # a grain file of another grid
    _, g2 = decks.polycrystal(8, 8, 32, ngrains=3, seed=1)
    other = str(tmp_path / "other.bin")
    decks.write_grain_file(other, g2)
    with pytest.raises(api.FxError) as e:
        api.FerroX(text + f'fx.grain_file = "{other}"\n')
    assert e.value.code == -2 and "differs" in str(e.value)
    # grains need the coordinate transformation
    with pytest.raises(api.FxError) as e:
        api.FerroX(text + f'Coordinate_Transformation = 0\nfx.grain_file = "{tmp_path / "grains.bin"}"\n')
    assert e.value.code == -2 and "Coordinate_Transformation" in str(e.value)
    # not a grain file
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"NOTGRAIN" + bytes(100))
    with pytest.raises(api.FxError) as e:
        api.FerroX(text + f'fx.grain_file = "{junk}"\n')
    assert e.value.code == -2


@pytest.mark.gpu
def test_executable_runs_a_file_defined_polycrystal(tmp_path):
    """The executable on a deck whose grains and initial P come from files
    writes the plotfile an API run with fx_set_grains / fx_set_initial_P
    writes, bit for bit."""
    from ferrox_b200 import build
    build.build()
    text, ftext, g, P = _file_deck(tmp_path, nsteps=4, plot_int=4)
    deck = tmp_path / "inputs"
    deck.write_text(ftext)
    run_dir = tmp_path / "exe"
    run_dir.mkdir()
    r = subprocess.run([os.path.join(ROOT, "ferrox_b200", "ferrox_b200"), str(deck)], cwd=run_dir,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    exe = plotfile.read(str(run_dir / "plt00000004"))
    f = _api_run(text, g, P)
    f.step(4)
    path = f.write_plotfile(4, str(tmp_path / "api"))
    ref = plotfile.read(path)
    assert exe["names"] == ref["names"]
    for n in ref["names"]:
        assert np.array_equal(exe["fields"][n], ref["fields"][n]), n
    f.close()
