"""GPU-vs-oracle parity at the benchmark sizes and on the reference's own
regression decks, in FP64 and in mixed precision.

* the 128x128x144 MFISM workload (5 nm HZO / 1 nm SiO2 / 30 nm p-Si,
  Boltzmann carriers, Newton-coupled Poisson, fixed-cadence voltage ramp):
  10 coupled steps;
* the 64-grain 256x256x128 polycrystalline film (5 nm HZO in seeded Voronoi
  grains with random polar axes and t-phase grains, on 4 nm Al2O3): 5 coupled
  steps;
* FerroX's regression decks Exec/regression_inputs/3D_MFIM/inputs_mfim_Noeb
  (64x64x18 MFIM, its own nsteps = 3) and Exec/regression_inputs/MIS/input_mis
  (256x256x128 metal / SiO2 / p-Si with Fermi-Dirac carriers and the
  steady-state-triggered voltage sweep, nsteps = 3), from the fixtures in
  tests/golden/decks.

FP64 fields are held to 1e-10 relative per field (max-norm), the mixed path's
fields to 1e-6 of the FP64 oracle.  Both sides solve the Poisson equation to
a relative residual of 1e-13 so that the solver tolerance does not enter the
comparison (the reference's own 1e-10 would allow differences of that size).
"""
import os

import numpy as np
import pytest

from ferrox_b200 import decks
from helpers import pair, relerr

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
RTOL = 1e-13
FP64_TOL = 1e-10
MIXED_TOL = 1e-6


def _fields(x, names):
    x.compute_E()
    return {n: x.field(n) for n in names}


def _run_pair(text, grains, precision, steps, names):
    f, o = pair(text, grains=grains, precision=precision, rtol=RTOL)
    done = f.step(steps)
    last = o.run(steps)
    got = _fields(f, names)
    st = f.stats()
    f.close()
    return got, _fields(o, names), (done, last), st, o


MFISM_NAMES = ["Pz", "Phi", "Ex", "Ey", "Ez", "charge", "electrons", "holes"]
POLY_NAMES = ["Pz", "Phi", "Ex", "Ey", "Ez"]


@pytest.fixture(scope="module")
def mfism_oracle():
    """The oracle's fields after 10 steps of the 128x128x144 MFISM deck."""
    from helpers import pair as _pair
    text = decks.mfism(128, 128, 144)
    _, o = _pair(text, rtol=RTOL)
    last = o.run(10)
    return text, _fields(o, MFISM_NAMES), last


@pytest.fixture(scope="module")
def poly_oracle():
    """The oracle's fields after 5 steps of the 64-grain 256x256x128 film."""
    import oracle.oracle as O
    from oracle import inputs as I
    text, g = decks.polycrystal(256, 256, 128, ngrains=64, seed=1)
    tph, ang = decks.grain_fields(g)
    o = O.Oracle(I.ferrox_params(I.parse_table(text)), tph, tuple(ang))
    o.set_scalar("mg_rtol", RTOL)
    last = o.run(5)
    return text, g, _fields(o, POLY_NAMES), last


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_mfism_128x128x144_ten_steps(mfism_oracle, precision, tol):
    from ferrox_b200 import api
    text, ref, last = mfism_oracle
    f = api.FerroX(text, precision=precision)
    f.set_param("fx.mg_rtol", RTOL)
    assert f.step(10) == last
    f.compute_E()
    for n in MFISM_NAMES:
        assert relerr(f.field(n), ref[n]) < tol, (n, relerr(f.field(n), ref[n]))
    f.close()


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_polycrystal_256x256x128_five_steps(poly_oracle, precision, tol):
    from ferrox_b200 import api
    text, g, ref, last = poly_oracle
    f = api.FerroX(text, precision=precision)
    f.set_grains(g["id"], g["angles"], g["tphase"])
    f.set_param("fx.mg_rtol", RTOL)
    assert f.step(5) == last
    f.compute_E()
    for n in POLY_NAMES:
        assert relerr(f.field(n), ref[n]) < tol, (n, relerr(f.field(n), ref[n]))
    f.close()


def _golden(name):
    with open(os.path.join(HERE, "golden", "decks", name)) as fh:
        return fh.read()


def test_regression_deck_3d_mfim():
    """Exec/regression_inputs/3D_MFIM/inputs_mfim_Noeb for its nsteps = 3."""
    text = _golden("3D_MFIM_inputs_mfim_Noeb.inputs")
    got, ref, (done, last), st, o = _run_pair(text, None, None, 3, POLY_NAMES)
    assert done == last
    for n in POLY_NAMES:
        assert relerr(got[n], ref[n]) < FP64_TOL, (n, relerr(got[n], ref[n]))
    assert st["steady_err_last"] == pytest.approx(o.scalar("steady_err"), rel=0, abs=2 * FP64_TOL)


def test_regression_deck_mis():
    """Exec/regression_inputs/MIS/input_mis for its nsteps = 3: Fermi-Dirac
    carriers, no ferroelectric, steady-state-triggered voltage sweep."""
    text = _golden("MIS_input_mis.inputs")
    names = ["Phi", "Ez", "charge", "electrons", "holes"]
    got, ref, (done, last), st, o = _run_pair(text, None, None, 3, names)
    assert done == last
    for n in names:
        assert relerr(got[n], ref[n]) < FP64_TOL, (n, relerr(got[n], ref[n]))
    for k in ["Phi_Bc_hi", "num_Vapp", "inc_step", "sign", "steady_state_step"]:
        assert st[k] == o.scalar(k), k
