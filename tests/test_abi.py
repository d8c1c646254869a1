"""The C ABI without a GPU: the library loads, exports every declared entry
point, parses inputs like the reference (checked against the oracle's reader),
sets up masks / permittivity / initial P bit-exactly, and refuses to compute
without a device instead of falling back to the CPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from ferrox_b200 import api, decks
from oracle import inputs as I
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DECK = """
domain.prob_lo = -8.e-9 -8.e-9 0.e-9
domain.prob_hi =  8.e-9  8.e-9 9.e-9
domain.n_cell = 16 16 18
domain.is_periodic = 1 1 0
boundary.hi = per per dir(Zmax)
boundary.lo = per per dir(Zmin)
prob_type = 2
TimeIntegratorOrder = 1
dt = 2.0e-13
P_BC_flag_lo = 3 3 0
P_BC_flag_hi = 3 3 1
lambda = 3.0e-9
my_constants.tlo = 5.0e-9
my_constants.w = 2*tlo
Coordinate_Transformation = 1
tphase_geom.tphase_geom_function(x,y,z) = "1.*(x >= -3.e-9)*(x <= 3.e-9)*(z >= tlo)
                                         + 0.*(y > 0)"
angle_alpha.alpha_function(x,y,z) = "if(x > 0, 30.0, -15.0)"
angle_beta.beta_function(x,y,z) = "10.0 + 20.0*(y > 1e-9)"
angle_theta.theta_function(x,y,z) = "5.0 * (z > w/3)"
SC_lo = -1.0 -1.0 -1.0
SC_hi = -1.0 -1.0 -1.0
DE_lo = -8.e-9 -8.e-9 0.0e-9
DE_hi =  8.e-9  8.e-9 4.0e-9
FE_lo = -8.e-9 -8.e-9 4.0e-9
FE_hi =  8.e-9  8.e-9 9.0e-9
epsilon_0 = 8.85e-12
epsilonX_fe = 24.0
epsilonX_fe_tphase = 40.0
epsilonZ_fe = 24.0
epsilon_de = 10.0
epsilon_si = 11.7
alpha = -2.5e9
beta = 6.0e10
gamma = 1.5e11
BigGamma = 100
g11 = 1.0e-9
g44 = 1.0e-9
g44_p = 0.0
g12 = 0.0
alpha_12 = 0.0
alpha_112 = 0.0
alpha_123 = 0.0
"""


def test_library_exports_every_declared_symbol():
    L = api.lib()
    with open(os.path.join(ROOT, "include", "ferrox_b200.h")) as f:
        hdr = f.read()
    declared = set(re.findall(r"\b(fx_\w+)\s*\(", hdr))
    assert declared == set(api.EXPORTS), declared ^ set(api.EXPORTS)
    for name in declared:
        assert hasattr(L, name), name
    assert b"sm_100a" in L.fx_version()


def _golden(name):
    with open(os.path.join(ROOT, "tests", "golden", "decks", name)) as f:
        return f.read()


@pytest.mark.parametrize("text", [decks.mfim(16, 16, 12), decks.mfism(16, 16, 48), REF_DECK,
                                  _golden("Examples_inputs_mfis_eb.inputs")],
                         ids=["mfim", "mfism", "ref_deck", "mfis_eb"])
def test_setup_matches_oracle(text):
    f = api.FerroX(text)
    table = I.parse_table(text)
    p = I.ferrox_params(table)
    tph, a, b, t = I.function_fields(table, p)
    o = O.Oracle(p, tph, (a, b, t))
    for name in ["mask", "epsilon", "Gamma", "tphase", "alpha", "beta", "theta", "Px", "Py", "Pz"]:
        assert np.array_equal(f.field(name), o.field(name)), name
    for key in ["dt", "lambda", "alpha", "beta", "gamma", "g11", "g44", "BigGamma", "epsilon_de", "delta",
                "phi_tolerance", "inc_step", "num_Vapp_max", "use_Fermi_Dirac", "prob_type"]:
        assert f.param(key) == pytest.approx(p[key], rel=0, abs=0), key
    for d in range(3):
        assert f.param(f"DE_lo[{d}]") == p["DE_lo"][d]
        assert f.param(f"P_BC_flag_hi[{d}]") == p["P_BC_flag_hi"][d]
    assert f.param("V_hi") == o.scalar("V_hi") and f.param("V_lo") == o.scalar("V_lo")


def test_reader_last_definition_comments_and_file(tmp_path):
    """ParmParse behaviour of the library's own reader: the last definition of a key wins,
    '#' starts a comment (whole line or after a value), `key=value` needs no spaces, and
    fx_create reads the same deck from a file path."""
    text = (decks.mfim(8, 8, 12) + "\ndt = 1.0e-13\n# dt = 9.0\nlambda=2.5e-9   # trailing comment\n"
            "dt = 3.0e-13\n")
    f = api.FerroX(text)
    assert f.param("dt") == 3.0e-13 and f.param("lambda") == 2.5e-9
    f.close()
    deck = tmp_path / "inputs"
    deck.write_text(text)
    g = api.FerroX(str(deck), is_text=False)
    assert g.param("dt") == 3.0e-13 and g.param("lambda") == 2.5e-9
    g.close()
    with pytest.raises(api.FxError) as e:
        api.FerroX(str(tmp_path / "missing"), is_text=False)
    assert "cannot open" in str(e.value)


@pytest.mark.parametrize("key,bad,good", [
    ("fx.phi_extrapolate", 7, 6), ("fx.phi_extrapolate", -1, 0), ("fx.phi_ghost_mode", 3, 1),
    ("fx.mg_max_iter", 0, 1), ("fx.newton_max_iter", 0, 1), ("fx.mg_nu1", -1, 0), ("fx.mg_nu2", -1, 0),
    ("fx.mg_rtol", 0.0, 1e-12), ("fx.mg_seg", 8, 16), ("fx.mg_seg_min", -1, 1000),
    ("fx.mg_nu1_coarse", 0, 1), ("fx.mg_nu2_coarse", -2, 0),
])
def test_solver_settings_out_of_range_are_rejected(key, bad, good):
    """fx_set_param refuses what the inputs reader refuses, and a refused call changes nothing."""
    f = api.FerroX(decks.mfim(8, 8, 12))
    before = f.param(key)
    with pytest.raises(api.FxError) as e:
        f.set_param(key, bad)
    assert e.value.code == -1 and key in str(e.value)
    assert f.param(key) == before
    f.set_param(key, good)
    assert f.param(key) == good
    f.close()
    if key in ("fx.phi_extrapolate", "fx.mg_max_iter", "fx.newton_max_iter", "fx.mg_rtol"):
        with pytest.raises(api.FxError) as e:
            api.FerroX(decks.mfim(8, 8, 12) + f"\n{key} = {bad}\n")
        assert e.value.code == -2 and key in str(e.value)


def test_multigrid_defaults_read_back():
    f = api.FerroX(decks.mfim(8, 8, 12))
    assert (f.param("fx.mg_nu1"), f.param("fx.mg_nu2"), f.param("fx.mg_mixed_cycles")) == (2, 1, 2)
    assert f.param("fx.alpha_tiles") == 1 and f.param("fx.phi_extrapolate") == 4
    assert (f.param("fx.mg_nu1_coarse"), f.param("fx.mg_nu2_coarse"), f.param("fx.mg_seg")) == (1, -1, 16)
    assert (f.param("fx.mg_split"), f.param("fx.mg_half")) == (1, 1)
    f.close()


def test_grains_setup_matches_oracle():
    text, g = decks.polycrystal(16, 16, 24, ngrains=6, seed=3)
    f = api.FerroX(text)
    f.set_grains(g["id"], g["angles"], g["tphase"])
    tph, ang = decks.grain_fields(g)
    o = O.Oracle(I.ferrox_params(I.parse_table(text)), tph, tuple(ang))
    for name in ["mask", "epsilon", "tphase", "alpha", "beta", "theta", "Pz"]:
        assert np.array_equal(f.field(name), o.field(name)), name
    assert f.param("num_variants") >= 2


@pytest.mark.parametrize("bad,code", [
    ("FE_lo = -1 -1 -1\n", -3),
    ("P_BC_flag_lo = 3 3 7\n", -2),
    ("prob_type = 9\n", -2),
    ("domain.is_periodic = 0 1 0\n", -3),
    ("fx.phi_ghost_mode = sideways\n", -2),
    ("tphase_geom.tphase_geom_function(x,y,z) = \"x +* 2\"\nCoordinate_Transformation = 1\n", -2),
])
def test_bad_inputs_are_rejected_with_a_message(bad, code):
    text = decks.mfim(8, 8, 12) + bad
    if code is None:
        api.FerroX(text).close()
        return
    with pytest.raises(api.FxError) as e:
        api.FerroX(text)
    assert e.value.code == code
    assert len(str(e.value)) > 20


def test_missing_required_key():
    text = "\n".join(l for l in decks.mfim(8, 8, 12).splitlines() if not l.startswith("BigGamma"))
    with pytest.raises(api.FxError) as e:
        api.FerroX(text)
    assert "BigGamma" in str(e.value)


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    f = api.FerroX(decks.mfim(8, 8, 12))
    for call in [f.compute_phi_rho, f.tdgl_euler, lambda: f.step(1), f.compute_E, f.compute_rho]:
        with pytest.raises(api.FxError) as e:
            call()
        assert e.value.code == -4
    with pytest.raises(api.FxError):
        f.field("Phi")


def test_odd_periodic_count_is_rejected():
    with pytest.raises(api.FxError) as e:
        api.FerroX(decks.mfim(9, 8, 12))
    assert e.value.code == -3


def test_gradient_entry_points_check_arguments_before_any_device_work():
    f = api.FerroX(decks.mfim(8, 8, 12))
    with pytest.raises(api.FxError) as e:
        f.backward()
    assert e.value.code == -1 and "fx_forward_record" in str(e.value)
    with pytest.raises(api.FxError) as e:
        f.grad_P0()
    assert e.value.code == -1
    with pytest.raises(api.FxError) as e:
        f.forward_record(np.zeros(0), 1.0)
    assert e.value.code == -1
    with pytest.raises(api.FxError) as e:
        f.forward_record(np.array([0.0, np.nan]), 1.0)
    assert e.value.code == -1
    with pytest.raises(api.FxError) as e:
        f.forward_record(np.zeros(4), 1.0, checkpoint_every=0)
    assert e.value.code == -1
    g = api.FerroX(decks.mfim(8, 8, 12, extra={"TimeIntegratorOrder": 2}))
    with pytest.raises(api.FxError) as e:
        g.forward_record(np.zeros(4), 1.0)
    assert e.value.code == -3
    h = api.FerroX(decks.mfim(4, 4, 12))
    with pytest.raises(api.FxError) as e:
        h.forward_record(np.zeros(4), 1.0)
    assert e.value.code == -3
