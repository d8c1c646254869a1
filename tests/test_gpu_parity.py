"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Each test runs one reference function, or several coupled steps, on the GPU
and on the oracle from identical seeded inputs.  Tolerances: FP64 fields
within 1e-10 relative (max-norm, per field) per step -- the stencil and
pointwise kernels agree to ~1e-15, the Poisson solves to the multigrid
tolerance, here 1e-13 on both sides; masks bit-exact; the mixed-precision
path within 1e-6 of the FP64 oracle.
"""
import numpy as np
import pytest

from ferrox_b200 import decks, plotfile
from helpers import pair, relerr, small_grains

pytestmark = pytest.mark.gpu


def rand_P(shape, seed, scale=0.01, vector=False):
    g = np.random.default_rng(seed)
    Pz = g.uniform(-scale, scale, shape)
    if not vector:
        return (None, None, Pz)
    return (g.uniform(-scale, scale, shape), g.uniform(-scale, scale, shape), Pz)


def test_masks_and_setup_bit_exact():
    f, o = pair(decks.mfism(16, 16, 48))
    for name in ["mask", "epsilon", "Gamma", "Pz", "tphase"]:
        assert np.array_equal(f.field(name), o.field(name)), name


@pytest.mark.parametrize("vector", [False, True])
def test_poisson_rhs(vector):
    text = decks.mfim(16, 16, 12, extra={"is_polarization_scalar": 0 if vector else 1})
    f, o = pair(text, P=rand_P((12, 16, 16), 1, vector=vector))
    f.compute_poisson_rhs()
    o.compute_poisson_rhs()
    assert relerr(f.field("PoissonRHS"), o.field("PoissonRHS")) < 1e-12


def test_poisson_rhs_rotated_grains():
    text, g = small_grains(16, 16, 24)
    f, o = pair(text, grains=g, P=rand_P((24, 16, 16), 2))
    f.compute_poisson_rhs()
    o.compute_poisson_rhs()
    assert relerr(f.field("PoissonRHS"), o.field("PoissonRHS")) < 1e-12


@pytest.mark.parametrize("fd", [0, 1])
def test_compute_rho(fd):
    f, o = pair(decks.mfism(8, 8, 24, extra={"use_Fermi_Dirac": fd}))
    phi = np.random.default_rng(4).uniform(-0.4, 1.2, f.shape)
    f.set_field("Phi", phi)
    o.set_field("Phi", phi)
    f.compute_rho()
    o.compute_rho()
    for name in ["charge", "electrons", "holes"]:
        assert relerr(f.field(name), o.field(name)) < 1e-12, name


@pytest.mark.parametrize("mode", ["extrap", "face", "zero"])
def test_compute_E(mode):
    text, g = small_grains(16, 16, 24)
    text += f"fx.phi_ghost_mode = {mode}\nPhi_Bc_hi = 0.7\nPhi_Bc_lo = -0.2\n"
    f, o = pair(text, grains=g)
    o.set_phi_bc()
    f.set_phi_bc()
    phi = np.random.default_rng(5).uniform(-0.5, 0.5, f.shape)
    f.set_field("Phi", phi)
    o.set_field("Phi", phi)
    f.compute_E()
    o.compute_E()
    for name in ["Ex", "Ey", "Ez"]:
        assert relerr(f.field(name), o.field(name)) < 1e-12, name


TDGL_CASES = [
    ("scalar-303-331", dict(P_BC_flag_lo=[3, 3, 0], P_BC_flag_hi=[3, 3, 1]), False, False),
    ("scalar-flag0", dict(P_BC_flag_lo=[3, 3, 0], P_BC_flag_hi=[3, 3, 0]), False, False),
    ("scalar-flag1", dict(P_BC_flag_lo=[3, 3, 1], P_BC_flag_hi=[3, 3, 1]), False, False),
    ("scalar-flag2", dict(P_BC_flag_lo=[3, 3, 2], P_BC_flag_hi=[3, 3, 2]), False, False),
    ("scalar-flag3", dict(P_BC_flag_lo=[3, 3, 3], P_BC_flag_hi=[3, 3, 3]), False, False),
    ("scalar-flag4", dict(P_BC_flag_lo=[3, 3, 4], P_BC_flag_hi=[3, 3, 4]), False, False),
    ("vector", dict(is_polarization_scalar=0, alpha_12=1.0e8, alpha_112=2.0e9, alpha_123=3.0e9,
                    g12=2.0e-11, g44_p=1.0e-11), True, False),
    ("no-landau", dict(include_Landau=0), False, False),
    ("no-elec", dict(include_Elec=0), False, False),
    ("rotated", dict(), False, True),
    ("rotated-vector", dict(is_polarization_scalar=0, g12=2.0e-11), True, True),
]


@pytest.mark.parametrize("name,extra,vector,rot", TDGL_CASES, ids=[c[0] for c in TDGL_CASES])
def test_tdgl_euler(name, extra, vector, rot):
    extra = dict(extra)
    extra["Phi_Bc_hi"] = 0.5
    if rot:
        text, g = decks.polycrystal(16, 16, 24, ngrains=6, seed=3, nsteps=10, extra=extra)
    else:
        text, g = decks.mfim(16, 16, 24, extra=extra), None
    P = rand_P((24, 16, 16), 7, scale=0.2, vector=vector)
    f, o = pair(text, grains=g, P=P)
    f.set_phi_bc(); o.set_phi_bc()
    phi = np.random.default_rng(8).uniform(-0.5, 0.5, f.shape)
    f.set_field("Phi", phi)
    o.set_field("Phi", phi)
    P0 = [o.field(c) for c in ["Px", "Py", "Pz"]]
    o.compute_E()
    o.tdgl_euler()
    f.tdgl_euler()
    for q, c in enumerate(["Px", "Py", "Pz"]):
        dg, do = f.field(c) - P0[q], o.field(c) - P0[q]
        assert relerr(dg, do) < 1e-10, (c, relerr(dg, do))
        assert relerr(f.field(c), o.field(c)) < 1e-13, c


def test_tdgl_euler_mixed_precision():
    text = decks.mfim(16, 16, 24, extra={"Phi_Bc_hi": 0.5})
    f, o = pair(text, P=rand_P((24, 16, 16), 9, scale=0.2), precision="mixed")
    f.set_phi_bc(); o.set_phi_bc()
    phi = np.random.default_rng(10).uniform(-0.5, 0.5, f.shape)
    f.set_field("Phi", phi)
    o.set_field("Phi", phi)
    P0 = o.field("Pz")
    o.compute_E(); o.tdgl_euler(); f.tdgl_euler()
    assert relerr(f.field("Pz") - P0, o.field("Pz") - P0) < 1e-5
    assert relerr(f.field("Pz"), o.field("Pz")) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_phi_rho_dielectric(precision):
    f, o = pair(decks.mfim(32, 32, 24, Phi_Bc_hi=0.8), P=rand_P((24, 32, 32), 11), precision=precision, rtol=1e-13)
    f.set_phi_bc(); o.set_phi_bc()
    f.compute_phi_rho()
    o.compute_phi_rho()
    st = f.stats()
    assert st["mg_resid_last"] <= st["mg_target_last"]
    assert relerr(f.field("Phi"), o.field("Phi")) < 1e-10
    assert relerr(f.field("PoissonRHS"), o.field("PoissonRHS")) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_phi_rho_semiconductor_newton(precision):
    text = decks.mfism(16, 16, 48, extra={"Phi_Bc_hi": 0.6})
    f, o = pair(text, P=rand_P((48, 16, 16), 12), precision=precision, rtol=1e-13)
    f.set_phi_bc(); o.set_phi_bc()
    f.compute_phi_rho()
    o.compute_phi_rho()
    assert f.stats()["newton_iters_last"] == o.scalar("newton_iters")
    for name in ["Phi", "charge", "electrons", "holes"]:
        assert relerr(f.field(name), o.field(name)) < 1e-10, name
    assert relerr(f.field("alpha_cc"), o.field("alpha_cc")) < 1e-7


def test_coupled_steps_mfim():
    f, o = pair(decks.mfim(16, 16, 24, Phi_Bc_hi=0.3), rtol=1e-13)
    for step in range(1, 21):
        f.step(1)
        o.step(step)
    for name in ["Pz", "Phi", "Ez"]:
        o.compute_E() if name == "Ez" else None
        assert relerr(f.field(name), o.field(name)) < 1e-10, name
    # steady_err = max|phi - phi_old| / max|phi| is already normalised by the
    # field scale: held in absolute terms, twice the fields' relative bound
    assert abs(f.stats()["steady_err_last"] - o.scalar("steady_err")) <= 2e-10


def test_coupled_steps_mfism_fixed_sweep():
    text = decks.mfism(16, 16, 48, steps_per_voltage=2, v_step=0.1, v_max=0.3)
    f, o = pair(text, rtol=1e-13)
    done = f.step(10)
    last = o.run(10)
    assert done == last
    assert f.stats()["Phi_Bc_hi"] == pytest.approx(o.scalar("Phi_Bc_hi"))
    assert f.stats()["num_Vapp"] == o.scalar("num_Vapp")
    for name in ["Pz", "Phi", "charge"]:
        assert relerr(f.field(name), o.field(name)) < 1e-10, name


def test_coupled_steps_polycrystal():
    text, g = decks.polycrystal(16, 16, 32, ngrains=8, seed=5, nsteps=10, extra={"Phi_Bc_hi": 1.0})
    f, o = pair(text, grains=g, rtol=1e-13)
    for step in range(1, 11):
        f.step(1)
        o.step(step)
    for name in ["Pz", "Phi"]:
        assert relerr(f.field(name), o.field(name)) < 1e-10, name


@pytest.mark.parametrize("sc", [False, True])
def test_order2_predictor_corrector(sc):
    # TimeIntegratorOrder = 2, main.cpp:308-348
    text = (decks.mfism(16, 16, 48, extra={"Phi_Bc_hi": 0.5, "TimeIntegratorOrder": 2}) if sc
            else decks.mfim(16, 16, 24, Phi_Bc_hi=0.4, extra={"TimeIntegratorOrder": 2}))
    f, o = pair(text, rtol=1e-13)
    for step in range(1, 9):
        f.step(1)
        o.step(step)
    for name in ["Pz", "Phi"]:
        assert relerr(f.field(name), o.field(name)) < 1e-10, name


def test_named_mfim_size_one_step():
    # the 64x64x36 MFIM workload: one coupled step against the oracle
    f, o = pair(decks.mfim(64, 64, 36), rtol=1e-12)
    f.step(1)
    o.step(1)
    for name in ["Pz", "Phi"]:
        assert relerr(f.field(name), o.field(name)) < 1e-10, name


def test_mixed_precision_coupled_steps():
    text = decks.mfim(32, 32, 24, Phi_Bc_hi=0.5)
    f, o = pair(text, precision="mixed", rtol=1e-12)
    for step in range(1, 21):
        f.step(1)
        o.step(step)
    for name in ["Pz", "Phi"]:
        assert relerr(f.field(name), o.field(name)) < 1e-6, name


def test_plotfile_roundtrip(tmp_path):
    text = decks.mfim(16, 16, 12, Phi_Bc_hi=0.2)
    f, _ = pair(text)
    f.step(2)
    path = f.write_plotfile(2, str(tmp_path))
    pf = plotfile.read(path)
    assert pf["names"][:5] == ["Px", "Py", "Pz", "Phi", "PoissonRHS"]
    assert pf["n"] == [16, 16, 12] and pf["step"] == 2
    for name in ["Pz", "Phi", "Ez", "mask", "epsilon"]:
        assert np.array_equal(pf["fields"][name], f.field(name)), name


def test_kernel_launches_counted():
    f, _ = pair(decks.mfim(16, 16, 12))
    a = f.stats()["kernel_launches"]
    f.step(1)
    assert f.stats()["kernel_launches"] > a


@pytest.mark.parametrize("deck", ["mfim", "mfism"])
def test_thousand_steps_drift(deck):
    # FP64 fields within 1e-8 of the oracle after 1000 coupled steps
    text = (decks.mfism(16, 16, 48, extra={"Phi_Bc_hi": 0.4}) if deck == "mfism"
            else decks.mfim(16, 16, 12, Phi_Bc_hi=0.6))
    f, o = pair(text, rtol=1e-13)
    done = f.step(1000)
    last = o.run(1000)
    assert done == last      # the same break step, if the steady-state test ends the loop
    for name in ["Pz", "Phi"] + (["charge"] if deck == "mfism" else []):
        assert relerr(f.field(name), o.field(name)) < 1e-8, (name, relerr(f.field(name), o.field(name)))


def test_steady_state_triggered_voltage_sweep():
    """The reference's own sweep schedule: CheckSteadyState sets inc_step =
    step once max|phi - phi_old| / max|phi| < phi_tolerance
    (ElectrostaticSolver.cpp:548-552); the loop then advances Phi_Bc_hi by
    sign * Phi_Bc_inc, reverses at Phi_Bc_hi_max, counts num_Vapp, re-solves
    ComputePhi_Rho and breaks at num_Vapp_max (main.cpp:572-611).  The sweep
    state is compared with the oracle after every step, and the run must see
    several increments and a reversal."""
    text = decks.mfism(16, 16, 48, v_step=0.1, v_max=0.3,
                       extra={"fx.sweep_mode": "steady", "phi_tolerance": 5.0e-2, "num_Vapp_max": 6})
    f, o = pair(text, rtol=1e-13)
    seen_sign = set()
    done_f = done_o = 0
    for step in range(1, 41):
        done_f = f.step(1)
        brk = o.step(step)
        st = f.stats()
        for k in ["Phi_Bc_hi", "num_Vapp", "sign", "inc_step", "steady_state_step"]:
            assert st[k] == o.scalar(k), (step, k, st[k], o.scalar(k))
        # steady_err is already normalised by max|phi|: hold it in absolute terms
        # (a difference of two nearly equal fields loses relative accuracy)
        assert abs(st["steady_err_last"] - o.scalar("steady_err")) <= 2e-10, step
        seen_sign.add(st["sign"])
        if brk == 1:
            assert st["finished"] == 1
            done_o = step
            break
        assert done_f == 1
    assert f.stats()["num_Vapp"] >= 3 and seen_sign == {1, -1}
    assert done_o > 0
    for name in ["Pz", "Phi", "charge"]:
        assert relerr(f.field(name), o.field(name)) < 1e-10, name
