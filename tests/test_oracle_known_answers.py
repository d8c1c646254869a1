"""Known-answer tests that pin the CPU oracle.

The reference ships no tests, golden vectors or benchmark plotfiles and it
cannot be compiled here (AMReX is absent), so the oracle is pinned against
closed forms of the reference's own formulas:

* Landau term        TotalEnergyDensity.cpp:88-114
* stencils           DerivativeAlgorithm.H:256-467 on polynomial profiles
* lambda BC forms    DerivativeAlgorithm.H:194-197, :408-411
* Poisson operator   ElectrostaticSolver.cpp:603-605 (uniform eps -> linear phi;
                     two-layer stack vs an independent tridiagonal solve)
* carriers           ChargeDensity.cpp:71-93 (mass-action law, FD -> MB limit)
* E from phi         ElectrostaticSolver.cpp:160-200, DerivativeAlgorithm.H:8-22
"""
import numpy as np
import pytest

from ferrox_b200 import decks
from oracle import inputs as I
from oracle import oracle as O


def make(text, **kw):
    return O.Oracle.from_text(text, **kw)


def small_mfim(nx=8, ny=8, nz=12, **extra):
    return decks.mfim(nx, ny, nz, extra=extra or None)


def test_parse_table_last_definition_and_quotes():
    t = I.parse_table('a = 1 2 3\n# comment = 5\nb = "x + y\n  + z"  # tail\na = 7\nc=4')
    assert t["a"] == ["7"]
    assert t["b"] == ["x + y\n  + z"]
    assert t["c"] == ["4"]


def test_defaults_match_reference():
    p = I.ferrox_params(I.parse_table(small_mfim()))
    # FerroX.cpp:333-571 defaults for keys the deck omits
    assert p["delta"] == 1e-6 and p["inc_step"] == -1 and p["phi_tolerance"] == 1e-7
    assert p["num_Vapp_max"] == 1 and p["use_work_function"] == 0
    assert p["epsilonX_fe_tphase"] == p["epsilonX_fe"]
    assert p["Channel_lo"] == [p["prob_lo"][d] - 1.0 for d in range(3)]


def test_material_mask_cell_centre_rule():
    o = make(small_mfim())
    m = o.mask_ghost()
    nz = 12
    dz = 9e-9 / nz
    zc = (np.arange(-1, nz + 1) + 0.5) * dz
    exp_layer = np.where((zc >= 4e-9) & (zc <= 9e-9), 0.0, 1.0)
    # valid and z-ghost layers (x/y ghosts are periodic images)
    assert np.array_equal(m[:, 1, 1], exp_layer)
    assert np.array_equal(m[:, 0, :], m[:, -2, :])     # periodic y ghost
    assert np.array_equal(m[:, :, 0], m[:, :, -2])     # periodic x ghost


def test_landau_closed_form():
    o = make(small_mfim())
    rng = np.random.default_rng(3)
    pz = rng.uniform(-0.3, 0.3, o.shape)
    mask = o.field("mask")
    pz = np.where(mask == 0, pz, 0.0)
    o.set_field("Pz", pz)
    L, G, E = o.tdgl_terms()
    a, b, g = -2.5e9, 6.0e10, 1.5e11
    Gam = np.where(mask == 0, 20.0, 0.0)
    expect = -Gam * (a * pz + b * pz ** 3 + g * pz ** 5)
    np.testing.assert_allclose(L[2], expect, rtol=1e-13, atol=1e-300)
    assert np.all(L[0] == 0) and np.all(L[1] == 0)   # is_polarization_scalar


def test_grad_interior_quadratic_profile():
    # Pz = c z^2: interior FE cells have d2/dz2 = 2c exactly, x/y terms vanish
    o = make(small_mfim())
    mask = o.field("mask")
    dz = 9e-9 / 12
    z = (np.arange(12) + 0.5) * dz
    c = 1e15
    pz = np.broadcast_to((c * z ** 2)[:, None, None], o.shape).copy()
    o.set_field("Pz", pz)
    L, G, E = o.tdgl_terms()
    fe = np.where(mask[:, 0, 0] == 0)[0]
    interior = fe[1:-1]
    g11 = 1e-10
    np.testing.assert_allclose(G[2][interior], -20.0 * (-g11 * 2 * c), rtol=1e-9)


@pytest.mark.parametrize("flag", [0, 1, 2, 3, 4])
def test_lower_fe_boundary_second_derivative_forms(flag):
    # first FE layer above the DE: DoubleDPDz lower-boundary branch
    o = make(small_mfim(**{"P_BC_flag_lo": [3, 3, flag], "P_BC_flag_hi": [3, 3, 2]}))
    mask = o.field("mask")
    dz = 9e-9 / 12
    z = (np.arange(12) + 0.5) * dz
    prof = 0.01 + 1e6 * z + 3e14 * z ** 2
    pz = np.broadcast_to(prof[:, None, None], o.shape).copy()
    o.set_field("Pz", pz)
    L, G, E = o.tdgl_terms()
    k = int(np.where(mask[:, 0, 0] == 0)[0][0])
    F0, F1, F2, Fm = prof[k], prof[k + 1], prof[k + 2], prof[k - 1]
    lam = 3e-9
    if flag == 0:
        d2 = 4. * (2. * 0.0 - 3. * F0 + F1) / 3. / dz / dz
    elif flag == 1:
        Flo = F0 / (1 + dz / 2 / lam)
        d2 = (-dz * Flo / lam - F0 + F1) / dz / dz
    elif flag == 2:
        d2 = (-F0 + F1) / dz / dz
    elif flag == 3:
        d2 = (Fm - 2. * F0 + F1) / dz / dz
    else:
        d2 = (F0 - 2. * F1 + F2) / dz / dz
    np.testing.assert_allclose(G[2][k], -20.0 * (-1e-10 * d2), rtol=1e-12)


def test_poisson_uniform_eps_gives_linear_phi():
    # no FE, uniform DE: the discrete solution with the maxorder-2 Dirichlet
    # ghost is exactly linear between the electrode values
    text = small_mfim(**{"FE_lo": [-1.0, -1.0, -1.0], "FE_hi": [-1.0, -1.0, -1.0],
                         "DE_lo": [-1.0, -1.0, -1.0], "DE_hi": [1.0, 1.0, 1.0],
                         "Phi_Bc_lo": 0.3, "Phi_Bc_hi": 1.1})
    o = make(text)
    phi, its, res = o.poisson_solve(np.zeros(o.shape), rtol=1e-13)
    z = (np.arange(12) + 0.5) * (9e-9 / 12)
    exact = 0.3 + (1.1 - 0.3) * z / 9e-9
    np.testing.assert_allclose(phi, np.broadcast_to(exact[:, None, None], o.shape), rtol=1e-11, atol=1e-12)


def test_poisson_two_layer_vs_independent_tridiagonal():
    o = make(small_mfim(Phi_Bc_hi=0.7))
    nz = 12
    dz = 9e-9 / nz
    eps_cc = np.where(o.field("mask")[:, 0, 0] == 0, 24.0, 9.0) * 8.85e-12
    bf = np.empty(nz + 1)
    bf[0], bf[-1] = eps_cc[0], eps_cc[-1]
    bf[1:-1] = 0.5 * (eps_cc[1:] + eps_cc[:-1])
    A = np.zeros((nz, nz)); b = np.zeros(nz)
    for k in range(nz):
        lo = 2 * bf[k] if k == 0 else bf[k]
        hi = 2 * bf[k + 1] if k == nz - 1 else bf[k + 1]
        A[k, k] = (lo + hi) / dz ** 2
        if k > 0: A[k, k - 1] = -bf[k] / dz ** 2
        if k < nz - 1: A[k, k + 1] = -bf[k + 1] / dz ** 2
    b[-1] = 2 * bf[-1] * 0.7 / dz ** 2
    exact = np.linalg.solve(A, b)
    phi, its, res = o.poisson_solve(np.zeros(o.shape), rtol=1e-13)
    np.testing.assert_allclose(phi, np.broadcast_to(exact[:, None, None], o.shape), rtol=1e-10, atol=1e-13)
    # and it is close to the continuous series-capacitor profile
    kint = int(np.where(eps_cc > 9 * 8.85e-12)[0][0])
    t_de, t_fe = kint * dz, (nz - kint) * dz
    V_fe_bottom = 0.7 * (t_de / 9.0) / (t_de / 9.0 + t_fe / 24.0)
    assert abs(0.5 * (exact[kint] + exact[kint - 1]) - V_fe_bottom) < 0.02


def test_operator_residual_of_solution_is_small():
    o = make(small_mfim(Phi_Bc_hi=0.4))
    rng = np.random.default_rng(5)
    rhs = rng.normal(size=o.shape) * 1e8
    phi, its, res = o.poisson_solve(rhs, rtol=1e-12)
    r = rhs - o.poisson_apply(phi)
    assert np.abs(r).max() <= 1e-11 * max(np.abs(rhs).max(), 1.0) * 10


def test_mass_action_law_and_fd_limit():
    text = decks.mfism(8, 8, 24)
    o = make(text)
    mask = o.field("mask")
    rng = np.random.default_rng(2)
    phi = rng.uniform(-0.3, 0.3, o.shape)
    o.set_field("Phi", phi)
    o.compute_rho()
    n, p = o.field("electrons"), o.field("holes")
    sc = mask >= 2
    ni = o.scalar("ni")
    np.testing.assert_allclose((n * p)[sc], ni ** 2, rtol=1e-12)
    # FD_half -> exp(eta) deep in the Boltzmann regime (eta << 0)
    o2 = make(decks.mfism(8, 8, 24, extra={"use_Fermi_Dirac": 1}))
    o2.set_field("Phi", phi)
    o2.compute_rho()
    np.testing.assert_allclose(o2.field("electrons")[sc], n[sc], rtol=5e-4)


@pytest.mark.parametrize("mode,factor", [("face", 1.0), ("extrap", 5.0 / 3.0)])
def test_E_from_linear_phi(mode, factor):
    text = small_mfim(**{"FE_lo": [-1.0, -1.0, -1.0], "FE_hi": [-1.0, -1.0, -1.0],
                         "DE_lo": [-1.0, -1.0, -1.0], "DE_hi": [1.0, 1.0, 1.0],
                         "Phi_Bc_hi": 0.9, "fx.phi_ghost_mode": mode})
    o = make(text)
    o.compute_phi_rho()
    o.compute_E()
    Ez = o.field("Ez")
    s = 0.9 / 9e-9
    np.testing.assert_allclose(Ez[1:-1], -s, rtol=1e-9)
    # electrode cells: one-sided DphiDz reading the ghost
    np.testing.assert_allclose(Ez[0], -s * factor, rtol=1e-9)
    np.testing.assert_allclose(Ez[-1], -s * factor, rtol=1e-9)
    assert np.abs(o.field("Ex")).max() < 1e-6 * s


def test_newton_loop_converges_with_semiconductor():
    o = make(decks.mfism(8, 8, 24, extra={"Phi_Bc_hi": 0.5}))
    o.set_phi_bc()
    o.compute_phi_rho()
    assert o.scalar("contains_sc") == 1
    assert 2 <= o.scalar("newton_iters") <= 50
    assert o.scalar("phi_err") <= 1e-5


def test_uniform_stream_is_splitmix64():
    # splitmix64: state += golden; mix(state); top 53 bits
    golden = 0x9E3779B97F4A7C15
    M = (1 << 64) - 1

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M
        z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M
        return z ^ (z >> 31)
    for n in [1, 2, 1000]:
        assert O.uniform(7, n) == (mix((7 + n * golden) & M) >> 11) * 2.0 ** -53


def test_oracle_is_independent_of_its_thread_count():
    """Every reduction of the oracle folds in a fixed order, so its fields do not depend
    on the OpenMP thread count (5 Newton-coupled steps of a small MFISM stack)."""
    L = O.lib()
    before = L.ofx_set_threads(0)       # 0 reads the current count without changing it
    try:
        runs = []
        for th in (1, 3, 8):
            o = make(decks.mfism(16, 16, 48), threads=th)
            for s in range(1, 6):
                o.step(s)
            runs.append({n: o.field(n).copy() for n in ["Pz", "Phi", "charge"]})
        for r in runs[1:]:
            for n in r:
                assert np.array_equal(r[n], runs[0][n]), n
    finally:
        L.ofx_set_threads(before)
