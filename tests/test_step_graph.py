"""A coupled step as one CUDA graph with its Newton and multigrid loop tests
on the device (fx.step_graph = 1, the default) against the host-driven loop
(fx.step_graph = 0).  Both launch the same kernels in the same order on the
same data, so every field must be bit-identical after several steps, and so
must the V-cycle and Newton counts; a failure in ComputePhi_Rho must stop the
step before the TDGL update with the same error in both.
"""
import numpy as np
import pytest

from ferrox_b200 import api, decks
from helpers import small_grains

pytestmark = pytest.mark.gpu


def start_P(shape, seed, vector=False):
    g = np.random.default_rng(seed)
    Pz = g.uniform(-0.05, 0.05, shape)
    if not vector:
        return (None, None, Pz)
    return (g.uniform(-0.05, 0.05, shape), g.uniform(-0.05, 0.05, shape), Pz)


def make(text, P, graph, precision=None, grains=None, params=None):
    f = api.FerroX(text, precision=precision)
    if grains is not None:
        f.set_grains(grains["id"], grains["angles"], grains["tphase"])
    f.set_initial_P(*P)
    f.set_param("fx.step_graph", graph)
    for k, v in (params or {}).items():
        f.set_param(k, v)
    return f


FIELDS = ["Px", "Py", "Pz", "Phi", "charge", "Ez"]

CASES = {
    # Newton-coupled semiconductor stack, the voltage stepping every 3 steps
    "mfism_fp64": dict(text=decks.mfism(16, 16, 48, steps_per_voltage=3, v_step=0.1), shape=(48, 16, 16)),
    "mfism_mixed": dict(text=decks.mfism(16, 16, 48, steps_per_voltage=3, v_step=0.1), shape=(48, 16, 16),
                        precision="mixed"),
    "mfism_order2": dict(text=decks.mfism(16, 16, 48, steps_per_voltage=4, extra={"TimeIntegratorOrder": 2}),
                         shape=(48, 16, 16)),
    "mfim_fp64": dict(text=decks.mfim(32, 32, 12, Phi_Bc_hi=0.8), shape=(12, 32, 32)),
    "mfim_mixed": dict(text=decks.mfim(32, 32, 12, Phi_Bc_hi=0.8), shape=(12, 32, 32), precision="mixed"),
    "mfim_order2_cold": dict(text=decks.mfim(32, 32, 12, Phi_Bc_hi=0.8, extra={"TimeIntegratorOrder": 2}),
                             shape=(12, 32, 32), params={"fx.warm_start": 0}),
    "mfim_no_extrapolation": dict(text=decks.mfim(32, 32, 12, Phi_Bc_hi=0.8), shape=(12, 32, 32),
                                  params={"fx.phi_extrapolate": 0}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_graph_step_bit_identical(case):
    cfg = CASES[case]
    P = start_P(cfg["shape"], 11)
    runs = []
    for graph in (0, 1):
        f = make(cfg["text"], P, graph, precision=cfg.get("precision"), params=cfg.get("params"))
        f.set_param("fx.mg_rtol", 1e-12)
        f.step(11)
        assert f.param("step_graph_ran") == graph
        runs.append(({n: f.field(n) for n in FIELDS}, f.stats()))
        f.close()
    (a, sa), (b, sb) = runs
    for n in FIELDS:
        assert np.array_equal(a[n], b[n]), (case, n)
    for k in ("mg_cycles_total", "newton_iters_total", "mg_cycles_last", "newton_iters_last", "step", "num_Vapp"):
        assert sa[k] == sb[k], (case, k, sa[k], sb[k])
    assert sa["mg_resid_last"] == sb["mg_resid_last"]
    assert sa["phi_err_last"] == sb["phi_err_last"]
    assert sa["steady_err_last"] == sb["steady_err_last"]


def test_graph_step_rotated_grains_vector_P():
    text, g = small_grains(16, 16, 24)
    text = text.replace("is_polarization_scalar = 1", "is_polarization_scalar = 0")
    P = start_P((24, 16, 16), 12, vector=True)
    out = []
    for graph in (0, 1):
        f = make(text, P, graph, precision="mixed", grains=g)
        f.step(6)
        assert f.param("step_graph_ran") == graph
        out.append({n: f.field(n) for n in FIELDS})
        f.close()
    for n in FIELDS:
        assert np.array_equal(out[0][n], out[1][n]), n


@pytest.mark.parametrize("key,val,fragment", [("fx.mg_max_iter", 1, "Poisson multigrid did not reach"),
                                               ("fx.newton_max_iter", 1, "Phi-rho Newton iteration did not reach")])
def test_graph_step_failure_stops_before_tdgl(key, val, fragment):
    text = decks.mfism(16, 16, 48)
    P = start_P((48, 16, 16), 13)
    res = []
    for graph in (0, 1):
        f = make(text, P, graph)
        f.set_param("fx.mg_rtol", 1e-13)
        f.step(2)
        before = f.field("Pz")
        f.set_param(key, val)
        with pytest.raises(api.FxError) as e:
            f.step(1)
        assert e.value.code == -5
        assert fragment in str(e.value)
        assert np.array_equal(f.field("Pz"), before)
        assert f.stats()["step"] == 2
        res.append(str(e.value))
        f.close()
    assert res[0] == res[1]


def test_graph_step_launches_counted():
    f = make(decks.mfism(16, 16, 48), start_P((48, 16, 16), 14), 1)
    f.step(1)
    l0 = f.stats()["kernel_launches"]
    f.step(3)
    s = f.stats()
    # per step at least the TDGL update, two Newton passes of charge and
    # linearisation kernels, and a V-cycle of a handful of levels
    assert s["kernel_launches"] - l0 >= 3 * 20
    f.close()


@pytest.mark.parametrize("precision", [None, "mixed"])
def test_programmatic_launch_bit_identical(precision):
    # fx.pdl lets a kernel be scheduled while its predecessor drains; every
    # kernel waits for its predecessor before touching memory, so the fields
    # are those of plain stream order
    text = decks.mfism(32, 32, 48, steps_per_voltage=3, v_step=0.1)
    P = start_P((48, 32, 32), 15)
    out = []
    try:
        for pdl in (0, 1):
            f = make(text, P, 1, precision=precision)
            f.set_param("fx.pdl", pdl)
            f.step(8)
            assert f.param("fx.pdl") == pdl
            out.append({n: f.field(n) for n in FIELDS})
            f.close()
    finally:
        f = api.FerroX(decks.mfim(8, 8, 12))
        f.set_param("fx.pdl", 1)
        f.close()
    for n in FIELDS:
        assert np.array_equal(out[0][n], out[1][n]), n


@pytest.mark.parametrize("precision", [None, "mixed"])
def test_coarse_alpha_tiles_bit_identical(precision):
    # every coarse Newton coefficient below level 1 from one tiled launch
    # equals the per-level averaging launches
    text = decks.mfism(32, 32, 48, steps_per_voltage=3, v_step=0.1)
    P = start_P((48, 32, 32), 16)
    out = []
    for tiles in (0, 1):
        f = make(text, P, 1, precision=precision, params={"fx.alpha_tiles": tiles})
        f.step(7)
        out.append(({n: f.field(n) for n in FIELDS}, f.stats()["mg_cycles_total"]))
        f.close()
    for n in FIELDS:
        assert np.array_equal(out[0][0][n], out[1][0][n]), n
    assert out[0][1] == out[1][1]


def test_fresh_contexts_bit_identical():
    # two contexts of the same deck give the same fields and cycle counts:
    # every reduction is order-fixed (the right-hand-side norms that set the
    # multigrid target on stacks without a semiconductor included)
    out = []
    for _ in range(2):
        f = api.FerroX(decks.mfim(32, 32, 12))
        f.step(60)
        out.append(({n: f.field(n) for n in FIELDS}, f.stats()["mg_cycles_total"]))
        f.close()
    for n in FIELDS:
        assert np.array_equal(out[0][0][n], out[1][0][n]), n
    assert out[0][1] == out[1][1]


INTERIOR_CASES = {
    # rotated scalar P in grains (the Hessian with its mixed derivatives)
    "polycrystal_fp64": dict(grains=True, precision=None, vector=False),
    "polycrystal_mixed": dict(grains=True, precision="mixed", vector=False),
    # vector P in rotated grains
    "polycrystal_vector": dict(grains=True, precision=None, vector=True),
    # layered stacks, scalar P, with the Newton-coupled semiconductor
    "mfism_fp64": dict(text=decks.mfism(32, 32, 48, steps_per_voltage=3, v_step=0.1), shape=(48, 32, 32)),
    "mfim_mixed": dict(text=decks.mfim(32, 32, 24, Phi_Bc_hi=0.8), shape=(24, 32, 32), precision="mixed"),
}


@pytest.mark.parametrize("case", sorted(INTERIOR_CASES))
def test_interior_fast_path_bit_identical(case):
    """Cells whose whole stencil is ferroelectric evaluate the TDGL gradient
    terms and the Poisson right-hand side through the interior views
    (fx.interior = 1, the default): the same stencil code with the mask tests
    known to pass.  With every cell on the general path (fx.interior = 0) the
    cycle counts are the same and the fields agree to 1e-12: the compiler may
    fuse a product into an add (FMA) on one path and not on the other, a
    last-bit difference."""
    cfg = INTERIOR_CASES[case]
    grains = None
    if cfg.get("grains"):
        extra = {"Phi_Bc_hi": 0.7}
        if cfg.get("vector"):
            extra.update({"is_polarization_scalar": 0, "g12": 2.0e-11})
        text, grains = decks.polycrystal(32, 32, 48, ngrains=6, seed=4, nsteps=10, extra=extra)
        shape = (48, 32, 32)
    else:
        text, shape = cfg["text"], cfg["shape"]
    P = start_P(shape, 5, vector=cfg.get("vector", False))
    runs = []
    for interior in (0, 1):
        f = make(text, P, 1, precision=cfg.get("precision"), grains=grains, params={"fx.interior": interior})
        f.step(6)
        f.compute_E()
        runs.append(({n: f.field(n) for n in FIELDS + ["PoissonRHS"]}, f.stats()["mg_cycles_total"],
                     f.stats()["newton_iters_total"]))
        f.close()
    (a, ca, na), (b, cb, nb) = runs
    assert (ca, na) == (cb, nb)
    for n in a:
        scale = np.abs(b[n]).max()
        assert np.abs(a[n] - b[n]).max() <= 1e-12 * scale, (n, np.abs(a[n] - b[n]).max() / scale)


SEG_CASES = {
    # level 0 from the material codes, coarse levels from face-beta arrays;
    # 256-cell rows: 32 FP32 segments per row, one row per warp
    "polycrystal_fp64": dict(grains=(256, 32, 48), precision=None),
    "polycrystal_mixed": dict(grains=(256, 32, 48), precision="mixed", split=True),
    # 64-cell rows: several rows per warp (the even-offsets-first row order)
    "polycrystal_mixed_64": dict(grains=(64, 64, 48), precision="mixed", split=True),
    # layered stacks: face beta by plane, alpha from the Newton-coupled semiconductor
    "mfism_fp64": dict(text=decks.mfism(32, 32, 48, steps_per_voltage=3, v_step=0.1), shape=(48, 32, 32)),
    "mfism_mixed": dict(text=decks.mfism(32, 32, 48, steps_per_voltage=3, v_step=0.1), shape=(48, 32, 32),
                        precision="mixed"),
    "mfim_mixed": dict(text=decks.mfim(64, 64, 24, Phi_Bc_hi=0.8), shape=(24, 64, 64), precision="mixed"),
    # level 0 -> 1 by z alone, so the mixed path takes the split layout, with alpha
    "mfism_mixed_split": dict(text=decks.mfism(32, 32, 144, steps_per_voltage=3, v_step=0.1), shape=(144, 32, 32),
                              precision="mixed", split=True),
}


@pytest.mark.parametrize("case", sorted(SEG_CASES))
def test_segment_smoother_bit_identical(case):
    """The row-segment red-black half sweep (fx.mg_seg = 16 or 32 bytes per
    thread; every level whose rows it can take, fx.mg_seg_min = 0) repeats the
    per-cell operations of the one-cell-per-thread sweep (fx.mg_seg = 0) with
    the same roundings, and so do the kernels on level 0's red-black split
    layout of the mixed path (fx.mg_split = 1, the default, against 0): fields
    and V-cycle counts are bit-identical, in the step graph and in the
    host-driven loop."""
    cfg = SEG_CASES[case]
    grains = None
    if cfg.get("grains"):
        nx, ny, nz = cfg["grains"]
        text, grains = decks.polycrystal(nx, ny, nz, ngrains=6, seed=4, nsteps=10, extra={"Phi_Bc_hi": 0.7})
        shape = (nz, ny, nx)
    else:
        text, shape = cfg["text"], cfg["shape"]
    P = start_P(shape, 7)
    for graph in (1, 0):
        runs = []
        settings = [(0, 1), (16, 1), (32, 1), (16, 0)]
        for seg, split in settings:
            f = make(text, P, graph, precision=cfg.get("precision"), grains=grains,
                     params={"fx.mg_seg": seg, "fx.mg_seg_min": 0, "fx.mg_split": split})
            f.step(5)
            runs.append(({n: f.field(n) for n in FIELDS}, f.stats()["mg_cycles_total"],
                         f.stats()["newton_iters_total"]))
            if cfg.get("split") and seg:
                assert f.param("mg_level0_split") == split, (seg, split)
            f.close()
        a, ca, na = runs[0]
        for (seg, split), (b, cb, nb) in zip(settings[1:], runs[1:]):
            assert (ca, na) == (cb, nb), (graph, seg, split, ca, cb, na, nb)
            for n in FIELDS:
                assert np.array_equal(a[n], b[n]), (graph, seg, split, n, np.abs(a[n] - b[n]).max())


def test_no_pre_smoothing_starts_from_a_zero_correction():
    """fx.mg_nu1 = 0 (no pre-smoothing on level 0): the mixed path's FP32
    correction cycle starts from zero without a sweep to clear it, so the
    smoother clears it; the fields match the default cycle's to the solver
    tolerance."""
    text = decks.mfim(32, 32, 24, Phi_Bc_hi=0.8)
    P = start_P((24, 32, 32), 3)
    out = []
    for nu1 in (2, 0):
        f = make(text, P, 1, precision="mixed", params={"fx.mg_nu1": nu1})
        f.step(4)
        out.append({n: f.field(n) for n in ("Pz", "Phi")})
        f.close()
    for n in ("Pz", "Phi"):
        scale = np.abs(out[0][n]).max()
        assert np.abs(out[0][n] - out[1][n]).max() <= 1e-7 * scale, n


@pytest.mark.parametrize("graph", [1, 0], ids=["step_graph", "host_loop"])
def test_fp16_coarse_faces_change_convergence_only(graph):
    """The FP32 correction cycle's coarse face beta in FP16 (fx.mg_half = 1,
    the default) against FP32 arrays (0): the coarse operators only
    precondition the FP64 refinement, so both runs solve the same FP64
    Poisson problem to the same residual bound; the fields agree to the
    solver tolerance."""
    text, grains = decks.polycrystal(64, 64, 48, ngrains=6, seed=4, nsteps=10, extra={"Phi_Bc_hi": 0.7})
    P = start_P((48, 64, 64), 9)
    out = []
    for half in (0, 1):
        f = api.FerroX(text, precision="mixed")
        f.set_param("fx.mg_half", half)
        f.set_grains(grains["id"], grains["angles"], grains["tphase"])
        f.set_initial_P(*P)
        f.set_param("fx.step_graph", graph)
        f.step(5)
        out.append({n: f.field(n) for n in ("Pz", "Phi", "Ez")})
        f.close()
    for n in out[0]:
        scale = np.abs(out[0][n]).max()
        assert np.abs(out[0][n] - out[1][n]).max() <= 1e-7 * scale, (n, np.abs(out[0][n] - out[1][n]).max() / scale)


@pytest.mark.parametrize("case", ["polycrystal_mixed", "polycrystal_fp64", "mfism_fp64"])
def test_rhs_segment_kernel_bit_identical(case):
    """The scalar Poisson right-hand side by row segments (fx.rhs_seg = 1, the
    default, process-wide) repeats the per-cell kernel's operations: fields,
    the right-hand side and the cycle counts are bit-identical."""
    if case.startswith("polycrystal"):
        text, grains = decks.polycrystal(64, 64, 48, ngrains=6, seed=4, nsteps=10, extra={"Phi_Bc_hi": 0.7})
        shape = (48, 64, 64)
    else:
        text, grains = decks.mfism(32, 32, 48, steps_per_voltage=3, v_step=0.1), None
        shape = (48, 32, 32)
    prec = "mixed" if case.endswith("mixed") else None
    P = start_P(shape, 5)
    runs = []
    try:
        for seg in (0, 1):
            f = make(text, P, 1, precision=prec, grains=grains)
            f.set_param("fx.rhs_seg", seg)
            f.step(5)
            f.compute_E()
            runs.append(({n: f.field(n) for n in FIELDS + ["PoissonRHS"]}, f.stats()["mg_cycles_total"]))
            f.close()
    finally:
        g = api.FerroX(decks.mfim(8, 8, 12))
        g.set_param("fx.rhs_seg", 1)
        g.close()
    (a, ca), (b, cb) = runs
    assert ca == cb
    for n in a:
        assert np.array_equal(a[n], b[n]), (n, np.abs(a[n] - b[n]).max())


@pytest.mark.parametrize("case", ["polycrystal_mixed", "polycrystal_fp64", "mfim_fp64"])
def test_dense_coarse_solve_changes_convergence_only(case):
    """With alpha absent the one-CTA levels are replaced by the exact solve
    with the dense inverse of their first level (fx.mg_dense = 1, the
    default); against the one-CTA V-cycle (0) the fields agree to the solver
    tolerance, in the step graph and in the host-driven loop."""
    if case.startswith("polycrystal"):
        text, grains = decks.polycrystal(64, 64, 48, ngrains=6, seed=4, nsteps=10, extra={"Phi_Bc_hi": 0.7})
        shape = (48, 64, 64)
    else:
        text, grains = decks.mfim(32, 32, 24, Phi_Bc_hi=0.8), None
        shape = (24, 32, 32)
    prec = "mixed" if case.endswith("mixed") else None
    P = start_P(shape, 13)
    for graph in (1, 0):
        out = []
        for dense in (0, 1):
            f = make(text, P, graph, precision=prec, grains=grains, params={"fx.mg_dense": dense})
            f.step(5)
            out.append({n: f.field(n) for n in ("Pz", "Phi", "Ez")})
            f.close()
        for n in out[0]:
            scale = np.abs(out[0][n]).max()
            assert np.abs(out[0][n] - out[1][n]).max() <= 1e-7 * scale, (graph, n)
