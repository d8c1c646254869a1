"""Embedded boundaries in the grid-aligned form of the reference's FET decks.

`domain.embedded_boundary = 1` hands the Poisson solve to AMReX's
MLEBABecLap with a Dirichlet value on the embedded surface
(ElectrostaticSolver.cpp:613-676; objects read by
EmbeddedBoundaries.cpp:66-140).  The reference's decks inputs_mfim_eb and
inputs_mfis_eb place one box with no fluid inside over the top of the stack,
its lower face on a grid face: the solve then runs on the fluid layers below
the face, which is a Dirichlet face at surf_soln, and the covered cells keep
the 0 each solve starts from.  Cut-cell geometries are refused.

CPU: the two decks are accepted with the layer count both readers find,
unsupported geometries are refused by both, and the oracle's solve with the
embedded face equals its solve of the deck cut at that face with the top
electrode at surf_soln.  GPU: coupled steps of both decks against the oracle.
"""
import os

import numpy as np
import pytest

from ferrox_b200 import api
from helpers import pair, relerr
from oracle import inputs as I
from oracle import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "decks")
MFIM_EB = "Examples_inputs_mfim_eb.inputs"
MFIS_EB = "Examples_inputs_mfis_eb.inputs"


def deck(name: str) -> str:
    with open(os.path.join(HERE, name)) as f:
        return f.read()


def with_keys(text: str, **kv) -> str:
    """The deck with keys replaced (dots written as '__'); None drops a key."""
    keys = {k.replace("__", "."): v for k, v in kv.items()}
    out = []
    for line in text.splitlines():
        k = line.split("=", 1)[0].strip()
        if k in keys:
            continue
        out.append(line)
    for k, v in keys.items():
        if v is not None:
            out.append(f"{k} = {v}")
    return "\n".join(out) + "\n"


@pytest.mark.parametrize("name,layers", [(MFIM_EB, 18), (MFIS_EB, 32)])
def test_reference_eb_decks_accepted(name, layers):
    text = deck(name)
    f = api.FerroX(text)
    try:
        assert f.param("eb_fluid_layers") == layers
        assert f.param("eb_surf_soln") == 0.0
    finally:
        f.close()
    table = I.parse_table(text)
    assert I.embedded_boundary(table, I.ferrox_params(table)) == (layers, 0.0)


REFUSED = [
    ({"MyGeom__geom_type": "plane"}, "geom_type plane"),
    ({"MyGeom__has_fluid_inside": "1"}, "has_fluid_inside = 1"),
    ({"MyGeom__box_lo": "-16.0e-9 -16.0e-9 9.2e-9"}, "not on a cell face"),
    ({"MyGeom__box_lo": "-8.0e-9 -16.0e-9 9.0e-9"}, "does not span the domain in x"),
    ({"MyGeom__box_hi": "16.0e-9 16.0e-9 9.5e-9"}, "does not reach the top"),
    ({"ebgeom__objects": "MyGeom Other"}, "a union of 2 objects"),
    ({"ebgeom__specify_input_using_eb2": "1"}, "specify_input_using_eb2"),
    ({"MyGeom__box_lo": "-16.0e-9 -16.0e-9 0.0"}, "leaves no fluid layer"),
]


@pytest.mark.parametrize("edit,why", REFUSED, ids=[w for _, w in REFUSED])
def test_unsupported_geometry_refused(edit, why):
    text = with_keys(deck(MFIM_EB), **edit)
    with pytest.raises(api.FxError) as e:
        api.FerroX(text)
    assert e.value.code == -3 and why in str(e.value), str(e.value)
    table = I.parse_table(text)
    with pytest.raises(ValueError):
        I.embedded_boundary(table, I.ferrox_params(table))


def test_without_embedded_boundary_the_top_must_be_an_electrode():
    """With the flag off the same deck has its Neumann top boundary back,
    which the electrode layout refuses; with electrodes it runs as before."""
    off = with_keys(deck(MFIM_EB), domain__embedded_boundary="0")
    with pytest.raises(api.FxError) as e:
        api.FerroX(off)
    assert e.value.code == -3 and "Dirichlet" in str(e.value)
    f = api.FerroX(with_keys(off, boundary__hi="per per dir(0.0)"))
    try:
        assert f.param("eb_fluid_layers") == 0
    finally:
        f.close()


def truncated(text: str, kb: int, V: float) -> str:
    """The deck cut at the embedded face: kb layers, the top electrode at V."""
    t = I.parse_table(text)
    p = I.ferrox_params(t)
    h = (p["prob_hi"][2] - p["prob_lo"][2]) / p["n_cell"][2]
    lo, hi, n = p["prob_lo"], p["prob_hi"], p["n_cell"]
    return with_keys(text, domain__embedded_boundary="0", boundary__hi="per per dir(0.0)",
                     domain__n_cell=f"{n[0]} {n[1]} {kb}", domain__max_grid_size=f"{n[0]} {n[1]} {kb}",
                     domain__prob_hi=f"{hi[0]!r} {hi[1]!r} {lo[2] + kb * h!r}", Phi_Bc_hi=repr(V))


@pytest.mark.parametrize("name", [MFIM_EB, MFIS_EB])
def test_oracle_embedded_face_is_a_dirichlet_face(name):
    """The oracle's solve on the fluid layers equals its solve of the deck
    cut at the embedded face with the top electrode at surf_soln (the same
    operator, built by its own non-EB path), for a nonzero surf_soln."""
    V = 0.37
    text = with_keys(deck(name), MyGeom__surf_soln=repr(V))
    t0 = I.parse_table(deck(name))
    n = I.ferrox_params(t0)["n_cell"]
    text = with_keys(text, domain__n_cell=f"8 8 {n[2]}", domain__max_grid_size=f"8 8 {n[2]}")
    o = O.Oracle.from_text(text)
    tab = I.parse_table(text)
    kb, Vs = I.embedded_boundary(tab, I.ferrox_params(tab))
    assert Vs == V
    ref = O.Oracle.from_text(truncated(text, kb, V))
    rng = np.random.default_rng(5)
    nz = n[2]
    rhs = rng.standard_normal((nz, 8, 8)) * 1e-3
    o.set_phi_bc(); ref.set_phi_bc()
    phi = o.poisson_solve(rhs, rtol=1e-13)[0]
    phi_t = ref.poisson_solve(np.ascontiguousarray(rhs[:kb]), rtol=1e-13)[0]
    assert relerr(phi[:kb], phi_t) < 1e-12
    assert np.all(phi[kb:] == 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", [MFIM_EB, MFIS_EB])
def test_eb_deck_coupled_steps(name, precision):
    """The reference's EB decks as given (64 x 64 x 20 and 64 x 64 x 34 with
    a semiconductor), five coupled steps on the GPU against the oracle; the
    bounds are those of the electrode decks' coupled steps (1e-10 in FP64,
    1e-6 for the mixed path's FP32 terms)."""
    tol = 1e-10 if precision == "fp64" else 1e-6
    f, o = pair(deck(name), precision=precision, rtol=1e-13)
    kb = int(f.param("eb_fluid_layers"))
    try:
        for step in range(1, 6):
            f.step(1)
            o.step(step)
        o.compute_E()
        for field in ["Pz", "Phi", "Ez"]:
            assert relerr(f.field(field), o.field(field)) < tol, field
        # the covered cells are not part of the solve: phi there stays 0
        assert np.all(f.field("Phi")[kb:] == 0.0)
    finally:
        f.close()


@pytest.mark.gpu
def test_executable_runs_the_reference_eb_deck(tmp_path):
    """The reference's inputs_mfim_eb file through the executable, as the
    reference's own binary takes it: plotfiles of the full 64 x 64 x 20 grid
    with phi 0 in the covered layers, and the library's fields to within the
    deck's solver tolerance (the executable also writes the step-0 plotfile)."""
    import subprocess

    from ferrox_b200 import build, plotfile
    build.build()
    exe = os.path.join(os.path.dirname(os.path.dirname(HERE)), "..", "ferrox_b200", "ferrox_b200")
    deck_path = tmp_path / "inputs_mfim_eb"
    deck_path.write_text(deck(MFIM_EB))
    r = subprocess.run([os.path.abspath(exe), str(deck_path), "nsteps=4", "plot_int=2"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for step in (0, 2, 4):
        assert (tmp_path / f"plt{step:08d}").is_dir(), step
    pf = plotfile.read(str(tmp_path / "plt00000004"))
    assert pf["n"] == [64, 64, 20] and pf["step"] == 4
    phi = pf["fields"]["Phi"]
    assert np.all(phi[18:] == 0.0) and np.abs(phi[:18]).max() > 0.0
    f = api.FerroX(with_keys(deck(MFIM_EB), nsteps="4", plot_int="2"))
    try:
        f.step(4)
        for name in ["Pz", "Phi", "Ez"]:
            assert relerr(pf["fields"][name], f.field(name)) < 1e-8, name
    finally:
        f.close()


def test_oracle_embedded_face_known_answer():
    """Without charge the layered MFIM stack under the embedded metal is a
    chain of conductances in z: eps of the bottom cell over half a cell to the
    electrode, the face averages 0.5 (eps_k + eps_k+1) between layers, and eps
    of the top fluid cell over half a cell to the embedded surface.  The
    oracle's 3D solve with the embedded face equals that chain's solution."""
    V, Vlo = 0.5, -0.2
    text = with_keys(deck(MFIM_EB), MyGeom__surf_soln=repr(V), Phi_Bc_lo=repr(Vlo),
                     domain__n_cell="8 8 20", domain__max_grid_size="8 8 20")
    o = O.Oracle.from_text(text)
    tab = I.parse_table(text)
    kb, _ = I.embedded_boundary(tab, I.ferrox_params(tab))
    o.set_phi_bc()
    phi = o.poisson_solve(np.zeros((20, 8, 8)), rtol=1e-14)[0]
    eps = o.field("epsilon")[:kb, 0, 0]
    assert np.all(o.field("epsilon")[:kb] == eps[:, None, None])   # layered
    # conductances per unit area times h: bottom, the kb - 1 interior faces, top
    g = np.concatenate([[2 * eps[0]], 0.5 * (eps[:-1] + eps[1:]), [2 * eps[-1]]])
    A = np.zeros((kb, kb))
    r = np.zeros(kb)
    for k in range(kb):
        A[k, k] = g[k] + g[k + 1]
        if k > 0:
            A[k, k - 1] = -g[k]
        if k < kb - 1:
            A[k, k + 1] = -g[k + 1]
    r[0] += g[0] * Vlo
    r[-1] += g[kb] * V
    chain = np.linalg.solve(A, r)
    for j in range(8):
        for i in range(8):
            assert np.allclose(phi[:kb, j, i], chain, rtol=0, atol=1e-12 * abs(V - Vlo))
    assert np.all(phi[kb:] == 0.0)


@pytest.mark.gpu
def test_set_phi_keeps_covered_cells_zero():
    """phi written through fx_set_field: the fluid layers take it, the
    covered layers keep 0 (they are not unknowns of the solve)."""
    f = api.FerroX(with_keys(deck(MFIM_EB), domain__n_cell="16 16 20", domain__max_grid_size="16 16 20"))
    try:
        kb = int(f.param("eb_fluid_layers"))
        f.set_field("Phi", np.full((20, 16, 16), 0.25))
        phi = f.field("Phi")
        assert np.all(phi[:kb] == 0.25) and np.all(phi[kb:] == 0.0)
    finally:
        f.close()
