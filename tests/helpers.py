"""Shared helpers: build the GPU context and the CPU oracle from one deck."""
import numpy as np

from ferrox_b200 import api, decks
from oracle import inputs as I
from oracle import oracle as O


def relerr(a, b) -> float:
    """max |a - b| / max |b| (absolute when b is identically zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    d = np.abs(a - b).max()
    return float(d / scale) if scale > 0 else float(d)


def pair(text, grains=None, P=None, precision=None, rtol=None):
    """(FerroX on the GPU, Oracle on the CPU) for the same inputs text."""
    f = api.FerroX(text, precision=precision)
    table = I.parse_table(text)
    p = I.ferrox_params(table)
    if grains is not None:
        tph, ang = decks.grain_fields(grains)
        o = O.Oracle(p, tph, tuple(ang))
        f.set_grains(grains["id"], grains["angles"], grains["tphase"])
    else:
        tph, a, b, t = I.function_fields(table, p)
        o = O.Oracle(p, tph, (a, b, t))
    eb = I.embedded_boundary(table, p)
    if eb is not None:
        o.set_eb(*eb)
    if P is not None:
        f.set_initial_P(*P)
        for name, comp in zip(["Px", "Py", "Pz"], P):
            o.set_field(name, np.zeros(o.shape) if comp is None else comp)
    if rtol is not None:
        f.set_param("fx.mg_rtol", rtol)
        o.set_scalar("mg_rtol", rtol)
    return f, o


def small_grains(nx, ny, nz, ngrains=6, seed=3):
    text, g = decks.polycrystal(nx, ny, nz, ngrains=ngrains, seed=seed, nsteps=10)
    return text, g
