"""Synthetic device decks in FerroX inputs-file syntax.

Each function returns the text of an inputs file that the reference's
``InitializeFerroXNamespace`` (Source/FerroX.cpp:273-572) would accept, plus
the ``fx.*`` keys of this library.  Sizes default to the named workloads:

* ``mfim``        -- MFIM stack, 5 nm HZO on 4 nm Al2O3, 64x64x36 cells
* ``mfism``       -- MFISM stack, 5 nm HZO / 1 nm SiO2 / 30 nm p-Si, 128x128x144
* ``polycrystal`` -- 256x256x128 film of 64 Voronoi grains (grain arrays
                     returned separately, they have no inputs-file form)
* ``hysteresis``  -- 128x128x48 MFIM stack under a triangular voltage sweep

All are synthetic: no dataset or checkpoint is involved.
"""
from __future__ import annotations

import numpy as np

_MAT = dict(epsilon_0=8.85e-12, epsilonZ_fe=24.0, epsilon_si=11.7, alpha=-2.5e9, beta=6.0e10, gamma=1.5e11,
            alpha_12=0.0, alpha_112=0.0, alpha_123=0.0, g44_p=0.0, g12=0.0)


def _fmt(v) -> str:
    if isinstance(v, (list, tuple)):
        return " ".join(_fmt(x) for x in v)
    if isinstance(v, float):
        return repr(v)
    return str(v)


def render(keys: dict) -> str:
    return "".join(f"{k} = {_fmt(v)}\n" for k, v in keys.items())


def _common(nx, ny, nz, lx, lz, dt, nsteps, seed):
    return {
        "domain.prob_lo": [-lx / 2, -lx / 2, 0.0],
        "domain.prob_hi": [lx / 2, lx / 2, lz],
        "domain.n_cell": [nx, ny, nz],
        "domain.max_grid_size": [nx, ny, nz],
        "domain.blocking_factor": [nx, ny, nz],
        "domain.is_periodic": [1, 1, 0],
        "domain.coord_sys": "cartesian",
        "boundary.lo": "per per dir(0.0)",
        "boundary.hi": "per per dir(0.0)",
        "prob_type": 2,
        "TimeIntegratorOrder": 1,
        "nsteps": nsteps,
        "plot_int": -1,
        "dt": dt,
        "random_seed": seed,
        "is_polarization_scalar": 1,
        "Remnant_P": [0.0, 0.0, 0.002],
        "P_BC_flag_lo": [3, 3, 0],
        "P_BC_flag_hi": [3, 3, 1],
        "lambda": 3.0e-9,
    }


def mfim(nx=64, ny=64, nz=36, dxy=0.5e-9, nsteps=1000, seed=1, BigGamma=20.0, Phi_Bc_hi=0.0, extra=None) -> str:
    """Plain MFIM stack: DE (eps_r 9) 0-4 nm, FE HZO (eps_r 24) 4-9 nm."""
    lx, lz = nx * dxy, 9.0e-9
    k = _common(nx, ny, nz, lx, lz, 1.0e-13, nsteps, seed)
    k.update({
        "Phi_Bc_lo": 0.0, "Phi_Bc_hi": Phi_Bc_hi,
        "DE_lo": [-lx / 2, -lx / 2, 0.0], "DE_hi": [lx / 2, lx / 2, 4.0e-9],
        "FE_lo": [-lx / 2, -lx / 2, 4.0e-9], "FE_hi": [lx / 2, lx / 2, 9.0e-9],
        "SC_lo": [-1.0, -1.0, -1.0], "SC_hi": [-1.0, -1.0, -1.0],
        "epsilonX_fe": 24.0, "epsilon_de": 9.0,
        "BigGamma": BigGamma, "g11": 1.0e-10, "g44": 1.0e-10,
        "use_Fermi_Dirac": 0,
    })
    k.update(_MAT)
    if extra:
        k.update(extra)
    return render(k)


def mfism(nx=128, ny=128, nz=144, dxy=0.5e-9, nsteps=4000, seed=1, steps_per_voltage=200, v_step=0.05,
          v_max=1.0, extra=None) -> str:
    """MFISM stack: p-Si (N_A 1e24 m^-3) 0-30 nm, SiO2 30-31 nm, HZO 31-36 nm,
    Boltzmann carriers, fixed-cadence voltage ramp 0 -> v_max."""
    lx, lz = nx * dxy, 36.0e-9
    k = _common(nx, ny, nz, lx, lz, 1.0e-13, nsteps, seed)
    k.update({
        "Phi_Bc_lo": 0.0, "Phi_Bc_hi": 0.0,
        "voltage_sweep": 1, "Phi_Bc_inc": v_step, "Phi_Bc_hi_max": v_max,
        "num_Vapp_max": int(round(v_max / v_step)),
        "fx.sweep_mode": "fixed", "fx.steps_per_voltage": steps_per_voltage,
        "SC_lo": [-lx / 2, -lx / 2, 0.0], "SC_hi": [lx / 2, lx / 2, 30.0e-9],
        "Channel_lo": [-lx / 2, -lx / 2, 0.0], "Channel_hi": [lx / 2, lx / 2, 30.0e-9],
        "DE_lo": [-lx / 2, -lx / 2, 30.0e-9], "DE_hi": [lx / 2, lx / 2, 31.0e-9],
        "FE_lo": [-lx / 2, -lx / 2, 31.0e-9], "FE_hi": [lx / 2, lx / 2, 36.0e-9],
        "epsilonX_fe": 24.0, "epsilon_de": 3.9,
        "BigGamma": 20.0, "g11": 1.0e-10, "g44": 1.0e-10,
        "acceptor_doping": 1.0e24, "donor_doping": 0.0, "use_Fermi_Dirac": 0,
    })
    k.update(_MAT)
    if extra:
        k.update(extra)
    return render(k)


def hysteresis(nx=128, ny=128, nz=48, dxy=0.5e-9, v_amp=3.0, steps_per_leg=400, seed=1, extra=None) -> str:
    """MFIM stack under a triangular sweep -v_amp -> +v_amp -> -v_amp, one
    leg per ramp (the voltage schedule itself is driven through the API)."""
    return mfim(nx, ny, nz, dxy, nsteps=2 * steps_per_leg, seed=seed, Phi_Bc_hi=-v_amp, extra=extra)


def _rng(seed: int):
    return np.random.Generator(np.random.PCG64(seed))


def polycrystal(nx=256, ny=256, nz=128, dxy=0.5e-9, ngrains=64, p_fe=0.7, seed=1, nsteps=2000, extra=None):
    """Polycrystalline HZO (4-9 nm) on Al2O3 (0-4 nm).

    Returns (text, grains) where grains = dict(id=uint8 (nz,ny,nx) with 255
    outside the HZO, angles=(ngrains,3) degrees for use_Euler_angles = 0,
    tphase=(ngrains,) 0/1).  Grain seeds are uniform in the HZO slab; cells
    take the nearest seed with periodic distance in x and y.  Rotations are
    uniform on SO(3) (random unit quaternions)."""
    text = mfim(nx, ny, nz, dxy, nsteps=nsteps, seed=seed,
                extra=dict({"Coordinate_Transformation": 1, "use_Euler_angles": 0, "epsilonX_fe_tphase": 40.0},
                           **(extra or {})))
    lx, lz = nx * dxy, 9.0e-9
    g = _rng(seed)
    sx = g.uniform(-lx / 2, lx / 2, ngrains)
    sy = g.uniform(-lx / 2, lx / 2, ngrains)
    sz = g.uniform(4.0e-9, lz, ngrains)
    q = g.normal(size=(ngrains, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, a, b, c = q.T
    R = np.empty((ngrains, 3, 3))
    R[:, 0, 0] = 1 - 2 * (b * b + c * c); R[:, 0, 1] = 2 * (a * b - c * w); R[:, 0, 2] = 2 * (a * c + b * w)
    R[:, 1, 0] = 2 * (a * b + c * w); R[:, 1, 1] = 1 - 2 * (a * a + c * c); R[:, 1, 2] = 2 * (b * c - a * w)
    R[:, 2, 0] = 2 * (a * c - b * w); R[:, 2, 1] = 2 * (b * c + a * w); R[:, 2, 2] = 1 - 2 * (a * a + b * b)
    # use_Euler_angles = 0 form (ElectrostaticSolver.cpp:54-62): R31 = -sin(beta),
    # R32 = sin(alpha) cos(beta), R33 = cos(alpha) cos(beta), R21 = cos(beta) sin(theta)
    beta = np.arcsin(np.clip(-R[:, 2, 0], -1, 1))
    alpha = np.arctan2(R[:, 2, 1], R[:, 2, 2])
    theta = np.arctan2(R[:, 1, 0], R[:, 0, 0])
    angles = np.degrees(np.stack([alpha, beta, theta], axis=1))
    tphase = (g.uniform(size=ngrains) >= p_fe).astype(np.uint8)
    dz = lz / nz
    x = -lx / 2 + (np.arange(nx) + 0.5) * dxy
    y = -lx / 2 + (np.arange(ny) + 0.5) * dxy
    z = (np.arange(nz) + 0.5) * dz
    gid = np.full((nz, ny, nx), 255, dtype=np.uint8)
    ddx = x[None, :] - sx[:, None]
    ddx -= lx * np.round(ddx / lx)
    ddy = y[None, :] - sy[:, None]
    ddy -= lx * np.round(ddy / lx)
    dxy2 = ddx[:, None, :] ** 2 + ddy[:, :, None] ** 2          # (g, ny, nx)
    for kk in range(nz):
        if not (4.0e-9 <= z[kk] <= lz):
            continue
        d2 = dxy2 + ((z[kk] - sz) ** 2)[:, None, None]
        gid[kk] = np.argmin(d2, axis=0).astype(np.uint8)
    return text, dict(id=gid, angles=angles, tphase=tphase)


def grain_fields(grains: dict):
    """Per-cell tphase and angle arrays (the reference's representation)."""
    gid = grains["id"]
    inside = gid != 255
    idx = np.where(inside, gid, 0)
    tph = np.where(inside, grains["tphase"][idx], 0).astype(np.float64)
    ang = [np.where(inside, grains["angles"][idx, d], 0.0) for d in range(3)]
    return tph, ang


GRAIN_MAGIC = b"FXGRAIN1"


def write_grain_file(path: str, grains: dict) -> None:
    """The fx.grain_file format: b"FXGRAIN1", int32 nx, ny, nz, ngrains
    (little-endian), per grain four float64 (Euler angles alpha, beta, theta
    in degrees, t-phase flag 0/1), then nx*ny*nz uint8 grain ids, x fastest
    (255: no grain)."""
    gid = np.ascontiguousarray(grains["id"], dtype=np.uint8)
    nz, ny, nx = gid.shape
    ng = len(grains["tphase"])
    per = np.zeros((ng, 4), dtype="<f8")
    per[:, :3] = grains["angles"]
    per[:, 3] = np.asarray(grains["tphase"], dtype=np.float64)
    with open(path, "wb") as f:
        f.write(GRAIN_MAGIC)
        f.write(np.array([nx, ny, nz, ng], dtype="<i4").tobytes())
        f.write(per.tobytes())
        f.write(gid.tobytes())


def read_grain_file(path: str) -> dict:
    """The grains of a file written by write_grain_file."""
    with open(path, "rb") as f:
        b = f.read()
    if b[:8] != GRAIN_MAGIC:
        raise ValueError(f"{path}: not a grain file")
    nx, ny, nz, ng = (int(v) for v in np.frombuffer(b, dtype="<i4", count=4, offset=8))
    per = np.frombuffer(b, dtype="<f8", count=4 * ng, offset=24).reshape(ng, 4)
    gid = np.frombuffer(b, dtype=np.uint8, count=nx * ny * nz, offset=24 + 32 * ng).reshape(nz, ny, nx)
    if len(b) != 24 + 32 * ng + nx * ny * nz:
        raise ValueError(f"{path}: wrong size")
    return dict(id=gid.copy(), angles=per[:, :3].copy(), tphase=per[:, 3].astype(np.uint8))


def write_P_file(path: str, Pz, Px=None, Py=None) -> None:
    """The fx.initial_P_file format: raw little-endian float64, x fastest;
    Pz alone, or the Px, Py and Pz blocks in that order."""
    with open(path, "wb") as f:
        if Px is not None or Py is not None:
            for a in (Px, Py):
                f.write(np.ascontiguousarray(np.zeros_like(Pz) if a is None else a, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(Pz, dtype="<f8").tobytes())


def read_P_file(path: str, shape) -> tuple:
    """(Px, Py, Pz) from an fx.initial_P_file (Px, Py None when it holds Pz only)."""
    v = np.fromfile(path, dtype="<f8")
    N = int(np.prod(shape))
    if v.size == N:
        return None, None, v.reshape(shape)
    if v.size == 3 * N:
        return tuple(v[q * N:(q + 1) * N].reshape(shape) for q in range(3))
    raise ValueError(f"{path}: {v.size} values, expected {N} or {3 * N}")


def triangular_sweep(v_amp: float, steps_per_leg: int) -> np.ndarray:
    """Phi_Bc_hi per step: a leg of steps_per_leg steps from -v_amp to
    +v_amp, then one back to -v_amp (2 * steps_per_leg values)."""
    up = np.linspace(-v_amp, v_amp, steps_per_leg, endpoint=False)
    down = np.linspace(v_amp, -v_amp, steps_per_leg, endpoint=False)
    return np.concatenate([up, down])


def target_loop(v: np.ndarray, seed: int = 7, ps: float = 0.02, vc: float = 1.0) -> np.ndarray:
    """Seeded synthetic tanh hysteresis target <Pz>(V) on the sweep."""
    g = _rng(seed)
    vc = vc * (1.0 + 0.1 * g.uniform(-1, 1))
    w = 0.4 * (1.0 + 0.1 * g.uniform(-1, 1))
    rising = np.concatenate([[True], np.diff(v) > 0])
    return ps * np.tanh((v - np.where(rising, vc, -vc)) / w)


__all__ = ["mfim", "mfism", "polycrystal", "hysteresis", "grain_fields", "triangular_sweep", "target_loop", "render"]
