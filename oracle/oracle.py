"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg use
this module, as the checker.  The product (ferrox_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build
from . import inputs as _inputs

FIELDS = ["Px", "Py", "Pz", "Phi", "PoissonRHS", "Ex", "Ey", "Ez", "holes", "electrons", "charge",
          "epsilon", "mask", "tphase", "alpha", "beta", "theta", "PhiDiff", "alpha_cc", "Gamma"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}

I3 = C.c_int * 3
D3 = C.c_double * 3


class Params(C.Structure):
    _fields_ = [
        ("n_cell", I3), ("prob_lo", D3), ("prob_hi", D3), ("is_periodic", I3),
        ("prob_type", C.c_int), ("TimeIntegratorOrder", C.c_int), ("nsteps", C.c_int), ("plot_int", C.c_int),
        ("dt", C.c_double),
        ("P_BC_flag_lo", I3), ("P_BC_flag_hi", I3), ("lambda", C.c_double),
        ("epsilon_0", C.c_double), ("epsilonX_fe", C.c_double), ("epsilonX_fe_tphase", C.c_double),
        ("epsilonZ_fe", C.c_double), ("epsilon_de", C.c_double), ("epsilon_si", C.c_double),
        ("alpha", C.c_double), ("beta", C.c_double), ("gamma", C.c_double), ("alpha_12", C.c_double),
        ("alpha_112", C.c_double), ("alpha_123", C.c_double),
        ("BigGamma", C.c_double), ("g11", C.c_double), ("g44", C.c_double), ("g12", C.c_double), ("g44_p", C.c_double),
        ("FE_lo", D3), ("FE_hi", D3), ("DE_lo", D3), ("DE_hi", D3), ("SC_lo", D3), ("SC_hi", D3),
        ("Channel_lo", D3), ("Channel_hi", D3), ("Remnant_P", D3),
        ("acceptor_doping", C.c_double), ("donor_doping", C.c_double),
        ("use_Fermi_Dirac", C.c_int), ("use_work_function", C.c_int), ("metal_work_function", C.c_double),
        ("is_polarization_scalar", C.c_int), ("delta", C.c_double),
        ("voltage_sweep", C.c_int), ("inc_step", C.c_int),
        ("Phi_Bc_lo", C.c_double), ("Phi_Bc_hi", C.c_double), ("Phi_Bc_inc", C.c_double),
        ("Phi_Bc_hi_max", C.c_double), ("phi_tolerance", C.c_double),
        ("num_Vapp_max", C.c_int), ("random_seed", C.c_int),
        ("include_Landau", C.c_int), ("include_Grad", C.c_int), ("include_Elec", C.c_int),
        ("Coordinate_Transformation", C.c_int), ("use_Euler_angles", C.c_int),
        ("mg_rtol", C.c_double), ("phi_ghost_mode", C.c_int), ("sweep_mode", C.c_int),
        ("steps_per_voltage", C.c_int), ("newton_max_iter", C.c_int), ("mg_max_iter", C.c_int),
        ("verbose", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.ofx_create.restype = vp
        L.ofx_create.argtypes = [C.POINTER(Params), dp, dp, dp, dp]
        L.ofx_destroy.argtypes = [vp]
        for name in ["ofx_compute_poisson_rhs", "ofx_compute_rho", "ofx_compute_phi_rho", "ofx_compute_E",
                     "ofx_tdgl_euler", "ofx_set_phi_bc"]:
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = C.c_int
        L.ofx_step.argtypes = [vp, C.c_int]
        L.ofx_run.argtypes = [vp, C.c_int]
        L.ofx_get_field.argtypes = [vp, C.c_int, dp]
        L.ofx_set_field.argtypes = [vp, C.c_int, dp]
        L.ofx_get_mask_ghost.argtypes = [vp, dp]
        L.ofx_get_phi_ghost.argtypes = [vp, dp]
        L.ofx_get_beta_faces.argtypes = [vp, dp, dp, dp]
        L.ofx_poisson_solve.argtypes = [vp, dp, dp, dp, C.c_double, ip, dp]
        L.ofx_poisson_apply.argtypes = [vp, dp, dp, C.c_int, dp]
        L.ofx_set_eb.argtypes = [vp, C.c_int, C.c_double]
        L.ofx_set_eb.restype = C.c_int
        L.ofx_tdgl_terms.argtypes = [vp, dp, dp, dp]
        L.ofx_get_scalar.argtypes = [vp, C.c_char_p]
        L.ofx_get_scalar.restype = C.c_double
        L.ofx_set_scalar.argtypes = [vp, C.c_char_p, C.c_double]
        L.ofx_uniform.argtypes = [C.c_ulonglong, C.c_ulonglong]
        L.ofx_uniform.restype = C.c_double
        L.ofx_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(p: dict) -> Params:
    P = Params()
    for name, typ in Params._fields_:
        v = p[name]
        if isinstance(v, (list, tuple)):
            getattr(P, name)[:] = v
        else:
            setattr(P, name, v)
    return P


class Oracle:
    """One oracle context: the reference's fields for one inputs deck."""

    def __init__(self, params: dict, tphase=None, angles=None, threads: int | None = None):
        self.p = dict(params)
        self.n = tuple(self.p["n_cell"])
        self.shape = (self.n[2], self.n[1], self.n[0])
        L = lib()
        if threads:
            L.ofx_set_threads(threads)
        self._keep = []

        def arr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(np.broadcast_to(a, self.shape), dtype=np.float64)
            self._keep.append(a)
            return a

        ang = angles if angles is not None else (None, None, None)
        self._P = make_params(self.p)
        self.h = L.ofx_create(C.byref(self._P), _dp(arr(tphase)), _dp(arr(ang[0])), _dp(arr(ang[1])), _dp(arr(ang[2])))
        if not self.h:
            raise ValueError("oracle: unsupported or invalid parameters")

    @classmethod
    def from_text(cls, text: str, **kw):
        table = _inputs.parse_table(text)
        p = _inputs.ferrox_params(table)
        tph, a, b, t = _inputs.function_fields(table, p)
        o = cls(p, tph, (a, b, t), **kw)
        eb = _inputs.embedded_boundary(table, p)
        if eb is not None:
            o.set_eb(*eb)
        if "fx.initial_P_file" in table:
            # the initial P file (format: ferrox_b200.decks.write_P_file)
            from ferrox_b200 import decks
            P = decks.read_P_file(table["fx.initial_P_file"][0], o.shape)
            for name, comp in zip(["Px", "Py", "Pz"], P):
                o.set_field(name, np.zeros(o.shape) if comp is None else comp)
        return o

    def set_eb(self, nz_fluid: int, V: float) -> None:
        """Embedded surface on the face below layer nz_fluid (0: none), Dirichlet value V."""
        if lib().ofx_set_eb(self.h, int(nz_fluid), float(V)) != 0:
            raise ValueError("oracle: embedded boundary layer out of range")

    def __del__(self):
        if getattr(self, "h", None):
            lib().ofx_destroy(self.h)
            self.h = None

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self.shape)
        rc = lib().ofx_get_field(self.h, FIELD_ID[name], _dp(out))
        assert rc == 0
        return out

    def set_field(self, name: str, v) -> None:
        v = np.ascontiguousarray(np.broadcast_to(v, self.shape), dtype=np.float64)
        assert lib().ofx_set_field(self.h, FIELD_ID[name], _dp(v)) == 0

    def mask_ghost(self) -> np.ndarray:
        out = np.empty((self.n[2] + 2, self.n[1] + 2, self.n[0] + 2))
        lib().ofx_get_mask_ghost(self.h, _dp(out))
        return out

    def phi_ghost(self) -> np.ndarray:
        out = np.empty((self.n[2] + 2, self.n[1] + 2, self.n[0] + 2))
        lib().ofx_get_phi_ghost(self.h, _dp(out))
        return out

    def beta_faces(self):
        nx, ny, nz = self.n
        bx = np.empty((nz, ny, nx + 1)); by = np.empty((nz, ny + 1, nx)); bz = np.empty((nz + 1, ny, nx))
        lib().ofx_get_beta_faces(self.h, _dp(bx), _dp(by), _dp(bz))
        return bx, by, bz

    def _call(self, name: str) -> int:
        rc = getattr(lib(), name)(self.h)
        if rc < 0:
            raise RuntimeError(f"oracle {name} failed ({rc})")
        return rc

    def compute_poisson_rhs(self): self._call("ofx_compute_poisson_rhs")
    def compute_rho(self): self._call("ofx_compute_rho")
    def compute_phi_rho(self): self._call("ofx_compute_phi_rho")
    def compute_E(self): self._call("ofx_compute_E")
    def tdgl_euler(self): self._call("ofx_tdgl_euler")
    def set_phi_bc(self): self._call("ofx_set_phi_bc")

    def step(self, step: int) -> int:
        rc = lib().ofx_step(self.h, step)
        if rc < 0:
            raise RuntimeError(f"oracle step failed ({rc})")
        return rc

    def run(self, nsteps: int) -> int:
        rc = lib().ofx_run(self.h, nsteps)
        if rc < 0:
            raise RuntimeError(f"oracle run failed ({rc})")
        return rc

    def tdgl_terms(self):
        N = int(np.prod(self.shape))
        L = np.empty((3,) + self.shape); G = np.empty_like(L); E = np.empty_like(L)
        lib().ofx_tdgl_terms(self.h, _dp(L), _dp(G), _dp(E))
        return L, G, E

    def poisson_solve(self, rhs, alpha_cc=None, phi0=None, rtol=1e-12):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        a = None if alpha_cc is None else np.ascontiguousarray(alpha_cc, dtype=np.float64)
        phi = np.zeros(self.shape) if phi0 is None else np.array(phi0, dtype=np.float64)
        it = C.c_int(0); res = C.c_double(0)
        rc = lib().ofx_poisson_solve(self.h, _dp(rhs), _dp(a), _dp(phi), rtol, C.byref(it), C.byref(res))
        if rc != 0:
            raise RuntimeError(f"oracle poisson solve did not converge ({rc}, {it.value} its, {res.value})")
        return phi, it.value, res.value

    def poisson_apply(self, phi, alpha_cc=None, inhomogeneous=True):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        a = None if alpha_cc is None else np.ascontiguousarray(alpha_cc, dtype=np.float64)
        out = np.empty(self.shape)
        lib().ofx_poisson_apply(self.h, _dp(a), _dp(phi), int(inhomogeneous), _dp(out))
        return out

    def scalar(self, name: str) -> float:
        return lib().ofx_get_scalar(self.h, name.encode())

    def set_scalar(self, name: str, v: float) -> None:
        assert lib().ofx_set_scalar(self.h, name.encode(), float(v)) == 0


def uniform(seed: int, n: int) -> float:
    return lib().ofx_uniform(seed, n)
