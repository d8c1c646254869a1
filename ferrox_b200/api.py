"""ctypes binding of libferrox_b200.so (include/ferrox_b200.h).

``FerroX`` mirrors the reference's hot-path functions (Source/Solver/*.H) on
one simulation context.  There is no Python or CPU compute path: every method
calls the native library, which runs the step on the GPU; a missing library or
device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libferrox_b200.so")

FIELDS = ["Px", "Py", "Pz", "Phi", "PoissonRHS", "Ex", "Ey", "Ez", "holes", "electrons", "charge",
          "epsilon", "mask", "tphase", "alpha", "beta", "theta", "PhiDiff", "alpha_cc", "Gamma"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}

STATUS = {0: "FX_OK", -1: "FX_ERR_INVALID_ARGUMENT", -2: "FX_ERR_INPUTS", -3: "FX_ERR_UNSUPPORTED",
          -4: "FX_ERR_CUDA", -5: "FX_ERR_NO_CONVERGENCE", -6: "FX_ERR_NONFINITE", -7: "FX_ERR_OUT_OF_MEMORY",
          -8: "FX_ERR_IO"}

# every entry point declared in include/ferrox_b200.h
EXPORTS = ["fx_version", "fx_create", "fx_create_error", "fx_destroy", "fx_last_error", "fx_get_dims",
           "fx_get_param", "fx_set_param", "fx_set_initial_P", "fx_set_grains", "fx_set_grain_alpha",
           "fx_set_precision", "fx_get_field", "fx_set_field", "fx_compute_poisson_rhs", "fx_compute_rho",
           "fx_compute_phi_rho", "fx_compute_E", "fx_tdgl_euler", "fx_set_phi_bc", "fx_check_steady_state",
           "fx_step", "fx_run", "fx_write_plotfile", "fx_get_stats", "fx_mean_P", "fx_sync", "fx_set_stream",
           "fx_get_kernel_times", "fx_reset_kernel_times", "fx_mean_P_noalloc", "fx_forward_record",
           "fx_backward", "fx_get_grad_P0"]

# gradient slots of fx_backward (enum fx_grad); per-grain alphas follow
GRADS = ["alpha", "beta", "gamma", "g11", "g44", "v_amp"]


class LossSpec(C.Structure):
    _fields_ = [("nsteps", C.c_int), ("checkpoint_every", C.c_int), ("v_amp", C.c_double),
                ("v_shape", C.POINTER(C.c_double)), ("target", C.POINTER(C.c_double))]

KERNEL_CLASSES = ["tdgl", "rhs_p", "newton", "rho", "steady", "smooth_l0", "restrict_l0", "prolong_l0",
                  "mg_coarse", "resid64", "efield", "mg_l1", "mg_l2", "coarse_cta"]


class FxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [("step", C.c_int), ("finished", C.c_int), ("newton_iters_last", C.c_int),
                ("mg_cycles_last", C.c_int), ("newton_iters_total", C.c_longlong),
                ("mg_cycles_total", C.c_longlong), ("kernel_launches", C.c_longlong),
                ("mg_resid_last", C.c_double), ("mg_target_last", C.c_double), ("phi_err_last", C.c_double),
                ("steady_err_last", C.c_double), ("Phi_Bc_hi", C.c_double), ("time", C.c_double),
                ("steady_state_step", C.c_int), ("inc_step", C.c_int), ("num_Vapp", C.c_int), ("sign", C.c_int),
                ("device_bytes", C.c_double)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def lib():
    """Load the native library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ferrox_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        vp, dp, ip, cp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_char_p
        L.fx_version.restype = cp
        L.fx_create.argtypes = [cp, C.c_int, C.POINTER(vp)]
        L.fx_create_error.restype = cp
        L.fx_destroy.argtypes = [vp]
        L.fx_last_error.argtypes = [vp]
        L.fx_last_error.restype = cp
        L.fx_get_dims.argtypes = [vp, ip, dp]
        L.fx_get_param.argtypes = [vp, cp, dp]
        L.fx_set_param.argtypes = [vp, cp, C.c_double]
        L.fx_set_initial_P.argtypes = [vp, dp, dp, dp, C.c_size_t]
        L.fx_set_grains.argtypes = [vp, C.POINTER(C.c_uint8), C.c_size_t, dp, C.POINTER(C.c_uint8), C.c_int]
        L.fx_set_grain_alpha.argtypes = [vp, dp, C.c_int]
        L.fx_set_precision.argtypes = [vp, C.c_int]
        L.fx_get_field.argtypes = [vp, C.c_int, dp, C.c_size_t]
        L.fx_set_field.argtypes = [vp, C.c_int, dp, C.c_size_t]
        for n in ["fx_compute_poisson_rhs", "fx_compute_rho", "fx_compute_phi_rho", "fx_compute_E", "fx_tdgl_euler",
                  "fx_set_phi_bc", "fx_sync"]:
            getattr(L, n).argtypes = [vp]
        L.fx_check_steady_state.argtypes = [vp, C.c_int]
        L.fx_step.argtypes = [vp, C.c_int, ip]
        L.fx_run.argtypes = [vp, ip]
        L.fx_write_plotfile.argtypes = [vp, C.c_int, cp]
        L.fx_get_stats.argtypes = [vp, C.POINTER(Stats)]
        L.fx_set_stream.argtypes = [vp, vp]
        L.fx_mean_P.argtypes = [vp, dp]
        L.fx_mean_P_noalloc.argtypes = [vp, vp, vp, vp, C.c_size_t, vp, vp]
        L.fx_get_kernel_times.argtypes = [vp, dp, C.POINTER(C.c_longlong), C.c_int]
        L.fx_reset_kernel_times.argtypes = [vp]
        L.fx_forward_record.argtypes = [vp, C.POINTER(LossSpec), dp]
        L.fx_backward.argtypes = [vp, dp, C.c_int]
        L.fx_get_grad_P0.argtypes = [vp, dp, dp, dp, C.c_size_t]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class FerroX:
    """One FerroX run on the GPU, created from inputs-file text or a path."""

    def __init__(self, inputs: str, is_text: bool = True, precision: str | None = None):
        L = lib()
        h = C.c_void_p()
        rc = L.fx_create(inputs.encode(), int(is_text), C.byref(h))
        if rc != 0:
            raise FxError(rc, L.fx_create_error().decode())
        self.h = h
        n = (C.c_int * 3)()
        dx = (C.c_double * 3)()
        L.fx_get_dims(self.h, n, dx)
        self.n = tuple(n)
        self.dx = tuple(dx)
        self.shape = (self.n[2], self.n[1], self.n[0])
        self.N = self.n[0] * self.n[1] * self.n[2]
        if precision is not None:
            self._check(L.fx_set_precision(self.h, {"fp64": 0, "mixed": 1}[precision]))

    def close(self):
        h = getattr(self, "h", None)
        if h and _lib is not None:
            _lib.fx_destroy(h)
        self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise FxError(rc, lib().fx_last_error(self.h).decode())
        return rc

    # -- parameters and fields -------------------------------------------
    def param(self, key: str) -> float:
        v = C.c_double()
        rc = lib().fx_get_param(self.h, key.encode(), C.byref(v))
        if rc:
            raise KeyError(key)
        return v.value

    def set_param(self, key: str, value: float) -> None:
        self._check(lib().fx_set_param(self.h, key.encode(), float(value)))

    def field(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """The field as a (nz, ny, nx) FP64 array; with `out` (C-contiguous
        float64 of nx*ny*nz values, e.g. a pinned buffer) the library copies
        straight into it."""
        if out is None:
            out = np.empty(self.shape)
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self.N:
            raise ValueError("out must be a C-contiguous float64 array of nx*ny*nz values")
        self._check(lib().fx_get_field(self.h, FIELD_ID[name], _dp(out), self.N))
        return out

    def set_field(self, name: str, value) -> None:
        v = np.ascontiguousarray(np.broadcast_to(value, self.shape), dtype=np.float64)
        self._check(lib().fx_set_field(self.h, FIELD_ID[name], _dp(v), self.N))

    def set_initial_P(self, Px=None, Py=None, Pz=None) -> None:
        conv = [None if a is None else np.ascontiguousarray(np.broadcast_to(a, self.shape), dtype=np.float64)
                for a in (Px, Py, Pz)]
        self._check(lib().fx_set_initial_P(self.h, _dp(conv[0]), _dp(conv[1]), _dp(conv[2]), self.N))

    def set_grains(self, grain_id, angles_deg, tphase) -> None:
        gid = np.ascontiguousarray(grain_id, dtype=np.uint8)
        ang = np.ascontiguousarray(angles_deg, dtype=np.float64)
        tph = np.ascontiguousarray(tphase, dtype=np.uint8)
        self._check(lib().fx_set_grains(self.h, gid.ctypes.data_as(C.POINTER(C.c_uint8)), gid.size, _dp(ang),
                                        tph.ctypes.data_as(C.POINTER(C.c_uint8)), len(tph)))

    def set_grain_alpha(self, alpha) -> None:
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        self._check(lib().fx_set_grain_alpha(self.h, _dp(a), len(a)))

    # -- the reference's functions ----------------------------------------
    def compute_poisson_rhs(self): self._check(lib().fx_compute_poisson_rhs(self.h))
    def compute_rho(self): self._check(lib().fx_compute_rho(self.h))
    def compute_phi_rho(self): self._check(lib().fx_compute_phi_rho(self.h))
    def compute_E(self): self._check(lib().fx_compute_E(self.h))
    def tdgl_euler(self): self._check(lib().fx_tdgl_euler(self.h))
    def set_phi_bc(self): self._check(lib().fx_set_phi_bc(self.h))
    def check_steady_state(self, step: int): self._check(lib().fx_check_steady_state(self.h, step))

    def step(self, nsteps: int = 1) -> int:
        done = C.c_int(0)
        self._check(lib().fx_step(self.h, nsteps, C.byref(done)))
        return done.value

    def run(self) -> int:
        done = C.c_int(0)
        self._check(lib().fx_run(self.h, C.byref(done)))
        return done.value

    def write_plotfile(self, step: int, directory: str) -> str:
        self._check(lib().fx_write_plotfile(self.h, step, directory.encode()))
        return os.path.join(directory, f"plt{step:08d}")

    def stats(self) -> dict:
        s = Stats()
        self._check(lib().fx_get_stats(self.h, C.byref(s)))
        return s.as_dict()

    def sync(self): self._check(lib().fx_sync(self.h))

    def mean_P(self) -> np.ndarray:
        out = np.zeros(3)
        self._check(lib().fx_mean_P(self.h, _dp(out)))
        return out

    def set_stream(self, cuda_stream: int) -> None:
        """Order all device work on the given cudaStream_t (an integer handle)."""
        self._check(lib().fx_set_stream(self.h, C.c_void_p(cuda_stream)))

    def kernel_times(self) -> dict:
        n = len(KERNEL_CLASSES)
        ms = np.zeros(n)
        cnt = (C.c_longlong * n)()
        self._check(lib().fx_get_kernel_times(self.h, _dp(ms), cnt, n))
        return {k: (float(ms[q]), int(cnt[q])) for q, k in enumerate(KERNEL_CLASSES)}

    def reset_kernel_times(self) -> None:
        self._check(lib().fx_reset_kernel_times(self.h))

    def forward_record(self, target, v_amp: float, v_shape=None, checkpoint_every: int = 50) -> float:
        """Run len(target) steps under Phi_Bc_hi = v_amp * v_shape[n], keeping
        checkpoints for backward(); returns L = mean_n (<Pz>^n - target[n])^2."""
        t = np.ascontiguousarray(target, dtype=np.float64)
        shp = None if v_shape is None else np.ascontiguousarray(v_shape, dtype=np.float64)
        if shp is not None and shp.shape != t.shape:
            raise ValueError("v_shape and target need the same length")
        self._keep = (t, shp)
        spec = LossSpec(len(t), int(checkpoint_every), float(v_amp), _dp(shp), _dp(t))
        loss = C.c_double()
        self._check(lib().fx_forward_record(self.h, C.byref(spec), C.byref(loss)))
        return loss.value

    def backward(self, ngrains: int = 0) -> np.ndarray:
        """Gradients of the recorded loss: alpha, beta, gamma, g11, g44, v_amp,
        then the per-grain alphas."""
        g = np.zeros(len(GRADS) + ngrains)
        self._check(lib().fx_backward(self.h, _dp(g), len(g)))
        return g

    def grad_P0(self, components=("Pz",)) -> dict:
        """dL/dP at the state the recorded run started from."""
        out = {c: np.zeros(self.N) for c in components}
        self._check(lib().fx_get_grad_P0(self.h, _dp(out.get("Px")), _dp(out.get("Py")), _dp(out.get("Pz")), self.N))
        return {c: a.reshape(self.shape) for c, a in out.items()}
