"""ctypes binding of the C ABI in include/henon_b200.h (libhenon_b200.so).

This is the thinnest host layer: every call maps 1:1 to an `hm_*` entry
point and a non-OK status raises the matching Python exception with the
library's message.  The library is loaded from this package's directory and
nowhere else; a missing library raises at import time of the caller.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_size_t, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libhenon_b200.so"

HM_OK = 0
HM_ERR_INVALID_ARG = 1
HM_ERR_BUDGET = 2
HM_ERR_CUDA = 3
HM_ERR_TIMEOUT = 4
HM_ERR_CANCELLED = 5
HM_ERR_OOM = 6
HM_ERR_UNKNOWN_MODULATION = 7
HM_ERR_NOT_SUPPORTED = 8
HM_ERR_NO_DEVICE = 9

ARITH_EXACT = 0
ARITH_FAST = 1

FIELD_X, FIELD_PX, FIELD_Y, FIELD_PY, FIELD_STEPS, FIELD_VALID, FIELD_GHOST, FIELD_IDX, \
    FIELD_IDX_BASE = range(9)
FIELD_DTYPE = {FIELD_X: np.float64, FIELD_PX: np.float64, FIELD_Y: np.float64,
               FIELD_PY: np.float64, FIELD_STEPS: np.uint32, FIELD_VALID: np.uint8,
               FIELD_GHOST: np.uint8, FIELD_IDX: np.uint64, FIELD_IDX_BASE: np.uint64}

OBS_RADIUS, OBS_ACTION, OBS_ACTION_X, OBS_ACTION_Y, OBS_ANGLE_X, OBS_ANGLE_Y = range(6)


class HMError(RuntimeError):
    """A non-OK hm_status; `.status` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class HMCancelled(HMError):
    """The cancel callback stopped an operation (state left consistent)."""


_PD = POINTER(c_double)
_PU32 = POINTER(c_uint32)

# name -> (restype, argtypes); restype None means hm_status (checked).
_SIGNATURES = {
    "hm_last_error": (c_char_p, []),
    "hm_version": (c_int, []),
    "hm_device_count": (c_int, []),
    "hm_set_cancel_callback": (None, [c_void_p, c_void_p]),
    "hm_set_track_config": (None, [c_int, c_int, c_uint32, c_uint32]),
    "hm_get_track_config": (None, [POINTER(c_int), POINTER(c_int), _PU32, _PU32]),
    "hm_set_track_staging": (None, [c_uint32]),
    "hm_get_track_staging": (None, [_PU32]),
    "hm_modulation": (None, [c_char_p, c_uint32, c_double, c_double, c_double, c_double,
                             c_uint32, _PD, _PD]),
    "hm_sps_modulation": (None, [c_double, c_double, ctypes.c_int32, ctypes.c_int32, _PD]),
    "hm_basic_modulation": (None, [c_double, c_double, c_double, ctypes.c_int32,
                                   ctypes.c_int32, _PD]),
    "hm_birkhoff_weights": (None, [c_uint32, _PD]),
    "hm_tracker_create": (None, [c_uint32, c_double, c_double, c_char_p, c_double, c_double,
                                 c_uint32, POINTER(c_void_p)]),
    "hm_tracker_compute_a_modulation": (None, [c_void_p, c_uint32, c_double, c_double, c_char_p,
                                               c_double, c_double, c_uint32]),
    "hm_tracker_destroy": (None, [c_void_p]),
    "hm_tracker_allowed_steps": (None, [c_void_p, POINTER(c_uint64)]),
    "hm_tracker_get_tables": (None, [c_void_p, _PD, _PD, _PD, _PD]),
    "hm_tracker_device_tables": (None, [c_void_p, POINTER(c_void_p)]),
    "hm_tracker_set_arith": (None, [c_void_p, c_int]),
    "hm_tracker_get_arith": (None, [c_void_p, POINTER(c_int)]),
    "hm_particles_create": (None, [_PD, _PD, _PD, _PD, c_size_t, POINTER(c_void_p)]),
    "hm_particles_destroy": (None, [c_void_p]),
    "hm_particles_reset": (None, [c_void_p]),
    "hm_particles_size": (None, [c_void_p, POINTER(c_size_t), POINTER(c_size_t),
                                 POINTER(c_size_t)]),
    "hm_particles_global_steps": (None, [c_void_p, _PU32]),
    "hm_particles_get": (None, [c_void_p, c_int, c_void_p]),
    "hm_particles_device_ptr": (None, [c_void_p, c_int, POINTER(c_void_p)]),
    "hm_particles_observable": (None, [c_void_p, c_int, _PD]),
    "hm_track": (None, [c_void_p, c_void_p, c_uint32, c_double, c_double, c_double, c_int]),
    "hm_particles_set_kick_seed": (None, [c_void_p, ctypes.c_uint64]),
    "hm_particles_get_kick_seed": (None, [c_void_p, POINTER(ctypes.c_uint64)]),
    "hm_track_workspace_bytes": (c_size_t, [c_size_t]),
    "hm_track_device": (None, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
                               c_void_p, c_uint64, c_uint32, c_uint32, c_double, c_double, c_int,
                               c_int, c_void_p, c_void_p]),
    "hm_track_device_noalloc": (None, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_size_t, c_void_p, c_uint64, c_uint32, c_uint32,
                                       c_double, c_double, c_int, c_int, c_void_p]),
    "hm_fp64_peak": (None, [c_double, _PD, _PD]),
    "hm_release_cached_memory": (None, []),
    "hm_set_profiling": (None, [c_int]),
    "hm_get_profile": (None, [_PD, POINTER(c_uint64)]),
    "hm_get_profile_work": (None, [c_void_p, c_void_p]),
    # tangent map
    "hm_matrices_create": (None, [c_size_t, POINTER(c_void_p)]),
    "hm_matrices_destroy": (None, [c_void_p]),
    "hm_matrices_size": (None, [c_void_p, POINTER(c_size_t)]),
    "hm_matrices_reset": (None, [c_void_p]),
    "hm_matrices_structured_multiply": (None, [c_void_p, c_void_p, c_void_p, c_double]),
    "hm_matrices_set_with_tracker": (None, [c_void_p, c_void_p, c_void_p, c_double]),
    "hm_matrices_copy": (None, [c_void_p, c_void_p]),
    "hm_matrices_get": (None, [c_void_p, _PD]),
    "hm_matrices_get_vector": (None, [c_void_p, _PD, _PD]),
    "hm_vectors_create": (None, [_PD, c_size_t, POINTER(c_void_p)]),
    "hm_vectors_destroy": (None, [c_void_p]),
    "hm_vectors_set": (None, [c_void_p, _PD, c_int]),
    "hm_vectors_multiply": (None, [c_void_p, c_void_p]),
    "hm_vectors_normalize": (None, [c_void_p]),
    "hm_vectors_get": (None, [c_void_p, _PD]),
    # constructs
    "hm_lyapunov_create": (None, [c_size_t, POINTER(c_uint64), c_size_t, POINTER(c_void_p)]),
    "hm_lyapunov_destroy": (None, [c_void_p]),
    "hm_lyapunov_reset": (None, [c_void_p]),
    "hm_lyapunov_change_weights": (None, [c_void_p, c_uint64]),
    "hm_lyapunov_add": (None, [c_void_p, c_void_p]),
    "hm_lyapunov_windows": (None, [c_void_p, POINTER(c_size_t)]),
    "hm_lyapunov_get_weights": (None, [c_void_p, c_size_t, _PD]),
    "hm_lyapunov_get": (None, [c_void_p, c_int, _PD]),
    "hm_megno_create": (None, [c_size_t, POINTER(c_void_p)]),
    "hm_megno_destroy": (None, [c_void_p]),
    "hm_megno_reset": (None, [c_void_p]),
    "hm_megno_add": (None, [c_void_p, c_void_p, c_void_p]),
    "hm_megno_get": (None, [c_void_p, _PD]),
    "hm_megno_birkhoff_create": (None, [c_size_t, POINTER(c_uint64), c_size_t,
                                        POINTER(c_void_p)]),
    "hm_megno_birkhoff_destroy": (None, [c_void_p]),
    "hm_megno_birkhoff_reset": (None, [c_void_p]),
    "hm_megno_birkhoff_add": (None, [c_void_p, c_void_p, c_void_p]),
    "hm_megno_birkhoff_get": (None, [c_void_p, _PD]),
    "hm_tune_birkhoff_create": (None, [c_size_t, POINTER(c_uint64), c_size_t,
                                       POINTER(c_void_p)]),
    "hm_tune_birkhoff_destroy": (None, [c_void_p]),
    "hm_tune_birkhoff_reset": (None, [c_void_p]),
    "hm_tune_birkhoff_first_add": (None, [c_void_p, c_void_p]),
    "hm_tune_birkhoff_add": (None, [c_void_p, c_void_p]),
    "hm_tune_birkhoff_get": (None, [c_void_p, c_int, _PD]),
    "hm_storage_create": (None, [c_size_t, c_size_t, POINTER(c_void_p)]),
    "hm_storage_destroy": (None, [c_void_p]),
    "hm_storage_store": (None, [c_void_p, c_void_p]),
    "hm_storage_reset": (None, [c_void_p]),
    "hm_storage_size": (None, [c_void_p, POINTER(c_size_t), POINTER(c_size_t),
                               POINTER(c_size_t)]),
    "hm_storage_get": (None, [c_void_p, c_int, _PD]),
    "hm_storage_device_ptr": (None, [c_void_p, c_int, POINTER(c_void_p)]),
    "hm_track_indicators": (None, [c_void_p, c_void_p, c_uint32, c_double, c_double, c_void_p]),
    # ghosts and host tangent matrices
    "hm_particles_add_ghost": (None, [c_void_p, c_double, c_char_p]),
    "hm_particles_renormalize": (None, [c_void_p, c_double]),
    "hm_particles_displacement_module": (None, [c_void_p, _PD]),
    "hm_particles_displacement_direction": (None, [c_void_p, _PD]),
    "hm_tracker_tangent_matrices": (None, [c_void_p, c_void_p, c_double, c_int, _PD]),
    "hm_track_ghost_lyapunov": (None, [c_void_p, c_void_p, c_uint32, c_uint32, c_double,
                                       c_double, c_double, _PD]),
    # batched heterogeneous tracking
    "hm_batch_create": (None, [c_size_t, c_void_p, POINTER(c_void_p)]),
    "hm_batch_destroy": (None, [c_void_p]),
    "hm_batch_configure": (None, [c_void_p, c_int, c_int, c_uint32, c_uint32]),
    "hm_batch_set_groups": (None, [c_void_p, c_int]),
    "hm_batch_set_grid_share": (None, [c_void_p, c_double]),
    "hm_batch_size": (None, [c_void_p, POINTER(c_uint64), POINTER(c_uint32)]),
    "hm_batch_load": (None, [c_void_p, _PD, _PD, _PD, _PD]),
    "hm_batch_run": (None, [c_void_p, c_int]),
    "hm_batch_get": (None, [c_void_p, c_int, c_void_p]),
    # tunes
    "hm_orbit_tunes": (None, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_size_t,
                              _PU32, _PU32, c_size_t, c_int, _PD]),
    "hm_tracker_megno": (None, [c_void_p, c_void_p, c_uint32, c_double, c_double, c_double,
                                c_int, POINTER(c_uint64), c_size_t, _PD]),
    "hm_tracker_orbit_tunes": (None, [c_void_p, c_void_p, c_uint32, c_double, c_double,
                                      c_double, c_int, _PU32, _PU32, c_size_t, c_int, _PD, _PD]),
    "hm_storage_tunes": (None, [c_void_p, _PU32, _PU32, c_size_t, c_int, _PD]),
    "hm_set_tune_slice_limit": (None, [c_size_t]),
    "hm_get_tune_slice_limit": (None, [POINTER(c_size_t)]),
    "hm_orbit_tunes_host": (None, [_PD, _PD, _PD, _PD, c_size_t, c_size_t, _PU32, _PU32,
                                   c_size_t, c_int, _PD]),
    # orbit-loss gradients
    "hm_adjoint_workspace_bytes": (c_size_t, [c_size_t, c_uint32, c_uint32]),
    "hm_set_adjoint_config": (None, [c_int]),
    "hm_get_adjoint_config": (None, [POINTER(c_int)]),
    "hm_adjoint": (None, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_double,
                          c_double, c_uint32, c_uint32, c_int, c_void_p, c_void_p, c_void_p,
                          c_void_p, c_void_p, c_void_p, c_void_p]),
}


class BatchSet(ctypes.Structure):
    """hm_batch_set (include/henon_b200.h)."""
    _fields_ = [("omega_x", c_double), ("omega_y", c_double), ("modulation_kind", c_char_p),
                ("omega_0", c_double), ("epsilon", c_double), ("offset", c_uint32),
                ("n_turns", c_uint32), ("n_particles", c_uint64), ("mu", c_double),
                ("barrier", c_double)]


class IndicatorSet(ctypes.Structure):
    """hm_indicator_set (include/henon_b200.h)."""
    _fields_ = [("matrix", c_void_p), ("matrix_old", c_void_p), ("megno", c_void_p),
                ("megno_birkhoff", c_void_p), ("vectors", c_void_p), ("lyapunov", c_void_p),
                ("tune", c_void_p), ("megno_sample_turns", POINTER(c_uint64)),
                ("n_megno_samples", c_size_t), ("megno_samples_out", _PD),
                ("jacobian_of_turn", c_int)]

_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Loads libhenon_b200.so from the package directory (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run `python -m henon_map_cpp_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        if not hasattr(lib, name):
            continue  # declared later in the header than this binding knows
        fn = getattr(lib, name)
        fn.restype = c_int if res is None else res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().hm_last_error().decode()


_EXC = {HM_ERR_INVALID_ARG: ValueError, HM_ERR_NOT_SUPPORTED: NotImplementedError,
        HM_ERR_OOM: MemoryError}


def check(status: int) -> None:
    if status == HM_OK:
        return
    msg = last_error()
    if status == HM_ERR_CANCELLED:
        raise HMCancelled(status, msg)
    base = _EXC.get(status)
    if base is None:
        raise HMError(status, msg)
    err = type(f"HM{base.__name__}", (HMError, base), {})(status, msg)
    raise err


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# ---- handle wrappers (ownership: the wrapper destroys its handle) -----------------

class Tracker:
    """hm_tracker: modulation tables on the device (henon_tracker_gpu)."""

    def __init__(self, n_turns: int, omega_x: float, omega_y: float, kind: str = "sps",
                 omega_0: float = float("nan"), epsilon: float = 0.0, offset: int = 0):
        self.h = c_void_p()
        call("hm_tracker_create", int(n_turns), float(omega_x), float(omega_y), kind.encode(),
             float(omega_0), float(epsilon), int(offset), ctypes.byref(self.h))

    def compute_a_modulation(self, n_turns, omega_x, omega_y, kind="sps",
                             omega_0=float("nan"), epsilon=0.0, offset=0):
        call("hm_tracker_compute_a_modulation", self.h, int(n_turns), float(omega_x),
             float(omega_y), kind.encode(), float(omega_0), float(epsilon), int(offset))

    @property
    def allowed_steps(self) -> int:
        v = c_uint64()
        call("hm_tracker_allowed_steps", self.h, ctypes.byref(v))
        return int(v.value)

    def tables(self):
        n = self.allowed_steps
        out = [np.empty(n) for _ in range(4)]
        call("hm_tracker_get_tables", self.h, *map(dptr, out))
        return tuple(out)

    def device_tables(self) -> int:
        v = c_void_p()
        call("hm_tracker_device_tables", self.h, ctypes.byref(v))
        return int(v.value or 0)

    @property
    def arith(self) -> int:
        v = c_int()
        call("hm_tracker_get_arith", self.h, ctypes.byref(v))
        return int(v.value)

    @arith.setter
    def arith(self, mode: int) -> None:
        call("hm_tracker_set_arith", self.h, int(mode))

    def track(self, particles: "Particles", n_turns: int, mu: float, barrier: float = 100.0,
              kick_module: float = float("nan"), inverse: bool = False) -> None:
        call("hm_track", self.h, particles.h, int(n_turns), float(mu), float(barrier),
             float(kick_module), int(bool(inverse)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib is not None:
            _lib.hm_tracker_destroy(self.h)
            self.h = c_void_p()


class Particles:
    """hm_particles: particle ensemble on the device (particles_4d_gpu)."""

    def __init__(self, x, px, y, py):
        x, px, y, py = (f64(a) for a in (x, px, y, py))
        if not (x.shape == px.shape == y.shape == py.shape) or x.ndim != 1:
            raise ValueError("x, px, y, py must be 1D arrays of the same shape")
        self.h = c_void_p()
        call("hm_particles_create", dptr(x), dptr(px), dptr(y), dptr(py), x.size,
             ctypes.byref(self.h))

    def size(self):
        a, b, c = c_size_t(), c_size_t(), c_size_t()
        call("hm_particles_size", self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return int(a.value), int(b.value), int(c.value)

    @property
    def n_total(self) -> int:
        return self.size()[0]

    @property
    def global_steps(self) -> int:
        v = c_uint32()
        call("hm_particles_global_steps", self.h, ctypes.byref(v))
        return int(v.value)

    @property
    def kick_seed(self) -> int:
        """Key of the reproducible random kicks of track(kick_module=...)."""
        v = ctypes.c_uint64()
        call("hm_particles_get_kick_seed", self.h, ctypes.byref(v))
        return int(v.value)

    @kick_seed.setter
    def kick_seed(self, seed: int) -> None:
        call("hm_particles_set_kick_seed", self.h, ctypes.c_uint64(int(seed)))

    def get(self, field: int) -> np.ndarray:
        out = np.empty(self.n_total, dtype=FIELD_DTYPE[field])
        call("hm_particles_get", self.h, field, out.ctypes.data_as(c_void_p))
        return out

    def device_ptr(self, field: int) -> int:
        v = c_void_p()
        call("hm_particles_device_ptr", self.h, field, ctypes.byref(v))
        return int(v.value or 0)

    def observable(self, kind: int) -> np.ndarray:
        out = np.empty(self.n_total)
        call("hm_particles_observable", self.h, kind, dptr(out))
        return out

    def state(self):
        return (self.get(FIELD_X), self.get(FIELD_PX), self.get(FIELD_Y), self.get(FIELD_PY),
                self.get(FIELD_STEPS))

    def reset(self) -> None:
        call("hm_particles_reset", self.h)

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib is not None:
            _lib.hm_particles_destroy(self.h)
            self.h = c_void_p()


class _Handle:
    """Owns one opaque handle; `_destroy` names its hm_*_destroy."""

    _destroy = ""

    def __init__(self):
        self.h = c_void_p()

    def __del__(self):
        if getattr(self, "h", None) and self.h.value and _lib is not None:
            getattr(_lib, self._destroy)(self.h)
            self.h = c_void_p()


def _u64(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.uint64).ravel())


class Matrices(_Handle):
    """hm_matrices: one 4x4 matrix per particle (matrix_4d_vector_gpu)."""
    _destroy = "hm_matrices_destroy"

    def __init__(self, n: int):
        super().__init__()
        self.n = int(n)
        call("hm_matrices_create", self.n, ctypes.byref(self.h))

    def reset(self):
        call("hm_matrices_reset", self.h)

    def structured_multiply(self, tracker: Tracker, particles: Particles, mu: float):
        call("hm_matrices_structured_multiply", self.h, tracker.h, particles.h, float(mu))

    def set_with_tracker(self, tracker: Tracker, particles: Particles, mu: float):
        call("hm_matrices_set_with_tracker", self.h, tracker.h, particles.h, float(mu))

    def explicit_copy(self, other: "Matrices"):
        call("hm_matrices_copy", self.h, other.h)

    def get(self) -> np.ndarray:
        out = np.empty((self.n, 4, 4))
        call("hm_matrices_get", self.h, dptr(out))
        return out

    def get_vector(self, rv) -> np.ndarray:
        rv = f64(rv).reshape(self.n, 4)
        out = np.empty((self.n, 4))
        call("hm_matrices_get_vector", self.h, dptr(rv), dptr(out))
        return out


class Vectors(_Handle):
    """hm_vectors: one 4-vector per particle (vector_4d_gpu)."""
    _destroy = "hm_vectors_destroy"

    def __init__(self, rv):
        super().__init__()
        rv = f64(rv).reshape(-1, 4)
        self.n = rv.shape[0]
        call("hm_vectors_create", dptr(rv), self.n, ctypes.byref(self.h))

    def set_vectors(self, rv):
        rv = f64(rv)
        if rv.size == 4 and self.n != 1:
            call("hm_vectors_set", self.h, dptr(rv), 1)
        else:
            call("hm_vectors_set", self.h, dptr(rv.reshape(self.n, 4)), 0)

    def multiply(self, m: Matrices):
        call("hm_vectors_multiply", self.h, m.h)

    def normalize(self):
        call("hm_vectors_normalize", self.h)

    def get(self) -> np.ndarray:
        out = np.empty((self.n, 4))
        call("hm_vectors_get", self.h, dptr(out))
        return out


class Lyapunov(_Handle):
    """hm_lyapunov: lyapunov_birkhoff_construct(_multi)."""
    _destroy = "hm_lyapunov_destroy"

    def __init__(self, n: int, n_weights):
        super().__init__()
        self.n = int(n)
        w = _u64(np.atleast_1d(n_weights))
        self.lengths = [int(v) for v in w]
        self.n_windows = w.size
        call("hm_lyapunov_create", self.n, w.ctypes.data_as(POINTER(c_uint64)), w.size,
             ctypes.byref(self.h))

    def reset(self):
        call("hm_lyapunov_reset", self.h)

    def change_weights(self, n_weights: int):
        call("hm_lyapunov_change_weights", self.h, int(n_weights))
        self.lengths = [int(n_weights)]

    def add(self, v: Vectors):
        call("hm_lyapunov_add", self.h, v.h)

    def weights(self, window: int = 0) -> np.ndarray:
        out = np.empty(self.lengths[window])
        call("hm_lyapunov_get_weights", self.h, int(window), dptr(out))
        return out

    def get(self, birkhoff: bool) -> np.ndarray:
        out = np.empty((self.n_windows, self.n))
        call("hm_lyapunov_get", self.h, int(bool(birkhoff)), dptr(out))
        return out


class Megno(_Handle):
    _destroy = "hm_megno_destroy"

    def __init__(self, n: int):
        super().__init__()
        self.n = int(n)
        call("hm_megno_create", self.n, ctypes.byref(self.h))

    def reset(self):
        call("hm_megno_reset", self.h)

    def add(self, a: Matrices, b: Matrices):
        call("hm_megno_add", self.h, a.h, b.h)

    def get(self) -> np.ndarray:
        out = np.empty(self.n)
        call("hm_megno_get", self.h, dptr(out))
        return out


class MegnoBirkhoff(_Handle):
    _destroy = "hm_megno_birkhoff_destroy"

    def __init__(self, n: int, turn_samples):
        super().__init__()
        self.n = int(n)
        t = _u64(turn_samples)
        self.n_samples = t.size
        call("hm_megno_birkhoff_create", self.n, t.ctypes.data_as(POINTER(c_uint64)), t.size,
             ctypes.byref(self.h))

    def reset(self):
        call("hm_megno_birkhoff_reset", self.h)

    def add(self, a: Matrices, b: Matrices):
        call("hm_megno_birkhoff_add", self.h, a.h, b.h)

    def get(self) -> np.ndarray:
        out = np.empty((self.n_samples, self.n))
        call("hm_megno_birkhoff_get", self.h, dptr(out))
        return out


class TuneBirkhoff(_Handle):
    _destroy = "hm_tune_birkhoff_destroy"

    def __init__(self, n: int, turn_samples):
        super().__init__()
        self.n = int(n)
        t = _u64(turn_samples)
        self.n_samples = t.size
        call("hm_tune_birkhoff_create", self.n, t.ctypes.data_as(POINTER(c_uint64)), t.size,
             ctypes.byref(self.h))

    def reset(self):
        call("hm_tune_birkhoff_reset", self.h)

    def first_add(self, p: Particles):
        call("hm_tune_birkhoff_first_add", self.h, p.h)

    def add(self, p: Particles):
        call("hm_tune_birkhoff_add", self.h, p.h)

    def get(self, which: int) -> np.ndarray:
        out = np.empty((self.n_samples, self.n))
        call("hm_tune_birkhoff_get", self.h, int(which), dptr(out))
        return out


class Storage(_Handle):
    _destroy = "hm_storage_destroy"

    def __init__(self, n: int, batch: int):
        super().__init__()
        self.n, self.batch = int(n), int(batch)
        call("hm_storage_create", self.n, self.batch, ctypes.byref(self.h))

    def store(self, p: Particles):
        call("hm_storage_store", self.h, p.h)

    def reset(self):
        call("hm_storage_reset", self.h)

    def get(self, field: int) -> np.ndarray:
        out = np.empty((self.batch, self.n))
        call("hm_storage_get", self.h, int(field), dptr(out))
        return out


def track_indicators(tracker: Tracker, particles: Particles, n_turns: int, mu: float,
                     barrier: float = 100.0, matrix=None, matrix_old=None, megno=None,
                     megno_birkhoff=None, vectors=None, lyapunov=None, tune=None,
                     megno_sample_turns=None, megno_samples_out=None,
                     jacobian_of_turn=False):
    """hm_track_indicators: n_turns of the fused per-turn indicator loop."""
    s = IndicatorSet()
    s.jacobian_of_turn = int(bool(jacobian_of_turn))
    for name, obj in (("matrix", matrix), ("matrix_old", matrix_old), ("megno", megno),
                      ("megno_birkhoff", megno_birkhoff), ("vectors", vectors),
                      ("lyapunov", lyapunov), ("tune", tune)):
        setattr(s, name, obj.h.value if obj is not None else None)
    keep = None
    if megno_sample_turns is not None:
        keep = _u64(megno_sample_turns)
        s.megno_sample_turns = keep.ctypes.data_as(POINTER(c_uint64))
        s.n_megno_samples = keep.size
        if megno_samples_out is not None:
            s.megno_samples_out = dptr(megno_samples_out)
    call("hm_track_indicators", tracker.h, particles.h, int(n_turns), float(mu), float(barrier),
         ctypes.byref(s))
    del keep


class Batch(_Handle):
    """hm_batch: heterogeneous parameter sets tracked together.

    `sets` is a sequence of dicts with keys omega_x, omega_y, epsilon, mu,
    n_turns, n_particles and optionally barrier (10.0), modulation_kind
    ("sps"), omega_0 (nan), offset (0)."""
    _destroy = "hm_batch_destroy"

    def __init__(self, sets):
        super().__init__()
        arr = (BatchSet * len(sets))()
        self._kinds = []
        for k, s in enumerate(sets):
            kind = str(s.get("modulation_kind", "sps")).encode()
            self._kinds.append(kind)
            arr[k] = BatchSet(float(s["omega_x"]), float(s["omega_y"]), kind,
                              float(s.get("omega_0", float("nan"))), float(s["epsilon"]),
                              int(s.get("offset", 0)), int(s["n_turns"]), int(s["n_particles"]),
                              float(s["mu"]), float(s.get("barrier", 10.0)))
        call("hm_batch_create", len(sets), ctypes.cast(arr, c_void_p), ctypes.byref(self.h))
        self.n_total = sum(int(s["n_particles"]) for s in sets)

    def configure(self, arith: int = ARITH_EXACT, per_thread: int = 1, chunk0: int = 512,
                  chunk_max: int = 16384):
        call("hm_batch_configure", self.h, int(arith), int(per_thread), int(chunk0),
             int(chunk_max))

    def set_groups(self, groups: int) -> None:
        """Number of concurrently tracked groups of sets (1..16)."""
        call("hm_batch_set_groups", self.h, int(groups))

    def set_grid_share(self, share: float) -> None:
        """Grid of each group's chunk kernel, as share x the group's fraction of
        the work of the whole device (0: every group spans the device)."""
        call("hm_batch_set_grid_share", self.h, float(share))

    def n_chunks(self) -> int:
        a, b = c_uint64(), c_uint32()
        call("hm_batch_size", self.h, ctypes.byref(a), ctypes.byref(b))
        return int(b.value)

    def load(self, x, px, y, py):
        x, px, y, py = (f64(a) for a in (x, px, y, py))
        if x.size != self.n_total:
            raise ValueError("initial conditions must cover every set's particles")
        call("hm_batch_load", self.h, dptr(x), dptr(px), dptr(y), dptr(py))

    def run(self, use_graph: bool = True):
        call("hm_batch_run", self.h, int(bool(use_graph)))

    def get(self, field: int) -> np.ndarray:
        out = np.empty(self.n_total, dtype=FIELD_DTYPE[field])
        call("hm_batch_get", self.h, int(field), out.ctypes.data_as(c_void_p))
        return out


def _windows(frm, to):
    f = np.ascontiguousarray(np.asarray(frm, dtype=np.uint32).ravel())
    t = np.ascontiguousarray(np.asarray(to, dtype=np.uint32).ravel())
    if f.size != t.size:
        raise ValueError("compute_tune: from and to must be of the same size")
    return f, t


def tracker_orbit_tunes(tracker: Tracker, particles: Particles, n_turns: int, mu: float,
                        barrier: float, frm, to, remove_mean: bool, fft: bool,
                        kick_module: float = float("nan"), inverse: bool = False):
    """hm_tracker_orbit_tunes: (birkhoff [n][2(W+1)], fft or None)."""
    f, t = _windows(frm, to)
    n = particles.n_total
    b = np.empty((n, 2 * (f.size + 1)))
    ff = np.empty_like(b) if fft else None
    call("hm_tracker_orbit_tunes", tracker.h, particles.h, int(n_turns), float(mu),
         float(barrier), float(kick_module), int(bool(inverse)), f.ctypes.data_as(_PU32),
         t.ctypes.data_as(_PU32), f.size, int(bool(remove_mean)), dptr(b),
         dptr(ff) if fft else None)
    return b, ff


def storage_tunes(storage: "Storage", frm, to, method: int) -> np.ndarray:
    f, t = _windows(frm, to)
    out = np.empty((storage.n, 2 * (f.size + 1)))
    call("hm_storage_tunes", storage.h, f.ctypes.data_as(_PU32), t.ctypes.data_as(_PU32), f.size,
         int(method), dptr(out))
    return out


def set_track_config(threads: int, per_thread: int, chunk0: int, chunk_max: int) -> None:
    call("hm_set_track_config", int(threads), int(per_thread), int(chunk0), int(chunk_max))


def get_track_config():
    a, b, c, d = c_int(), c_int(), c_uint32(), c_uint32()
    call("hm_get_track_config", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
         ctypes.byref(d))
    return int(a.value), int(b.value), int(c.value), int(d.value)


def set_track_staging(stage_turns: int) -> None:
    """0: turn records read from global memory; else staged into shared
    memory by bulk copies, stage_turns turns at a time."""
    call("hm_set_track_staging", int(stage_turns))


def get_track_staging() -> int:
    v = c_uint32()
    call("hm_get_track_staging", ctypes.byref(v))
    return int(v.value)


def get_profile_work():
    """(list particles, chunk turns) summed over the timed tracking launches."""
    a, b = c_uint64(), c_uint64()
    call("hm_get_profile_work", ctypes.byref(a), ctypes.byref(b))
    return int(a.value), int(b.value)


def release_cached_memory() -> None:
    """Returns the unused blocks of the library's device memory pools."""
    call("hm_release_cached_memory")


def set_profiling(on: bool) -> None:
    call("hm_set_profiling", int(bool(on)))


def get_profile():
    """(summed kernel ms, launches) of the tracking kernels since profiling began."""
    ms, n = c_double(), c_uint64()
    call("hm_get_profile", ctypes.byref(ms), ctypes.byref(n))
    return float(ms.value), int(n.value)


def fp64_peak(seconds: float = 0.2):
    """(TFLOP/s, ms) of the FP64 FMA-chain microbenchmark on the current device."""
    tf, ms = c_double(), c_double()
    call("hm_fp64_peak", float(seconds), ctypes.byref(tf), ctypes.byref(ms))
    return float(tf.value), float(ms.value)
