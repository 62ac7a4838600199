"""Python access to the CPU oracle (oracle/henon_oracle.c) and to the
reference build (oracle/_ref/).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the library.

The C restatement follows the reference's arithmetic line by line (each C
function cites the reference file:line).  It is pinned two ways:
  * against golden values recorded in the reference's own notebooks
    (tests/golden/notebook_values.json), and
  * bit for bit against the reference itself, built from its sources by
    oracle/build_ref.sh, on seeded inputs (tests/golden/ref_track_*.npz,
    made by tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import importlib.util
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
SRC = HERE / "henon_oracle.c"
REF_DIR = HERE / "_ref"

_D = ctypes.c_double
_PD = ctypes.POINTER(ctypes.c_double)
_PU32 = ctypes.POINTER(ctypes.c_uint32)


def build(force: bool = False) -> Path:
    """Compiles the C restatement (no FMA contraction, no -march)."""
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < SRC.stat().st_mtime:
        cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-ffp-contract=off",
               "-fno-fast-math", "-fopenmp", str(SRC), "-o", str(LIB_PATH), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.or_sps_modulation.argtypes = [_D, _D, ctypes.c_int32, ctypes.c_int32, _PD]
        L.or_basic_modulation.argtypes = [_D, _D, _D, ctypes.c_int32, ctypes.c_int32, _PD]
        L.or_tables.argtypes = [_PD, ctypes.c_size_t, _PD, _PD]
        L.or_birkhoff_weights.argtypes = [ctypes.c_uint32, _PD]
        L.or_track.argtypes = [_PD, _PD, _PD, _PD, _PU32, ctypes.c_size_t, _PD, _PD, _PD, _PD,
                               ctypes.c_uint32, _D, _D, ctypes.c_int, ctypes.c_int]
        L.or_max_threads.restype = ctypes.c_int
        L.or_tangent_matrix.argtypes = [_D] * 9 + [_PD]
        L.or_matmul4.argtypes = [_PD, _PD, _PD]
        L.or_philox4x32_10.argtypes = [_PU32, _PU32, _PU32]
        L.or_kick_direction.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, _PD]
        L.or_track_kicked.argtypes = [_PD, _PD, _PD, _PD, _PU32, ctypes.c_size_t, _PD, _PD, _PD,
                                      _PD, ctypes.c_uint32, _D, _D, ctypes.c_int, _D,
                                      ctypes.c_uint64, ctypes.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray, ct=_PD):
    return a.ctypes.data_as(ct)


def max_threads() -> int:
    return int(lib().or_max_threads())


# ---- modulation -------------------------------------------------------------

def sps_modulation(tune: float, epsilon: float, start: int, end: int) -> np.ndarray:
    out = np.empty(end - start, dtype=np.float64)
    lib().or_sps_modulation(tune, epsilon, start, end, _p(out))
    return out


def basic_modulation(tune: float, omega: float, epsilon: float, start: int, end: int) -> np.ndarray:
    out = np.empty(end - start, dtype=np.float64)
    lib().or_basic_modulation(tune, omega, epsilon, start, end, _p(out))
    return out


def omegas(n_turns: int, omega_x: float, omega_y: float, kind: str = "sps",
           omega_0: float = float("nan"), epsilon: float = 0.0, offset: int = 0):
    """pick_a_modulation (src/modulation.cpp:101-134) for the deterministic kinds."""
    if kind == "sps":
        return (sps_modulation(omega_x, epsilon, offset, offset + n_turns),
                sps_modulation(omega_y, epsilon, offset, offset + n_turns))
    if kind == "basic":
        return (basic_modulation(omega_x, omega_0, epsilon, offset, offset + n_turns),
                basic_modulation(omega_y, omega_0, epsilon, offset, offset + n_turns))
    raise ValueError(f"oracle has no deterministic modulation '{kind}'")


def tables(n_turns: int, omega_x: float, omega_y: float, kind: str = "sps",
           omega_0: float = float("nan"), epsilon: float = 0.0, offset: int = 0):
    """(sin wx, cos wx, sin wy, cos wy) with libm, as henon.cu:2679-2682."""
    wx, wy = omegas(n_turns, omega_x, omega_y, kind, omega_0, epsilon, offset)
    out = [np.empty(n_turns) for _ in range(4)]
    lib().or_tables(_p(wx), n_turns, _p(out[0]), _p(out[1]))
    lib().or_tables(_p(wy), n_turns, _p(out[2]), _p(out[3]))
    return tuple(out)


def birkhoff_weights(n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    lib().or_birkhoff_weights(n, _p(out))
    return out


# ---- tracking -----------------------------------------------------------------

def track(x, px, y, py, steps, tabs, n_turns: int, mu: float, barrier: float,
          inverse: bool = False, n_threads: int = 0):
    """henon_tracker::track (src/henon.cu:2701-2752) on copies of the inputs.

    Returns (x, px, y, py, steps) after n_turns turns."""
    x = np.array(x, dtype=np.float64, copy=True)
    px = np.array(px, dtype=np.float64, copy=True)
    y = np.array(y, dtype=np.float64, copy=True)
    py = np.array(py, dtype=np.float64, copy=True)
    steps = np.array(steps, dtype=np.uint32, copy=True)
    sx, cx, sy, cy = (np.ascontiguousarray(t, dtype=np.float64) for t in tabs)
    lib().or_track(_p(x), _p(px), _p(y), _p(py), _p(steps, _PU32), x.size,
                   _p(sx), _p(cx), _p(sy), _p(cy), n_turns, mu, barrier,
                   int(bool(inverse)), int(n_threads))
    return x, px, y, py, steps


# ---- reproducible random kicks -------------------------------------------------------

def philox4x32_10(ctr, key) -> np.ndarray:
    """One Philox4x32-10 block (Salmon et al., SC'11) of a 4-word counter and
    a 2-word key."""
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    lib().or_philox4x32_10(_p(c, _PU32), _p(k, _PU32), _p(out, _PU32))
    return out


def kick_direction(seed: int, idx: int, turn: int) -> np.ndarray:
    """Unit 4-vector of the kick of particle idx at table index turn."""
    out = np.empty(4)
    lib().or_kick_direction(int(seed), int(idx), int(turn), _p(out))
    return out


def track_kicked(x, px, y, py, steps, tabs, n_turns: int, mu: float, barrier: float,
                 kick_module: float, seed: int, inverse: bool = False, n_threads: int = 0):
    """track with a kick of module kick_module per turn along the direction
    of (seed, particle index, table index); returns (x, px, y, py, steps)."""
    x = np.array(x, dtype=np.float64, copy=True)
    px = np.array(px, dtype=np.float64, copy=True)
    y = np.array(y, dtype=np.float64, copy=True)
    py = np.array(py, dtype=np.float64, copy=True)
    steps = np.array(steps, dtype=np.uint32, copy=True)
    sx, cx, sy, cy = (np.ascontiguousarray(t, dtype=np.float64) for t in tabs)
    lib().or_track_kicked(_p(x), _p(px), _p(y), _p(py), _p(steps, _PU32), x.size,
                          _p(sx), _p(cx), _p(sy), _p(cy), n_turns, mu, barrier,
                          int(bool(inverse)), kick_module, int(seed), int(n_threads))
    return x, px, y, py, steps


def tangent_matrix(x, px, y, py, sx, cx, sy, cy, mu) -> np.ndarray:
    out = np.empty(16)
    lib().or_tangent_matrix(x, px, y, py, sx, cx, sy, cy, mu, _p(out))
    return out.reshape(4, 4)


def matmul4(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty(16)
    lib().or_matmul4(_p(a), _p(b), _p(out))
    return out.reshape(4, 4)


# ---- the reference build ------------------------------------------------------

def reference_module(variant: str = "fmad_off"):
    """Imports oracle/_ref/<variant>/henon_map_engine (the unmodified
    reference, built by oracle/build_ref.sh), or returns None when absent."""
    d = REF_DIR / variant
    cands = sorted(d.glob("henon_map_engine*.so")) if d.exists() else []
    if not cands:
        return None
    name = f"_hm_reference_{variant}"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location("henon_map_engine", cands[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules[name] = mod
    return mod


_CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import oracle as O
d = np.load(sys.argv[3])
R = O.reference_module(sys.argv[2])
kind, cls_t, cls_p = (("gpu", R.henon_tracker_gpu, R.particles_4d_gpu) if int(d["gpu"])
                      else ("cpu", R.henon_tracker, R.particles_4d))
t = cls_t(int(d["n_turns"]), float(d["tunes"][0]), float(d["tunes"][1]), "sps", float("nan"),
          float(d["epsilon"]), 0)
p = cls_p(d["x"], d["px"], d["y"], d["py"])
t.track(p, int(d["n_turns"]), float(d["mu"]), float(d["barrier"]))
if int(d["n_back"]):
    t.track(p, int(d["n_back"]), float(d["mu"]), float(d["barrier"]), float("nan"), True)
np.savez(sys.argv[4], x=np.asarray(p.get_x()), px=np.asarray(p.get_px()),
         y=np.asarray(p.get_y()), py=np.asarray(p.get_py()), steps=np.asarray(p.get_steps()))
"""


def reference_track_subprocess(variant: str, x, px, y, py, n_turns: int, tunes, epsilon: float,
                               mu: float, barrier: float = 10.0, gpu: bool = True,
                               n_back: int = 0):
    """Tracks with the reference build `variant` in a child interpreter:
    n_turns forward, then n_back backward (track(..., inverse=True)).

    Two builds of the reference share one pybind11 module name, so only one
    of them can live in a process; the child keeps them apart.  Returns
    (x, px, y, py, steps) or None when the build is absent."""
    import tempfile

    if not (REF_DIR / variant).exists():
        return None
    with tempfile.TemporaryDirectory() as tmp:
        inp, out = Path(tmp) / "in.npz", Path(tmp) / "out.npz"
        np.savez(inp, x=np.asarray(x, float), px=np.asarray(px, float), y=np.asarray(y, float),
                 py=np.asarray(py, float), n_turns=n_turns, tunes=np.asarray(tunes, float),
                 epsilon=epsilon, mu=mu, barrier=barrier, gpu=int(gpu), n_back=int(n_back))
        subprocess.run([sys.executable, "-c", _CHILD, str(HERE.parent), variant, str(inp),
                        str(out)], check=True)
        d = np.load(out)
        return d["x"], d["px"], d["y"], d["py"], d["steps"].astype(np.uint32)


def build_reference(ref: str | os.PathLike | None = None) -> bool:
    """Runs oracle/build_ref.sh on the reference checkout `ref` (default: the
    REF environment variable) when its sources are present."""
    ref = ref if ref is not None else os.environ.get("REF")
    if not ref or not Path(ref, "src").exists():
        return False
    subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True,
                   env={**os.environ, "REF": str(ref)})
    return True
