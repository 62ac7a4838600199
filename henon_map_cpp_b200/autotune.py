"""Autotuner for the launch shape of the tracking kernels.

Results never depend on the launch shape (the tests check this bit for bit),
so the tuner only measures: it times candidate (threads per block,
particles per thread, first chunk, chunk cap, turn records per staged
copy) shapes of the chunked tracker, and (groups, particles per thread,
chunk schedule) of the batched path, on
a calibration workload with CUDA events, and keeps the fastest.  Results
are cached per GPU model and arithmetic in a JSON file next to this module
(HENON_B200_TUNING overrides the path).

    from henon_map_cpp_b200 import autotune
    autotune.apply()            # tracker shape: cached result, or tune now (~10-30 s)
    autotune.configure_batch(batch, autotune.batch_shape(), arith)   # batched path
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

from . import _capi as C

CACHE = Path(os.environ.get("HENON_B200_TUNING", Path(__file__).with_name("tuning.json")))

TRACK_SPACE = {"threads": (64, 128, 256), "per_thread": (1, 2, 4), "chunk0": (256, 512, 1024),
               "chunk_max": (8192, 16384, 32768), "stage_turns": (0, 64, 256, 512)}


def _set_shape(shape) -> None:
    C.set_track_config(shape["threads"], shape["per_thread"], shape["chunk0"], shape["chunk_max"])
    C.set_track_staging(shape.get("stage_turns", C.get_track_staging()))


def _current_shape() -> dict:
    shape = dict(zip(("threads", "per_thread", "chunk0", "chunk_max"), C.get_track_config()))
    shape["stage_turns"] = C.get_track_staging()
    return shape
BATCH_SPACE = {"groups": (16, 8, 4, 1), "grid_share": (1.5, 1.0, 2.0, 0.0),
               "per_thread": (1, 2, 4), "chunk0": (256, 512, 1024),
               "chunk_max": (4096, 8192, 16384)}


def _device_name() -> str:
    import torch

    return torch.cuda.get_device_name()


def _calibration(side: int = 1024, turns: int = 20_000):
    """The dynamic-aperture scan's grid (1024^2 on [0, 0.6]^2) over a shorter
    horizon: the shapes are ranked on the workload they will run."""
    v = np.linspace(0.0, 0.6, side)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    return x, np.zeros_like(x), y, np.zeros_like(y), turns


def time_track_shape(shape, arith: int, data, repeats: int = 2) -> float:
    """Summed device time (ms) of the tracking kernels for one shape."""
    import torch

    x, px, y, py, turns = data
    _set_shape(shape)
    tr = C.Tracker(turns, 0.168, 0.201, "sps", float("nan"), 16.0, 0)
    tr.arith = arith
    n = x.size
    dev0 = [torch.from_numpy(a).cuda() for a in (x, px, y, py)]
    work = [torch.empty_like(d) for d in dev0]
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    ws = torch.empty(C.load().hm_track_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    best = float("inf")
    for _ in range(repeats):
        for w, d in zip(work, dev0):
            w.copy_(d)
        st.zero_()
        torch.cuda.synchronize()
        C.set_profiling(True)
        C.call("hm_track_device", *[w.data_ptr() for w in work], st.data_ptr(), n,
               tr.device_tables(), turns, 0, turns, 0.2, 10.0, 0, arith, ws.data_ptr(),
               torch.cuda.current_stream().cuda_stream)
        ms, _ = C.get_profile()
        C.set_profiling(False)
        best = min(best, ms)
    return best


def tune_track(arith: int = C.ARITH_EXACT, budget_s: float = 30.0, data=None):
    """Coordinate search over TRACK_SPACE from the default shape; returns
    (best shape, its time in ms, every timing)."""
    data = data or _calibration()
    cur = _current_shape()
    timings = {}

    def cost(shape):
        key = tuple(shape[k] for k in TRACK_SPACE)
        if key not in timings:
            timings[key] = time_track_shape(shape, arith, data)
        return timings[key]

    start = time.perf_counter()
    best = cost(cur)
    improved = True
    while improved and time.perf_counter() - start < budget_s:
        improved = False
        for name, values in TRACK_SPACE.items():
            for v in values:
                if time.perf_counter() - start > budget_s:
                    break
                cand = dict(cur, **{name: v})
                c = cost(cand)
                if c < best * 0.995:
                    best, cur, improved = c, cand, True
    _set_shape(cur)
    return cur, best, {str(k): v for k, v in timings.items()}


BATCH_DEFAULT = {"groups": 16, "grid_share": 1.5, "per_thread": 1, "chunk0": 512,
                 "chunk_max": 4096}


def configure_batch(b, shape, arith: int) -> None:
    """Applies a BATCH_SPACE shape to a C.Batch."""
    b.set_groups(int(shape["groups"]))
    b.set_grid_share(float(shape["grid_share"]))
    b.configure(arith, int(shape["per_thread"]), int(shape["chunk0"]), int(shape["chunk_max"]))


def tune_batch(sets, coords, arith: int = C.ARITH_EXACT, budget_s: float = 30.0):
    """Coordinate search over BATCH_SPACE from BATCH_DEFAULT for one batch
    (wall time of a graph replay, best of two); returns (best shape, its
    time in s, every timing)."""
    b = C.Batch(sets)
    b.load(*coords)
    res = {}
    start = time.perf_counter()

    def cost(shape):
        key = tuple(shape[k] for k in BATCH_SPACE)
        if key not in res:
            configure_batch(b, shape, arith)
            b.run(True)  # capture + warm-up
            best = float("inf")
            for _ in range(2):
                t0 = time.perf_counter()
                b.run(True)
                best = min(best, time.perf_counter() - t0)
            res[key] = best
        return res[key]

    cur = dict(BATCH_DEFAULT)
    best = cost(cur)
    improved = True
    while improved and time.perf_counter() - start < budget_s:
        improved = False
        for name, values in BATCH_SPACE.items():
            for v in values:
                if time.perf_counter() - start > budget_s:
                    break
                cand = dict(cur, **{name: v})
                if cand["chunk_max"] < cand["chunk0"]:
                    continue
                c = cost(cand)
                if c < best * 0.99:
                    best, cur, improved = c, cand, True
    return cur, best, {str(k): v for k, v in res.items()}


def _load() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def _key(arith: int) -> str:
    return f"{_device_name()}|{'fast' if arith == C.ARITH_FAST else 'exact'}"


def _store(key: str, entry: dict) -> None:
    cache = _load()
    cache.setdefault(key, {}).update(entry)
    try:
        CACHE.write_text(json.dumps(cache, indent=1, sort_keys=True) + "\n")
    except OSError:
        pass


def batch_shape(sets=None, coords=None, arith: int = C.ARITH_EXACT, retune: bool = False,
                budget_s: float = 60.0) -> dict:
    """The batched path's shape for this GPU model and arithmetic from the
    cache; tuned first (on `sets`/`coords`, default the mixed-size sweep of
    sweep.heterogeneous_sets) when absent or when retune is set."""
    key = _key(arith)
    entry = _load().get(key, {})
    if retune or "batch" not in entry:
        if sets is None:
            from .sweep import heterogeneous_sets  # noqa: PLC0415

            sets, coords = heterogeneous_sets()
        shape, secs, _ = tune_batch(sets, coords, arith, budget_s)
        _store(key, {"batch": shape, "batch_s": secs,
                     "batch_when": time.strftime("%Y-%m-%dT%H:%M:%S")})
        return shape
    return entry["batch"]


def apply(arith: int = C.ARITH_EXACT, retune: bool = False, budget_s: float = 30.0) -> dict:
    """Sets the tracker's launch shape from the cache (tuning first when the
    GPU model/arithmetic has no entry or retune is set); returns it."""
    key = _key(arith)
    entry = _load().get(key, {})
    if retune or "track" not in entry:
        shape, ms, _ = tune_track(arith, budget_s)
        _store(key, {"track": shape, "track_ms": ms,
                     "when": time.strftime("%Y-%m-%dT%H:%M:%S")})
        return shape
    shape = entry["track"]
    _set_shape(shape)
    return shape
