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
    autotune.apply()            # cached result, or tune now (~10-30 s)
"""
from __future__ import annotations

import itertools
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


def _calibration(side: int = 512, turns: int = 20_000):
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


def tune_batch(sets, coords, arith: int = C.ARITH_EXACT, budget_s: float = 30.0):
    """Grid search over BATCH_SPACE for one batch (wall time of a replay)."""
    b = C.Batch(sets)
    b.load(*coords)
    res = {}
    start = time.perf_counter()
    groups = None
    for g, share, k, c0, cm in itertools.product(*BATCH_SPACE.values()):
        if cm < c0 or time.perf_counter() - start > budget_s:
            continue
        if g != groups:
            b.set_groups(g)
            groups = g
        b.set_grid_share(share)
        b.configure(arith, k, c0, cm)
        b.run(True)
        t0 = time.perf_counter()
        b.run(True)
        res[(g, share, k, c0, cm)] = time.perf_counter() - t0
    best = min(res, key=res.get)
    return dict(zip(BATCH_SPACE, best)), res[best], {str(k): v for k, v in res.items()}


def _load() -> dict:
    try:
        return json.loads(CACHE.read_text())
    except (OSError, ValueError):
        return {}


def apply(arith: int = C.ARITH_EXACT, retune: bool = False, budget_s: float = 30.0) -> dict:
    """Sets the tracker's launch shape from the cache (tuning first when the
    GPU model/arithmetic has no entry or retune is set); returns it."""
    key = f"{_device_name()}|{'fast' if arith == C.ARITH_FAST else 'exact'}"
    cache = _load()
    if retune or key not in cache:
        shape, ms, timings = tune_track(arith, budget_s)
        cache[key] = {"track": shape, "track_ms": ms, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
        try:
            CACHE.write_text(json.dumps(cache, indent=1) + "\n")
        except OSError:
            pass
    shape = cache[key]["track"]
    _set_shape(shape)
    return shape
