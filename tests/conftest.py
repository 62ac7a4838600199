"""Shared pytest setup: the `gpu` marker, import paths and input builders.

Tests marked `gpu` need a CUDA device and the built library; the rest run on
CPU only (oracle pinning, host numerics, the C ABI's exports, the host-side
sharding logic).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

TUNES = (0.168, 0.201)
NAN = float("nan")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def grid(extent: float, side: int, px0: float = 0.0, py0: float = 0.0):
    """side x side grid of (x0, y0) in [0, extent]^2 with constant momenta."""
    v = np.linspace(0.0, extent, side)
    xx, yy = np.meshgrid(v, v)
    x = xx.ravel()
    y = yy.ravel()
    return x, np.full_like(x, px0), y, np.full_like(y, py0)


def bits(a: np.ndarray) -> np.ndarray:
    """Bit patterns of a float64 array with every NaN mapped to one pattern."""
    a = np.asarray(a, dtype=np.float64).copy()
    a[np.isnan(a)] = np.nan
    return a.view(np.uint64)


def assert_bitwise(actual, expected, what=""):
    a = bits(actual)
    e = bits(expected)
    bad = np.flatnonzero(a != e)
    assert bad.size == 0, (f"{what}: {bad.size} of {a.size} differ, first at {bad[:5]}: "
                           f"{np.asarray(actual).ravel()[bad[:5]]} vs {np.asarray(expected).ravel()[bad[:5]]}")


def golden_json(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


def golden_npz(name: str):
    return np.load(GOLDEN / name)


def cuda_available() -> bool:
    try:
        from henon_map_cpp_b200 import _capi
        return _capi.load().hm_device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Skips nothing: a gpu-marked test on a machine without a device fails
    loudly, so a silent CPU fallback can never pass."""
    from henon_map_cpp_b200 import _capi
    lib = _capi.load()
    assert lib.hm_device_count() > 0, "no CUDA device visible to libhenon_b200"
    return lib


def edge_barriers(x, px, y, py, n_turns, eps, mu, n_particles=4, spread=3):
    """Barriers whose square lies within a few representable doubles of the
    largest radius (x*x + px*px) + (y*y + py*py) some particles reach in
    n_turns turns: their loss turn hangs on the last bit of that separately
    rounded sum.  Returns (barriers, index of the particle each targets,
    largest radius of every particle)."""
    from oracle import oracle as O

    tabs = O.tables(n_turns, *TUNES, "sps", epsilon=eps)
    st = (x, px, y, py, np.zeros(x.size, np.uint32))
    rmax = np.zeros(x.size)
    with np.errstate(all="ignore"):
        for _ in range(n_turns):
            st = O.track(*st, tabs, 1, mu, 1e200)
            r = (st[0] * st[0] + st[1] * st[1]) + (st[2] * st[2] + st[3] * st[3])
            rmax = np.fmax(rmax, r)
    ok = np.flatnonzero(np.isfinite(rmax) & (rmax > 0.05) & (rmax < 50.0))
    picks = ok[np.linspace(0, ok.size - 1, n_particles).astype(int)]
    out, who = [], []
    for i in picks:
        b = np.sqrt(rmax[i])
        for d in range(-spread, spread + 1):
            out.append(float(b + d * np.spacing(b)))
            who.append(int(i))
    return out, who, rmax
