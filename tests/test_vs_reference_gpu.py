"""The reference's own GPU tracking path against ours on the same B200.

The reference tracks with one `gpu_henon_track` launch per turn
(henon_tracker_gpu::track, src/henon.cu:3155-3185 and :636-691), moving 72 B
per particle through HBM every turn.  Its build as shipped (`oracle/_ref/
default`, FMA contraction on) is timed in a child interpreter, since two
builds of the reference cannot share one process, on a 1024^2 grid of the
dynamic-aperture scan.  Our exact-arithmetic tracker runs the same inputs.
The test prints both rates and requires ours to be clearly faster; the
measured figures are summarised with their command under profiles/.
"""
from __future__ import annotations

import json
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import pytest

from conftest import NAN, TUNES
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")

REPO = Path(__file__).resolve().parent.parent
SIDE, TURNS, EPS, MU, BARRIER = 1024, 10_000, 16.0, 0.2, 10.0

_CHILD = r"""
import json, sys, time
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import oracle as O
side, turns, eps, mu, barrier = int(sys.argv[2]), int(sys.argv[3]), float(sys.argv[4]), float(sys.argv[5]), float(sys.argv[6])
tunes = (float(sys.argv[7]), float(sys.argv[8]))
R = O.reference_module("default")
v = np.linspace(0.0, 0.6, side)
xx, yy = np.meshgrid(v, v)
x, y = xx.ravel(), yy.ravel()
z = np.zeros_like(x)
t = R.henon_tracker_gpu(turns + 10, tunes[0], tunes[1], "sps", float("nan"), eps, 0)
warm = R.particles_4d_gpu(x[:4096], z[:4096], y[:4096], z[:4096])
t.track(warm, 10, mu, barrier)
np.asarray(warm.get_steps())
p = R.particles_4d_gpu(x, z, y, z)
np.asarray(p.get_steps())
t0 = time.perf_counter()
t.track(p, turns, mu, barrier)
steps = np.asarray(p.get_steps())  # synchronous copy: the launches have finished
dt = time.perf_counter() - t0
print(json.dumps({"seconds": dt, "survivors": int((steps == turns).sum())}))
"""


def _grid():
    v = np.linspace(0.0, 0.6, SIDE)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    return x, np.zeros_like(x), y, np.zeros_like(y)


@pytest.mark.skipif(not (O.REF_DIR / "default").exists(), reason="reference build absent")
def test_faster_than_reference_gpu_path(gpu):
    out = subprocess.run([sys.executable, "-c", _CHILD, str(REPO), str(SIDE), str(TURNS),
                          str(EPS), str(MU), str(BARRIER), str(TUNES[0]), str(TUNES[1])],
                         check=True, capture_output=True, text=True)
    ref = json.loads(out.stdout.strip().splitlines()[-1])

    x, px, y, py = _grid()
    t = C.Tracker(TURNS + 10, TUNES[0], TUNES[1], "sps", NAN, EPS, 0)
    warm = C.Particles(x[:4096], px[:4096], y[:4096], py[:4096])
    t.track(warm, 10, MU, BARRIER)
    best = None
    for _ in range(3):
        p = C.Particles(x, px, y, py)
        t0 = time.perf_counter()
        t.track(p, TURNS, MU, BARRIER)
        steps = p.get(C.FIELD_STEPS)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    survivors = int((steps == TURNS).sum())

    n = x.size
    ref_rate, our_rate = n * TURNS / ref["seconds"], n * TURNS / best
    print(f"\nreference GPU path (as shipped): {ref_rate:.3e} particle-turns/s "
          f"({ref['seconds'] * 1e3:.1f} ms); ours (exact): {our_rate:.3e} ({best * 1e3:.1f} ms); "
          f"ratio {our_rate / ref_rate:.1f}x; survivors {ref['survivors']} vs {survivors}")
    # The reference build contracts FMAs, so loss turns inside the chaotic
    # sea may differ; the stable core must agree.
    assert abs(ref["survivors"] - survivors) <= 0.01 * n
    assert our_rate > 3.0 * ref_rate
