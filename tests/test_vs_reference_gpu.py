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


_TUNES_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import oracle as O
d = np.load(sys.argv[2])
R = O.reference_module("default")
t = R.henon_tracker(int(d["n_turns"]), float(d["tunes"][0]), float(d["tunes"][1]), "sps",
                    float("nan"), float(d["epsilon"]), 0)
frm, to = [int(v) for v in d["frm"]], [int(v) for v in d["to"]]
p = R.particles_4d(d["x"], d["px"], d["y"], d["py"])
b = np.asarray(t.birkhoff_tunes(p, int(d["n_turns"]), float(d["mu"]), 10.0, float("nan"), False,
                                frm, to))
p = R.particles_4d(d["x"], d["px"], d["y"], d["py"])
ab, af = t.all_tunes(p, int(d["n_turns"]), float(d["mu"]), 10.0, float("nan"), False, frm, to)
np.savez(sys.argv[3], birkhoff=b, all_birkhoff=np.asarray(ab), all_fft=np.asarray(af))
"""


@pytest.mark.skipif(not (O.REF_DIR / "default").exists(), reason="reference build absent")
def test_tunes_match_the_reference_cpu_tracker(gpu, tmp_path):
    # birkhoff_tunes and all_tunes of the reference's own henon_tracker
    # (src/henon.cu:2890-3078: CPU tracking, Birkhoff sums, FFTW tunes --
    # cuFFTW in the checker build) against ours on the same particles.
    # Birkhoff: 1e-13 (our sums run in segments of turns); FFT: 1e-10.
    from henon_map_cpp_b200 import henon_map_engine as E

    x, px, y, py = (np.ascontiguousarray(a) for a in _grid_small())
    n_turns, eps, mu = 2000, 16.0, 0.2
    frm, to = [0, 100, 700], [500, 1001, 1999]
    inp, out = tmp_path / "in.npz", tmp_path / "out.npz"
    np.savez(inp, x=x, px=px, y=y, py=py, n_turns=n_turns, tunes=np.asarray(TUNES),
             epsilon=eps, mu=mu, frm=np.asarray(frm), to=np.asarray(to))
    subprocess.run([sys.executable, "-c", _TUNES_CHILD, str(REPO), str(inp), str(out)],
                   check=True, capture_output=True, text=True)
    ref = np.load(out)
    t = E.henon_tracker_gpu(n_turns, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    b = np.asarray(t.birkhoff_tunes(E.particles_4d_gpu(x, px, y, py), n_turns, mu, 10.0, NAN,
                                    False, frm, to))
    ab, af = (np.asarray(a) for a in t.all_tunes(E.particles_4d_gpu(x, px, y, py), n_turns, mu,
                                                  10.0, NAN, False, frm, to))
    for got, want, rtol, what in ((b, ref["birkhoff"], 1e-13, "birkhoff_tunes"),
                                  (ab, ref["all_birkhoff"], 1e-13, "all_tunes birkhoff"),
                                  (af, ref["all_fft"], 1e-10, "all_tunes fft")):
        assert got.shape == want.shape, what
        if what == "all_tunes fft":
            # The reference's NaN scan of a window reads from the window's
            # start to past the end of the orbit vector
            # (src/dynamic_indicator.cpp:284-287), so it may report NaN for a
            # window without one; here the window itself is scanned.  Where
            # the reference gives a value, ours must match it; the full
            # orbit (its last two columns) is scanned correctly by both.
            full = slice(-2, None)
            assert np.array_equal(np.isnan(got[:, full]), np.isnan(want[:, full])), what
            assert np.all(np.isnan(got) <= np.isnan(want)), what
        else:
            assert np.array_equal(np.isnan(got), np.isnan(want)), what
        m = ~np.isnan(want)
        np.testing.assert_allclose(got[m], want[m], rtol=rtol, atol=1e-14, err_msg=what)
    assert np.isnan(ab).any() and np.isfinite(af).any()
    # the window scan: a window of a particle that survives all turns is
    # finite here whatever the reference's scan past the vector end found
    alive = np.all(np.isfinite(ab), axis=1)
    assert np.all(np.isfinite(af[alive]))


def _grid_small():
    v = np.linspace(0.0, 0.55, 12)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    return x, np.full_like(x, 0.001), y, np.zeros_like(y)
