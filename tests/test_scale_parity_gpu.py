"""Parity at the benchmark configurations' own sizes, against the reference's
own CUDA path built with --fmad=false (oracle/_ref/fmad_off).

* The modulated dynamic-aperture scan as the bench runs it: the 1024^2 grid
  on [0, 0.6]^2, all six (epsilon, mu) scans, 10^5 turns.  Exact arithmetic
  must give the reference GPU tracker's coordinates and survival turns bit
  for bit (henon_tracker_gpu::track, src/henon.cu:3155-3185, one
  gpu_henon_track launch per turn).  The reference runs in a child
  interpreter (about 16 s per scan on a B200).
* The tangent-map indicators at the indicator configuration's shape: a
  subsample of the 512^2 grid on [0, 0.4]^2, epsilon 32, mu 0, 10^4 turns
  in one fused call (three 4096-turn launches), with the 13 log-spaced
  windows 10^2..10^5 of MEGNO-Birkhoff, Lyapunov and Birkhoff tunes and
  MEGNO sampled at the window turns.  The fused kernel must give the values
  of the reference's own per-turn construct loop on its GPU classes
  (src/henon.cu:1694-2655) bit for bit.
* The inverse tangent matrix (inverse_tangent_matrix, src/henon.cu:224-249)
  through get_tangent_matrix(..., reverse=True).
* The scan's second horizon, 10^6 turns, on every 16th point of the
  1024^2 grid per axis (4096 particles) for two of the six scans.
* Backward tracking (track(..., inverse=True): the reverse turn with
  table[steps - 1], steps decreasing, src/henon.cu:510-528) after forward
  turns, on a 256^2 grid, against the reference's GPU tracker.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, grid
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")

needs_ref = pytest.mark.skipif(not (O.REF_DIR / "fmad_off").exists(),
                               reason="reference build absent")

SCAN_SIDE, SCAN_TURNS = 1024, 100_000
WINDOWS = [int(t) for t in np.unique(np.round(np.logspace(2, 5, 13)))]


def _scan_grid():
    v = np.linspace(0.0, 0.6, SCAN_SIDE)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    return x, np.zeros_like(x), y, np.zeros_like(y)


@needs_ref
@pytest.mark.parametrize("eps,mu", [(1.0, 0.0), (1.0, 0.2), (16.0, 0.0), (16.0, 0.2),
                                    (64.0, 0.0), (64.0, 0.2)])
def test_da_scan_bit_exact_vs_reference_gpu(gpu, eps, mu):
    x, px, y, py = _scan_grid()
    ref = O.reference_track_subprocess("fmad_off", x, px, y, py, SCAN_TURNS, TUNES, eps, mu,
                                       10.0, gpu=True)
    t = C.Tracker(SCAN_TURNS, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = C.Particles(x, px, y, py)
    t.track(p, SCAN_TURNS, mu, 10.0)
    got = p.state()
    np.testing.assert_array_equal(got[4], ref[4], err_msg=f"steps eps={eps} mu={mu}")
    for a, b, name in zip(got[:4], ref[:4], ("x", "px", "y", "py")):
        assert_bitwise(a, b, f"{name} eps={eps} mu={mu}")
    survivors = int(np.sum(got[4] == SCAN_TURNS))
    assert 0 < survivors < x.size


def _c3_sample():
    v = np.linspace(0.0, 0.4, 512)[::8]  # 64^2 points of the 512^2 grid
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    return x, np.zeros_like(x), y, np.zeros_like(y)


def _reference_construct_loop(R, x, px, y, py, n_turns, eps, mu):
    n = x.size
    t = R.henon_tracker_gpu(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = R.particles_4d_gpu(x, px, y, py)
    M, M_old, J = (R.matrix_4d_vector_gpu(n) for _ in range(3))
    v = R.vector_4d_gpu(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1)))
    ly = R.lyapunov_birkhoff_construct_multi(n, WINDOWS)
    mg = R.megno_construct(n)
    mb = R.megno_birkhoff_construct(n, WINDOWS)
    tu = R.tune_birkhoff_construct(n, WINDOWS)
    tu.reset()  # the reference leaves its tune accumulators uninitialised
    tu.first_add(p)
    snaps = {}
    for k in range(1, n_turns + 1):
        M_old.explicit_copy(M)
        t.track(p, 1, mu, 10.0)
        M.structured_multiply(t, p, mu)
        mg.add(M, M_old)
        mb.add(M, M_old)
        J.set_with_tracker(t, p, mu)
        v.multiply(J)
        ly.add(v)
        v.normalize()
        tu.add(p)
        if k in WINDOWS:
            snaps[k] = np.asarray(mg.get_values()).copy()
    return dict(x=np.asarray(p.get_x()), px=np.asarray(p.get_px()), y=np.asarray(p.get_y()),
                py=np.asarray(p.get_py()), steps=np.asarray(p.get_steps()),
                M=np.asarray(M.get_matrix()), v=np.asarray(v.get_vectors()),
                megno=np.asarray(mg.get_values()), mb=np.asarray(mb.get_values()),
                ly_raw=np.asarray(ly.get_values_raw()), ly_b=np.asarray(ly.get_values_b()),
                t1x=np.asarray(tu.get_tune1_x()), t1y=np.asarray(tu.get_tune1_y()),
                t2x=np.asarray(tu.get_tune2_x()), t2y=np.asarray(tu.get_tune2_y()),
                snaps=snaps)


@needs_ref
def test_fused_indicators_c3_shape_vs_reference_gpu_classes(gpu):
    R = O.reference_module("fmad_off")
    x, px, y, py = _c3_sample()
    n, n_turns, eps, mu = x.size, 10_000, 32.0, 0.0
    assert len(WINDOWS) == 13

    t = C.Tracker(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = C.Particles(x, px, y, py)
    M, M_old = C.Matrices(n), C.Matrices(n)
    v = C.Vectors(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1)))
    ly, mg = C.Lyapunov(n, WINDOWS), C.Megno(n)
    mb, tu = C.MegnoBirkhoff(n, WINDOWS), C.TuneBirkhoff(n, WINDOWS)
    tu.first_add(p)
    samples = [w for w in WINDOWS if w <= n_turns]
    snap = np.full((len(samples), n), -1.0)
    # one call: the kernel crosses two 4096-turn launch boundaries inside it
    C.track_indicators(t, p, n_turns, mu, 10.0, matrix=M, matrix_old=M_old, megno=mg,
                       megno_birkhoff=mb, vectors=v, lyapunov=ly, tune=tu,
                       megno_sample_turns=samples, megno_samples_out=snap)

    ref = _reference_construct_loop(R, x, px, y, py, n_turns, eps, mu)
    st = p.state()
    for a, name in zip(st[:4], ("x", "px", "y", "py")):
        assert_bitwise(a, ref[name], name)
    np.testing.assert_array_equal(st[4], ref["steps"])
    assert_bitwise(M.get(), ref["M"], "tangent matrices")
    assert_bitwise(v.get(), ref["v"], "tangent vectors")
    assert_bitwise(mg.get(), ref["megno"], "megno")
    assert_bitwise(mb.get(), ref["mb"], "megno birkhoff (13 windows)")
    assert_bitwise(ly.get(False), ref["ly_raw"], "lyapunov raw (13 windows)")
    assert_bitwise(ly.get(True), ref["ly_b"], "lyapunov birkhoff (13 windows)")
    for j, k in enumerate(("t1x", "t1y", "t2x", "t2y")):
        assert_bitwise(tu.get(j), ref[k], f"tune {k} (13 windows)")
    for j, s in enumerate(samples):
        assert_bitwise(snap[j], ref["snaps"][s], f"megno at turn {s}")
    # the sample holds lost particles and a chaotic border
    lost = np.sum(st[4] < n_turns)
    assert 0 < lost < n
    assert np.isnan(mg.get()).any() and np.isfinite(mg.get()).any()


@needs_ref
@pytest.mark.parametrize("mu", [0.0, 0.2])
def test_reverse_tangent_matrix_vs_reference_gpu(gpu, mu):
    R = O.reference_module("fmad_off")
    x, px, y, py = grid(0.45, 12, px0=0.01, py0=-0.02)
    n_turns = 137
    t = C.Tracker(n_turns + 5, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)
    p = C.Particles(x, px, y, py)
    t.track(p, n_turns, mu, 10.0)
    rt = R.henon_tracker_gpu(n_turns + 5, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)
    rp = R.particles_4d_gpu(x, px, y, py)
    rt.track(rp, n_turns, mu, 10.0)
    n = x.size
    for reverse in (True, False):
        ours = np.empty(16 * n)
        C.call("hm_tracker_tangent_matrices", t.h, p.h, mu, int(reverse), C.dptr(ours))
        theirs = np.asarray(rt.get_tangent_matrix(rp, mu, reverse), dtype=np.float64)
        assert_bitwise(ours.reshape(theirs.shape), theirs, f"reverse={reverse}")
        assert np.isfinite(ours).any()


@needs_ref
@pytest.mark.parametrize("mu", [0.0, 0.2])
def test_backward_tracking_bit_exact_vs_reference_gpu(gpu, mu):
    v = np.linspace(0.0, 0.5, 256)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    px = np.full_like(x, 1e-3)
    py = np.zeros_like(x)
    n_fwd, n_back = 3000, 2000
    ref = O.reference_track_subprocess("fmad_off", x, px, y, py, n_fwd, TUNES, 16.0, mu, 10.0,
                                       gpu=True, n_back=n_back)
    t = C.Tracker(n_fwd, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)
    p = C.Particles(x, px, y, py)
    t.track(p, n_fwd, mu, 10.0)
    t.track(p, n_back, mu, 10.0, float("nan"), True)
    got = p.state()
    np.testing.assert_array_equal(got[4], ref[4], err_msg=f"steps mu={mu}")
    for a, b, name in zip(got[:4], ref[:4], ("x", "px", "y", "py")):
        assert_bitwise(a, b, f"{name} mu={mu}")
    assert p.global_steps == n_fwd - n_back
    lost = np.isnan(got[0])
    assert lost.any() and not lost.all()


@needs_ref
@pytest.mark.parametrize("eps,mu", [(1.0, 0.0), (64.0, 0.2)])
def test_long_horizon_subsample_bit_exact_vs_reference_gpu(gpu, eps, mu):
    x, px, y, py = (c.reshape(SCAN_SIDE, SCAN_SIDE)[::16, ::16].ravel() for c in _scan_grid())
    n_turns = 1_000_000
    ref = O.reference_track_subprocess("fmad_off", x, px, y, py, n_turns, TUNES, eps, mu, 10.0,
                                       gpu=True)
    t = C.Tracker(n_turns, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = C.Particles(x, px, y, py)
    t.track(p, n_turns, mu, 10.0)
    got = p.state()
    np.testing.assert_array_equal(got[4], ref[4], err_msg=f"steps eps={eps} mu={mu}")
    for a, b, name in zip(got[:4], ref[:4], ("x", "px", "y", "py")):
        assert_bitwise(a, b, f"{name} eps={eps} mu={mu}")
    survivors = int(np.sum(got[4] == n_turns))
    assert 0 < survivors < x.size
