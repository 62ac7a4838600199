"""Tangent map and indicator constructs on the GPU.

Three levels, all through the C ABI:
1. the per-call classes (matrix, vector, constructs) against the numpy
   restatement of the reference loop (oracle/indicators.py): products and
   sums bit for bit, log/log10/atan2-derived values to 1e-12 relative;
2. the same classes against the reference's own GPU classes built with
   --fmad=false (oracle/_ref): bit for bit, same CUDA libm;
3. the fused multi-turn kernel (hm_track_indicators) against the per-call
   loop: bit for bit, including lost particles and whole lost warps.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, golden_json, grid
from oracle import indicators as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")

LY_W = [10, 100, 257]
MB_W = [10, 100]
TU_W = [50, 120]


def _close(a, b, rtol=1e-12, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert np.array_equal(np.isnan(a), np.isnan(b)), f"{what}: NaN patterns differ"
    m = ~np.isnan(b)
    np.testing.assert_allclose(a[m], b[m], rtol=rtol, atol=1e-300, err_msg=what)


def per_call_loop(x, px, y, py, n_turns, eps, mu, v0=(1.0, 0.0, 0.0, 0.0), barrier=10.0):
    n = len(x)
    t = C.Tracker(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = C.Particles(x, px, y, py)
    M, M_old, J = C.Matrices(n), C.Matrices(n), C.Matrices(n)
    v = C.Vectors(np.tile(np.asarray(v0, float), (n, 1)))
    ly = C.Lyapunov(n, LY_W)
    mg = C.Megno(n)
    mb = C.MegnoBirkhoff(n, MB_W)
    tu = C.TuneBirkhoff(n, TU_W)
    tu.first_add(p)
    for _ in range(n_turns):
        M_old.explicit_copy(M)
        t.track(p, 1, mu, barrier)
        M.structured_multiply(t, p, mu)
        mg.add(M, M_old)
        mb.add(M, M_old)
        J.set_with_tracker(t, p, mu)
        v.multiply(J)
        ly.add(v)
        v.normalize()
        tu.add(p)
    return dict(state=p.state(), M=M.get(), M_old=M_old.get(), v=v.get(), megno=mg.get(),
                mb=mb.get(), ly_raw=ly.get(False), ly_b=ly.get(True),
                t1x=tu.get(0), t1y=tu.get(1), t2x=tu.get(2), t2y=tu.get(3))


def fused(x, px, y, py, n_turns, eps, mu, v0=(1.0, 0.0, 0.0, 0.0), barrier=10.0, split=None,
          samples=None):
    n = len(x)
    t = C.Tracker(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = C.Particles(x, px, y, py)
    M, M_old = C.Matrices(n), C.Matrices(n)
    v = C.Vectors(np.tile(np.asarray(v0, float), (n, 1)))
    ly = C.Lyapunov(n, LY_W)
    mg = C.Megno(n)
    mb = C.MegnoBirkhoff(n, MB_W)
    tu = C.TuneBirkhoff(n, TU_W)
    tu.first_add(p)
    snap = None
    if samples is not None:
        snap = np.full((len(samples), n), -1.0)
    for part in (split or [n_turns]):
        C.track_indicators(t, p, part, mu, barrier, matrix=M, matrix_old=M_old, megno=mg,
                           megno_birkhoff=mb, vectors=v, lyapunov=ly, tune=tu,
                           megno_sample_turns=samples, megno_samples_out=snap)
    return dict(state=p.state(), M=M.get(), M_old=M_old.get(), v=v.get(), megno=mg.get(),
                mb=mb.get(), ly_raw=ly.get(False), ly_b=ly.get(True),
                t1x=tu.get(0), t1y=tu.get(1), t2x=tu.get(2), t2y=tu.get(3), snap=snap,
                global_steps=p.global_steps)


def test_per_call_classes_match_oracle(gpu):
    x, px, y, py = grid(0.5, 12)
    got = per_call_loop(x, px, y, py, 300, 16.0, 0.2)
    tabs = O.tables(301, TUNES[0], TUNES[1], "sps", epsilon=16.0)
    L = I.ConstructLoop(x, px, y, py, tabs, 0.2, 10.0, [1, 0, 0, 0], LY_W, MB_W, TU_W).run(300)
    for a, b in zip(got["state"][:4], (L.x, L.px, L.y, L.py)):
        assert_bitwise(a, b)
    np.testing.assert_array_equal(got["state"][4], L.steps)
    assert_bitwise(got["M"], L.M, "tangent matrices")
    _close(got["v"], L.v, 1e-13, "tangent vectors")
    _close(got["megno"], L.m_l3, 1e-12, "megno")
    _close(got["mb"], L.mb_l2, 1e-12, "megno birkhoff")
    _close(got["ly_raw"], L.ly_raw, 1e-12, "lyapunov raw")
    _close(got["ly_b"], L.ly_b, 1e-12, "lyapunov birkhoff")
    for k, ref in (("t1x", L.t1x), ("t1y", L.t1y), ("t2x", L.t2x), ("t2y", L.t2y)):
        _close(got[k], ref, 1e-12, k)
    assert np.isnan(got["megno"]).any() and (~np.isnan(got["megno"])).any()


@pytest.mark.parametrize("eps,mu", [(16.0, 0.2), (64.0, 0.0)])
def test_fused_equals_per_call_loop(gpu, eps, mu):
    # 32 large-amplitude particles first (a whole warp that is lost early),
    # then a grid with a chaotic border.
    x, px, y, py = grid(0.55, 14)
    x = np.concatenate([np.full(32, 0.9), x])
    y = np.concatenate([np.linspace(0.7, 0.9, 32), y])
    px = np.concatenate([np.zeros(32), px])
    py = np.concatenate([np.zeros(32), py])
    n_turns = 700
    ref = per_call_loop(x, px, y, py, n_turns, eps, mu)
    got = fused(x, px, y, py, n_turns, eps, mu, split=[1, 250, 449])
    for a, b in zip(got["state"], ref["state"]):
        assert_bitwise(a, b) if a.dtype == np.float64 else np.testing.assert_array_equal(a, b)
    for k in ("M", "M_old", "v", "megno", "mb", "ly_raw", "ly_b", "t1x", "t1y", "t2x", "t2y"):
        assert_bitwise(got[k], ref[k], k)
    assert got["global_steps"] == n_turns
    assert np.isnan(got["megno"][:32]).all()


@pytest.mark.parametrize("use", ["MVT", "MV", "MT", "VT", "M", "V", "T"])
def test_fused_subsets_equal_per_call_loop(gpu, use):
    # Every combination of constructs runs its own kernel variant (with the
    # matrix and the vector or tune work split over two warps per particle
    # when both are present); each must give the per-call loop's values.
    x, px, y, py = grid(0.55, 12)
    n_turns = 400
    ref = per_call_loop(x, px, y, py, n_turns, 32.0, 0.2)
    n = len(x)
    t = C.Tracker(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, 32.0, 0)
    p = C.Particles(x, px, y, py)
    kw = {}
    if "M" in use:
        M, M_old = C.Matrices(n), C.Matrices(n)
        mg, mb = C.Megno(n), C.MegnoBirkhoff(n, MB_W)
        kw.update(matrix=M, matrix_old=M_old, megno=mg, megno_birkhoff=mb)
    if "V" in use:
        v = C.Vectors(np.tile(np.asarray((1.0, 0.0, 0.0, 0.0)), (n, 1)))
        ly = C.Lyapunov(n, LY_W)
        kw.update(vectors=v, lyapunov=ly)
    if "T" in use:
        tu = C.TuneBirkhoff(n, TU_W)
        tu.first_add(p)
        kw.update(tune=tu)
    for part in (150, 250):
        C.track_indicators(t, p, part, 0.2, 10.0, **kw)
    for a, b in zip(p.state(), ref["state"]):
        assert_bitwise(a, b) if a.dtype == np.float64 else np.testing.assert_array_equal(a, b)
    if "M" in use:
        for k, got in (("M", M.get()), ("M_old", M_old.get()), ("megno", mg.get()),
                       ("mb", mb.get())):
            assert_bitwise(got, ref[k], f"{use}:{k}")
    if "V" in use:
        for k, got in (("v", v.get()), ("ly_raw", ly.get(False)), ("ly_b", ly.get(True))):
            assert_bitwise(got, ref[k], f"{use}:{k}")
    if "T" in use:
        for j, k in enumerate(("t1x", "t1y", "t2x", "t2y")):
            assert_bitwise(tu.get(j), ref[k], f"{use}:{k}")


def test_fused_megno_samples(gpu):
    x, px, y, py = grid(0.5, 10)
    samples = [1, 7, 64, 200, 399, 400, 401, 10_000]
    got = fused(x, px, y, py, 400, 32.0, 0.0, samples=samples)
    tabs = O.tables(401, TUNES[0], TUNES[1], "sps", epsilon=32.0)
    L = I.ConstructLoop(x, px, y, py, tabs, 0.0, 10.0, [1, 0, 0, 0], LY_W, MB_W, TU_W).run(400)
    for j, s in enumerate(samples):
        if s <= 400:
            _close(got["snap"][j], L.megno_history[s - 1], 1e-12, f"sample {s}")
        else:
            assert np.all(got["snap"][j] == -1.0)  # never reached: left untouched
    assert_bitwise(got["snap"][samples.index(400)], got["megno"])


@pytest.mark.skipif(O.reference_module("fmad_off") is None, reason="reference build absent")
def test_per_call_classes_equal_reference_gpu_classes(gpu):
    R = O.reference_module("fmad_off")
    x, px, y, py = grid(0.5, 10)
    n, n_turns, eps, mu = x.size, 200, 16.0, 0.2
    t = R.henon_tracker_gpu(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = R.particles_4d_gpu(x, px, y, py)
    M, M_old, J = (R.matrix_4d_vector_gpu(n) for _ in range(3))
    v = R.vector_4d_gpu(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1)))
    ly = R.lyapunov_birkhoff_construct_multi(n, LY_W)
    mg = R.megno_construct(n)
    mb = R.megno_birkhoff_construct(n, MB_W)
    tu = R.tune_birkhoff_construct(n, TU_W)
    tu.reset()  # the reference leaves its tune accumulators uninitialised
    tu.first_add(p)
    for _ in range(n_turns):
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
    ours = per_call_loop(x, px, y, py, n_turns, eps, mu)
    assert_bitwise(ours["M"], np.asarray(M.get_matrix()), "matrices")
    assert_bitwise(ours["v"], np.asarray(v.get_vectors()), "vectors")
    assert_bitwise(ours["megno"], np.asarray(mg.get_values()), "megno")
    assert_bitwise(ours["mb"], np.asarray(mb.get_values()), "megno birkhoff")
    assert_bitwise(ours["ly_raw"], np.asarray(ly.get_values_raw()), "lyapunov raw")
    assert_bitwise(ours["ly_b"], np.asarray(ly.get_values_b()), "lyapunov birkhoff")
    assert_bitwise(ours["t1x"], np.asarray(tu.get_tune1_x()), "tune1_x")
    assert_bitwise(ours["t2y"], np.asarray(tu.get_tune2_y()), "tune2_y")
    assert_bitwise(ours["state"][0], np.asarray(p.get_x()), "x")


def test_notebook_known_answers_on_gpu(gpu):
    nb = golden_json("notebook_values.json")
    t = C.Tracker(1000, TUNES[0], TUNES[1], "sps", NAN, 0.0, 0)
    p = C.Particles(np.full(3, 0.1), np.zeros(3), np.full(3, 0.1), np.zeros(3))
    m1, m2 = C.Matrices(3), C.Matrices(3)
    m1.set_with_tracker(t, p, 0.0)
    t.track(p, 1, 0.0, 10.0)
    m2.set_with_tracker(t, p, 0.0)
    np.testing.assert_allclose(m1.get()[0], nb["tangent_matrix_x0"]["matrix"], rtol=1e-7, atol=1e-8)
    np.testing.assert_allclose(m2.get()[0], nb["tangent_matrix_x1"]["matrix"], rtol=1e-7, atol=1e-8)
    np.testing.assert_allclose(p.get(C.FIELD_X), nb["x_after_one_turn"]["value"], rtol=1e-7)
    # lyapunov_birkhoff_construct_multi(3, [5, 10, 15]) fed v = (1, 1, 0, 0)
    v = C.Vectors(np.tile([1.0, 1.0, 0.0, 0.0], (3, 1)))
    ly = C.Lyapunov(3, [5, 10, 15])
    lw = nb["lyapunov_multi_windows"]
    for tag in ("5", "10", "15"):
        for _ in range(5):
            ly.add(v)
        np.testing.assert_allclose(ly.get(False)[:, 0], lw[f"raw_after_{tag}"], rtol=1e-7, atol=5e-9)
        np.testing.assert_allclose(ly.get(True)[:, 0], lw[f"b_after_{tag}"], rtol=1e-7, atol=5e-9)
    single = C.Lyapunov(3, 7)
    single.change_weights(10)
    np.testing.assert_allclose(single.weights(0), nb["birkhoff_weights_10"]["value"], rtol=1e-7,
                               atol=1e-12)
    # v = (1, 0, 0, 0); v.multiply(DF(x0)); normalize()
    v = C.Vectors(np.tile([1.0, 0.0, 0.0, 0.0], (3, 1)))
    v.multiply(m1)
    vm = nb["vector_multiply_normalize"]
    np.testing.assert_allclose(v.get()[0], vm["multiplied"], rtol=1e-7)
    v.normalize()
    np.testing.assert_allclose(v.get()[0], vm["normalized"], rtol=1e-7)


def test_storage_and_matrix_helpers(gpu):
    x, px, y, py = grid(0.3, 5)
    n = x.size
    t = C.Tracker(10, TUNES[0], TUNES[1], "sps", NAN, 8.0, 0)
    p = C.Particles(x, px, y, py)
    st = C.Storage(n, 3)
    st.store(p)
    t.track(p, 2, 0.1, 10.0)
    st.store(p)
    xs = st.get(C.FIELD_X)
    assert_bitwise(xs[0], x)
    assert_bitwise(xs[1], p.get(C.FIELD_X))
    assert np.all(xs[2] == 0.0)
    st.store(p)
    with pytest.raises(ValueError, match="full"):
        st.store(p)
    st.reset()
    assert np.all(st.get(C.FIELD_PY) == 0.0)
    m = C.Matrices(n)
    m.set_with_tracker(t, p, 0.1)
    rv = np.random.default_rng(1).normal(size=(n, 4))
    M = m.get()
    want = (((M[:, :, 0] * rv[:, [0]]) + M[:, :, 1] * rv[:, [1]]) + M[:, :, 2] * rv[:, [2]]) \
        + M[:, :, 3] * rv[:, [3]]
    assert_bitwise(m.get_vector(rv), want)
    m.reset()
    assert_bitwise(m.get(), np.tile(np.eye(4), (n, 1, 1)))
    with pytest.raises(ValueError, match="add_first"):
        C.TuneBirkhoff(n, [5]).add(p)


def test_fused_many_windows_in_any_order(gpu):
    # The fused kernel sorts each kind's windows by closing index into a
    # table and keeps the accumulators in that order: 40 MEGNO-Birkhoff
    # windows and 8 Lyapunov and 8 tune windows (88 of the 96 accumulator
    # slots), given out of order and with repeated lengths, must come back
    # in the construct's order with the per-call loop's values.
    rng = np.random.default_rng(11)
    x, px, y, py = grid(0.5, 6)
    n, n_turns = x.size, 300
    mb_w = [int(t) for t in rng.permutation(np.r_[np.linspace(5, 400, 37).round(), 5, 100, 300])]
    ly_w = [int(t) for t in rng.permutation([3, 50, 50, 120, 299, 300, 301, 1])]
    tu_w = [int(t) for t in rng.permutation([2, 40, 40, 150, 151, 75, 149, 10])]
    t = C.Tracker(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)
    p = C.Particles(x, px, y, py)
    M, Mo, mg, mb = C.Matrices(n), C.Matrices(n), C.Megno(n), C.MegnoBirkhoff(n, mb_w)
    V, ly, tu = C.Vectors(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))), C.Lyapunov(n, ly_w), C.TuneBirkhoff(n, tu_w)
    tu.first_add(p)
    C.track_indicators(t, p, n_turns, 0.2, 10.0, matrix=M, matrix_old=Mo, megno=mg,
                       megno_birkhoff=mb, vectors=V, lyapunov=ly, tune=tu,
                       megno_sample_turns=[7, 300], megno_samples_out=None)
    t2 = C.Tracker(n_turns + 1, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)
    p2 = C.Particles(x, px, y, py)
    M2, Mo2, mg2, mb2 = C.Matrices(n), C.Matrices(n), C.Megno(n), C.MegnoBirkhoff(n, mb_w)
    V2, ly2, tu2 = C.Vectors(np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))), C.Lyapunov(n, ly_w), C.TuneBirkhoff(n, tu_w)
    tu2.first_add(p2)
    J = C.Matrices(n)
    for _ in range(n_turns):
        Mo2.explicit_copy(M2)
        t2.track(p2, 1, 0.2, 10.0)
        M2.structured_multiply(t2, p2, 0.2)
        mg2.add(M2, Mo2)
        mb2.add(M2, Mo2)
        J.set_with_tracker(t2, p2, 0.2)
        V2.multiply(J)
        ly2.add(V2)
        V2.normalize()
        tu2.add(p2)
    assert_bitwise(mb.get(), mb2.get(), "megno birkhoff, 40 windows")
    assert_bitwise(mg.get(), mg2.get(), "megno")
    assert_bitwise(M.get(), M2.get(), "matrices")
    assert_bitwise(V.get(), V2.get(), "vectors")
    assert_bitwise(ly.get(False), ly2.get(False), "lyapunov")
    assert_bitwise(ly.get(True), ly2.get(True), "lyapunov birkhoff")
    for j in range(4):
        assert_bitwise(tu.get(j), tu2.get(j), f"tunes {j}")
