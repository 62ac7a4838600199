"""Tune estimates on the GPU (Birkhoff and FFT over orbit windows, the
tracker's whole-orbit tunes and MEGNO, storage tunes) against the oracle
(oracle/tunes.py) and the values recorded in the reference's notebooks."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, golden_json, grid
from oracle import oracle as O
from oracle import tunes as T

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")
hm = pytest.importorskip("henon_map_cpp_b200")


def _close(a, b, rtol, what=""):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert np.array_equal(np.isnan(a), np.isnan(b)), what
    m = ~np.isnan(b)
    np.testing.assert_allclose(a[m], b[m], rtol=rtol, atol=0, err_msg=what)


def test_tune_all_reproduces_notebook(gpu):
    nb = golden_json("notebook_values.json")["tunes_0p1_eps0"]
    p = hm.particles(np.full(4, 0.1), np.zeros(4), np.full(4, 0.1), np.zeros(4))
    t = hm.henon_tracker(10000, *TUNES, "sps")
    df = t.tune_all(p, 10000, 0.0, from_idx=np.array([0, 500]), to_idx=np.array([500, 1000]))
    assert list(df["from"]) == [0, 500, 0] and list(df["to"]) == [500, 1000, 10000]
    bx = [np.asarray(df["tune_x_birkhoff"][i]) for i in range(3)]
    fx = [np.asarray(df["tune_x_fft"][i]) for i in range(3)]
    fy = [np.asarray(df["tune_y_fft"][i]) for i in range(3)]
    np.testing.assert_allclose(bx[0], nb["birkhoff_x"]["0-500"], rtol=1e-13)
    np.testing.assert_allclose(bx[1], nb["birkhoff_x"]["500-1000"], rtol=1e-13)
    np.testing.assert_allclose(bx[2], nb["birkhoff_x"]["0-10000"], rtol=1e-13)
    np.testing.assert_allclose(fx[2], nb["fft_x"]["1-10000"], rtol=1e-12)
    np.testing.assert_allclose(fy[2], nb["fft_y"]["1-10000"], rtol=1e-12)


@pytest.mark.parametrize("remove_mean", [False, True])
def test_tracker_orbit_tunes_match_oracle(gpu, remove_mean):
    x, px, y, py = grid(0.6, 10, px0=0.002)
    n_turns = 1200
    frm, to = [0, 100, 300, 37], [99, 700, 1200, 37]
    tr = C.Tracker(n_turns, *TUNES, "sps", NAN, 16.0, 0)
    p = C.Particles(x, px, y, py)
    b, f = C.tracker_orbit_tunes(tr, p, n_turns, 0.2, 10.0, frm, to, remove_mean, True)
    orb = T.orbit(x, px, y, py, O.tables(n_turns, *TUNES, "sps", epsilon=16.0), n_turns, 0.2)
    if remove_mean:
        orb = T.remove_mean(orb)
    want_b = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "birkhoff")
                       for i in range(x.size)])
    want_f = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "fft")
                       for i in range(x.size)])
    _close(b, want_b, 1e-13, "birkhoff")
    _close(f, want_f, 1e-10, "fft")
    assert np.isnan(b[:, 0]).any() and np.isfinite(b[:, 0]).any()
    assert p.global_steps == n_turns
    steps = p.get(C.FIELD_STEPS)
    want = O.track(x, px, y, py, np.zeros(x.size, np.uint32),
                   O.tables(n_turns, *TUNES, "sps", epsilon=16.0), n_turns, 0.2, 10.0)
    np.testing.assert_array_equal(steps, want[4])


@pytest.mark.parametrize("remove_mean", [False, True])
def test_tracker_fft_tunes_window_lengths(gpu, remove_mean):
    # Window lengths across the transform's cases: one sample; lengths of
    # radices 2, 3, 4 and 5 only, transformed directly (up to the longest
    # row one block holds, 12800); Bluestein's convolution for other
    # lengths (7, 1001 = 7 * 11 * 13, the prime 4001, 5001 = 3 * 1667, and
    # 6400, whose convolution of 12799 values takes the longest row); and
    # lengths beyond both (6401, 12801), which take the library transform.
    x, px, y, py = grid(0.25, 3, px0=0.001)
    lengths = [1, 2, 3, 7, 16, 64, 125, 1001, 4001, 5001, 6400, 6401, 10000, 12800, 12801]
    n_turns = 13000
    frm = [(37 * j) % 150 for j in range(len(lengths))]
    to = [f + n - 1 for f, n in zip(frm, lengths)]
    tr = C.Tracker(n_turns, *TUNES, "sps", NAN, 8.0, 0)
    p = C.Particles(x, px, y, py)
    _, f = C.tracker_orbit_tunes(tr, p, n_turns, 0.0, 10.0, frm, to, remove_mean, True)
    orb = T.orbit(x, px, y, py, O.tables(n_turns, *TUNES, "sps", epsilon=8.0), n_turns, 0.0)
    if remove_mean:
        orb = T.remove_mean(orb)
    want = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "fft")
                     for i in range(x.size)])
    assert np.isfinite(want).all()
    _close(f, want, 1e-10, "fft")


@pytest.mark.parametrize("remove_mean", [False, True])
def test_fft_tunes_of_a_resting_particle(gpu, remove_mean):
    # A particle at the origin stays there: every window's spectrum is zero,
    # whose first maximum is bin 0, so the FFT tune is 1.0 on the direct
    # (1000, 2^3 5^3), Bluestein (1001, 4001) and library (12801) transforms
    # alike, as in the oracle; the moving particle beside it is compared too.
    x = np.array([0.0, 0.1])
    z = np.zeros(2)
    y = np.array([0.0, 0.1])
    n_turns = 13000
    frm, to = [0, 10, 100, 0], [999, 1010, 4100, 12800]
    tr = C.Tracker(n_turns, *TUNES, "sps", NAN, 0.0, 0)
    p = C.Particles(x, z, y, z)
    b, f = C.tracker_orbit_tunes(tr, p, n_turns, 0.0, 10.0, frm, to, remove_mean, True)
    assert (f[0] == 1.0).all()
    orb = T.orbit(x, z, y, z, O.tables(n_turns, *TUNES, "sps", epsilon=0.0), n_turns, 0.0)
    if remove_mean:
        orb = T.remove_mean(orb)
    want = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "fft")
                     for i in range(2)])
    _close(f, want, 1e-10, "fft")


def test_tracker_orbit_tunes_in_slices(gpu):
    # A cap on the particles of one slice (hm_set_tune_slice_limit) splits
    # the orbit into slices of 7 particles: every slice's record continues the
    # same particles (kicks keyed by the global index), the FFT rows are the
    # same rows, and only the Birkhoff sums' segments change (1e-13).
    x, px, y, py = grid(0.3, 5, px0=0.001)
    frm, to = [0, 100, 300], [99, 700, 1500]

    def run(limit):
        C.call("hm_set_tune_slice_limit", limit)
        try:
            tr = C.Tracker(1500, *TUNES, "sps", NAN, 16.0, 0)
            p = C.Particles(x, px, y, py)
            p.kick_seed = 77
            b, f = C.tracker_orbit_tunes(tr, p, 1500, 0.2, 10.0, frm, to, True, True,
                                         kick_module=1e-7)
            return b, f, p.get(C.FIELD_X), p.get(C.FIELD_STEPS)
        finally:
            C.call("hm_set_tune_slice_limit", 0)

    b0, f0, x0, s0 = run(0)
    b7, f7, x7, s7 = run(7)
    assert_bitwise(f7, f0)
    assert_bitwise(x7, x0)
    np.testing.assert_array_equal(s7, s0)
    _close(b7, b0, 1e-13, "birkhoff")
    got = ctypes.c_size_t(1)
    C.call("hm_get_tune_slice_limit", ctypes.byref(got))
    assert got.value == 0


def test_storage_tunes_match_oracle(gpu):
    x, px, y, py = grid(0.3, 6)
    n = x.size
    tr = C.Tracker(300, *TUNES, "sps", NAN, 8.0, 0)
    p = C.Particles(x, px, y, py)
    st = C.Storage(n, 301)
    st.store(p)
    for _ in range(300):
        tr.track(p, 1, 0.0, 10.0)
        st.store(p)
    frm, to = [0, 50], [149, 300]
    b = C.storage_tunes(st, frm, to, 0)
    f = C.storage_tunes(st, frm, to, 1)
    orb = np.stack([st.get(k) for k in (C.FIELD_X, C.FIELD_PX, C.FIELD_Y, C.FIELD_PY)])
    want_b = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "birkhoff")
                       for i in range(n)])
    want_f = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "fft")
                       for i in range(n)])
    _close(b, want_b, 1e-13, "birkhoff")
    _close(f, want_f, 1e-10, "fft")
    # the host-side facade storage gives the same
    hp = hm.particles(x, px, y, py)
    ht = hm.henon_tracker(300, *TUNES, "sps", np.nan, 8.0, 0)
    hs = hm.storage(n)
    hs.store(hp)
    for _ in range(300):
        ht.track(hp, 1, 0.0)
        hs.store(hp)
    df = hs.tune_birkhoff(frm, to, 300)
    _close(np.stack(df["tune_x"].to_list()), b[:, 0::2].T, 0, "facade storage")


def test_tracker_megno_equals_construct_loop(gpu):
    x, px, y, py = grid(0.5, 8)
    n = x.size
    t = hm.henon_tracker(500, *TUNES, "sps", np.nan, 16.0, 0)
    p = hm.particles(x, px, y, py)
    got = t.megno(p, 500, 0.2, turn_samples=np.array([100, 500]))
    assert got.shape == (n, 2)
    # the same by the per-call classes: tangent map of each turn, then track
    t2 = hm.henon_tracker(500, *TUNES, "sps", np.nan, 16.0, 0)
    p2 = hm.particles(x, px, y, py)
    M, Mo, mg = hm.matrix_4d_vector(n), hm.matrix_4d_vector(n), hm.megno_construct(n)
    snaps = {}
    for k in range(500):
        Mo.explicit_copy(M)
        M.structured_multiply(t2, p2, 0.2)
        t2.track(p2, 1, 0.2)
        mg.add(M, Mo)
        if k + 1 in (100, 500):
            snaps[k + 1] = mg.get_values()
    assert_bitwise(got[:, 0], snaps[100])
    assert_bitwise(got[:, 1], snaps[500])
    assert np.isfinite(got[:, 1]).any() and np.isnan(got[:, 1]).any()


def test_engine_get_tunes_matches_oracle(gpu):
    # get_tunes(x, px) of the engine (src/dynamic_indicator.cpp:333-362):
    # (FFT tune, Birkhoff tune) of one plane's whole orbit.
    from henon_map_cpp_b200 import henon_map_engine as E

    x, px, y, py = grid(0.3, 3)
    orb = T.orbit(x, px, y, py, O.tables(2000, *TUNES, "sps", epsilon=16.0), 2000, 0.2)
    for i in range(x.size):
        q, p = orb[0][:, i], orb[1][:, i]
        fft, birk = E.get_tunes(q, p)
        np.testing.assert_allclose(birk, T.birkhoff_tune(q, p), rtol=1e-13)
        np.testing.assert_allclose(fft, T.fft_tune(q, p), rtol=1e-10)
    q = orb[0][:, 0].copy()
    q[7] = np.nan
    assert np.all(np.isnan(E.get_tunes(q, orb[1][:, 0])))
    with pytest.raises(RuntimeError, match="same size"):
        E.get_tunes(orb[0][:10, 0], orb[1][:9, 0])


@pytest.mark.parametrize("kick,inverse", [(1e-6, False), (float("nan"), True), (1e-6, True)])
def test_tracker_orbit_tunes_with_kicks_and_inverse(gpu, kick, inverse):
    # birkhoff_tunes / all_tunes accept the reference's kick_module and
    # inverse (src/henon.cu:2890-3078): the orbit is hm_track's (reproducible
    # kicks keyed by kick_seed, particle and table index; backward turns from
    # the particles' steps), then the same tunes.
    x, px, y, py = grid(0.6, 9, px0=0.002)
    n_fwd, n_turns, seed = 900, 600, 4242
    frm, to = [0, 50], [99, 600]
    tabs = O.tables(n_fwd, *TUNES, "sps", epsilon=16.0)
    tr = C.Tracker(n_fwd, *TUNES, "sps", NAN, 16.0, 0)
    p = C.Particles(x, px, y, py)
    p.kick_seed = seed
    start = (x, px, y, py, np.zeros(x.size, np.uint32))
    if inverse:
        tr.track(p, n_fwd, 0.2, 10.0)
        start = O.track(x, px, y, py, start[4], tabs, n_fwd, 0.2, 10.0)
    b, f = C.tracker_orbit_tunes(tr, p, n_turns, 0.2, 10.0, frm, to, True, True,
                                 kick_module=kick, inverse=inverse)
    orb = T.orbit(*start[:4], tabs, n_turns, 0.2, kick_module=kick, seed=seed, inverse=inverse,
                  steps0=start[4])
    got_state = p.state()
    for c in range(4):
        assert_bitwise(got_state[c], orb[c, -1], f"coordinate {c}")
    assert p.global_steps == (n_fwd - n_turns if inverse else n_turns)
    raw = orb
    orb = T.remove_mean(orb)
    want_b = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "birkhoff")
                       for i in range(x.size)])
    want_f = np.array([T.tune_vec(*(orb[c, :, i] for c in range(4)), frm, to, "fft")
                       for i in range(x.size)])
    _close(b, want_b, 1e-13, "birkhoff")
    _close(f, want_f, 1e-10, "fft")
    # through the engine's reference-named methods too
    from henon_map_cpp_b200 import henon_map_engine as E
    et = E.henon_tracker_gpu(n_fwd, *TUNES, "sps", NAN, 16.0, 0)
    ep = E.particles_4d_gpu(x, px, y, py)
    ep.kick_seed = seed
    if inverse:
        et.track(ep, n_fwd, 0.2, 10.0)
    eb = np.asarray(et.birkhoff_tunes(ep, n_turns, 0.2, 10.0, kick, inverse, frm, to))
    want_raw = np.array([T.tune_vec(*(raw[c, :, i] for c in range(4)), frm, to, "birkhoff")
                         for i in range(x.size)])
    _close(eb[:, :2 * len(frm)], want_raw[:, :2 * len(frm)], 1e-13, "engine birkhoff_tunes")


def test_tracker_megno_with_kicks_equals_construct_loop(gpu):
    # megno(kick_module=...) (src/henon.cu:2755-2887 accepts kicks): the
    # Jacobian of each turn at the point before it, then the kicked turn --
    # the per-call loop with hm_track's reproducible kicks, bit for bit.
    x, px, y, py = grid(0.5, 8)
    n, kick, seed = x.size, 1e-7, 99
    t = hm.henon_tracker(400, *TUNES, "sps", np.nan, 16.0, 0)
    p = hm.particles(x, px, y, py)
    p.particles.kick_seed = seed
    got = t.megno(p, 400, 0.2, kick_module=kick, turn_samples=np.array([50, 400]))
    t2 = hm.henon_tracker(400, *TUNES, "sps", np.nan, 16.0, 0)
    p2 = hm.particles(x, px, y, py)
    p2.particles.kick_seed = seed
    M, Mo, mg = hm.matrix_4d_vector(n), hm.matrix_4d_vector(n), hm.megno_construct(n)
    snaps = {}
    for k in range(400):
        Mo.explicit_copy(M)
        M.structured_multiply(t2, p2, 0.2)
        t2.track(p2, 1, 0.2, kick_module=kick)
        mg.add(M, Mo)
        if k + 1 in (50, 400):
            snaps[k + 1] = mg.get_values()
    assert_bitwise(got[:, 0], snaps[50])
    assert_bitwise(got[:, 1], snaps[400])
    assert_bitwise(p.get_x(), p2.get_x())
    # without the kick the values differ (the kick is applied)
    p3 = hm.particles(x, px, y, py)
    plain = t.megno(p3, 400, 0.2, turn_samples=np.array([400]))
    assert not np.array_equal(plain[:, 0], got[:, 1], equal_nan=True)


def _inv_jacobian(x, px, y, py, sx, cx, sy, cy, mu):
    """inverse_tangent_matrix (src/henon.cu:224-249) elementwise, [n][4][4]."""
    u = cx * x - px * sx
    w = cy * y - py * sy
    d2 = u * u - w * w
    gp = (3.0 * mu) * u + 1.0
    gm = (-3.0 * mu) * u - 1.0
    z = np.zeros_like(x)
    m = np.empty((x.size, 4, 4))
    rows = [[np.full_like(x, cx), np.full_like(x, -sx), z, z],
            [(((-3.0 * cx) * mu) * d2 - (2.0 * cx) * u) + sx,
             (cx + ((3.0 * mu) * sx) * d2) + (2.0 * sx) * u,
             ((2.0 * cy) * w) * gp, ((2.0 * sy) * w) * gm],
            [z, z, np.full_like(x, cy), np.full_like(x, -sy)],
            [((2.0 * cx) * w) * gp, ((2.0 * sx) * w) * gm,
             (((3.0 * cy) * mu) * d2 + (2.0 * cy) * u) + sy,
             (cy - ((3.0 * mu) * sy) * d2) - (2.0 * sy) * u]]
    for i in range(4):
        for j in range(4):
            m[:, i, j] = rows[i][j]
    return m


def test_tracker_megno_inverse_matches_oracle(gpu):
    # megno(inverse=True): backward turns from the particles' steps, each
    # with the Jacobian of the backward turn at the point before it; the
    # MEGNO construct's accumulation (src/henon.cu:2253-2284).  Checked
    # against a numpy restatement on the oracle's backward orbit (log10 of
    # numpy against CUDA's: 1e-12).
    x, px, y, py = grid(0.45, 7)
    n, n_fwd, n_back, mu = x.size, 500, 300, 0.2
    t = hm.henon_tracker(n_fwd, *TUNES, "sps", np.nan, 16.0, 0)
    p = hm.particles(x, px, y, py)
    t.track(p, n_fwd, mu)
    got = t.megno(p, n_back, mu, inverse=True, turn_samples=np.array([100, 300]))
    assert p.particles.get_global_steps() == n_fwd - n_back
    sx, cx, sy, cy = O.tables(n_fwd, *TUNES, "sps", epsilon=16.0)
    st = O.track(x, px, y, py, np.zeros(n, np.uint32), (sx, cx, sy, cy), n_fwd, mu, 10.0)
    M = np.tile(np.eye(4), (n, 1, 1))
    old = np.sqrt(np.sum(M.reshape(n, 16) ** 2, axis=1))
    l1 = np.zeros(n)
    l2 = np.zeros(n)
    want = {}
    s = n_fwd
    with np.errstate(all="ignore"):
        for k in range(1, n_back + 1):
            s -= 1
            J = _inv_jacobian(*st[:4], sx[s], cx[s], sy[s], cy[s], mu)
            out = np.zeros_like(M)
            for q in range(4):
                out = out + J[:, :, q][:, :, None] * M[:, q, :][:, None, :]
            M = out
            sq = np.zeros(n)
            for e in range(16):
                sq = sq + M.reshape(n, 16)[:, e] ** 2
            new = np.sqrt(sq)
            lr = np.log10(new / old)
            di = float(k)
            l1 = l1 + lr * di
            l2 = l2 + (1.0 / di) * l1
            if k in (100, 300):
                want[k] = (1.0 / di) * l2
            old = new
            st = O.track(*st, (sx, cx, sy, cy), 1, mu, 10.0, inverse=True)
    for j, k in enumerate((100, 300)):
        a, b = got[:, j], want[k]
        assert np.array_equal(np.isnan(a), np.isnan(b))
        m = ~np.isnan(b)
        np.testing.assert_allclose(a[m], b[m], rtol=1e-12, atol=1e-14)
    assert np.isfinite(got[:, 1]).any()
