"""Tune estimates on the GPU (Birkhoff and FFT over orbit windows, the
tracker's whole-orbit tunes and MEGNO, storage tunes) against the oracle
(oracle/tunes.py) and the values recorded in the reference's notebooks."""
from __future__ import annotations

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
