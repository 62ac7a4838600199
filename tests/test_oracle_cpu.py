"""Pins the CPU oracle before anything is checked against it.

1. Against the golden fixtures made by running the reference itself
   (tests/golden/ref_*.npz, tests/golden/make_golden.py): bit for bit.
2. Against known answers recorded in the reference's notebooks
   (tests/golden/notebook_values.json): to their printed precision.
3. Against the reference build live when oracle/_ref/ is present.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, golden_json, golden_npz, grid
from oracle import oracle as O

CASES = ["c1_like", "eps16_mu02", "eps64_mu02", "eps1_mu0", "eps32_mum05"]


@pytest.mark.parametrize("case", CASES)
def test_oracle_track_equals_reference_fixture(case):
    g = golden_npz(f"ref_track_{case}.npz")
    nt = int(g["n_turns"])
    tabs = O.tables(nt, *g["tunes"], "sps", epsilon=float(g["epsilon"]))
    got = O.track(g["x0"], g["px0"], g["y0"], g["py0"], np.zeros(g["x0"].size, np.uint32),
                  tabs, nt, float(g["mu"]), 10.0)
    for a, k in zip(got[:4], ("x", "px", "y", "py")):
        assert_bitwise(a, g[k], k)
    np.testing.assert_array_equal(got[4], g["steps"])


def test_oracle_reverse_equals_reference_fixture():
    g = golden_npz("ref_reverse.npz")
    tabs = O.tables(1000, *g["tunes"], "sps", epsilon=64.0)
    f = O.track(g["x0"], g["px0"], g["y0"], g["py0"], np.zeros(200, np.uint32), tabs, 1000,
                0.1, 10.0)
    for a, k in zip(f, ("fx", "fpx", "fy", "fpy", "fsteps")):
        assert_bitwise(a, g[k], k) if a.dtype == np.float64 else np.testing.assert_array_equal(a, g[k])
    b = O.track(*f, tabs, 1000, 0.1, 10.0, inverse=True)
    for a, k in zip(b, ("bx", "bpx", "by", "bpy", "bsteps")):
        assert_bitwise(a, g[k], k) if a.dtype == np.float64 else np.testing.assert_array_equal(a, g[k])


def test_oracle_modulation_equals_reference_fixture():
    g = golden_npz("ref_modulation.npz")
    assert_bitwise(O.sps_modulation(TUNES[0], 16.0, 0, 4000), g["sps_x_eps16"])
    assert_bitwise(O.sps_modulation(TUNES[1], 64.0, 12345, 12345 + 3000), g["sps_y_eps64_off"])
    assert_bitwise(O.basic_modulation(0.31, 0.01, 0.5, 0, 2000), g["basic_x"])
    assert_bitwise(O.birkhoff_weights(10), g["bw10"])
    assert_bitwise(O.birkhoff_weights(1000), g["bw1000"])


def test_oracle_notebook_known_answers():
    nb = golden_json("notebook_values.json")
    sx, cx, sy, cy = O.tables(1000, *TUNES, "sps", epsilon=0.0)
    m0 = O.tangent_matrix(0.1, 0.0, 0.1, 0.0, sx[0], cx[0], sy[0], cy[0], 0.0)
    np.testing.assert_allclose(m0, nb["tangent_matrix_x0"]["matrix"], rtol=1e-7, atol=1e-8)
    x1 = O.track([0.1], [0.0], [0.1], [0.0], [0], (sx, cx, sy, cy), 1, 0.0, 10.0)
    np.testing.assert_allclose(x1[0][0], nb["x_after_one_turn"]["value"], rtol=1e-7)
    m1 = O.tangent_matrix(x1[0][0], x1[1][0], x1[2][0], x1[3][0], sx[1], cx[1], sy[1], cy[1], 0.0)
    np.testing.assert_allclose(m1, nb["tangent_matrix_x1"]["matrix"], rtol=1e-7, atol=1e-8)
    np.testing.assert_allclose(O.birkhoff_weights(10), nb["birkhoff_weights_10"]["value"],
                               rtol=1e-7, atol=1e-12)
    v = m0 @ np.array([1.0, 0.0, 0.0, 0.0])
    vm = nb["vector_multiply_normalize"]
    np.testing.assert_allclose(v, vm["multiplied"], rtol=1e-7)
    np.testing.assert_allclose(np.log(np.linalg.norm(v)), vm["log_norm"], rtol=1e-12)


def test_indicator_oracle_pinned():
    from oracle import indicators as I

    nb = golden_json("notebook_values.json")
    sx, cx, sy, cy = O.tables(1001, *TUNES, "sps", epsilon=0.0)
    m = I.tangent_matrix([0.1], [0.1], sx[0], cx[0], sy[0], cy[0], 0.0)[0]
    np.testing.assert_allclose(m, nb["tangent_matrix_x0"]["matrix"], rtol=1e-7, atol=1e-8)
    rng = np.random.default_rng(3)
    for mu in (0.0, 0.3, -0.7):
        xs, ys = rng.normal(size=5), rng.normal(size=5)
        mats = I.tangent_matrix(xs, ys, sx[7], cx[7], sy[7], cy[7], mu)
        for k in range(5):
            c = O.tangent_matrix(xs[k], 0.0, ys[k], 0.0, sx[7], cx[7], sy[7], cy[7], mu)
            assert_bitwise(mats[k], c)
            assert_bitwise(I.matmul(mats[k:k + 1], mats[k:k + 1])[0], O.matmul4(c, c))
    # Lyapunov windows of the notebook: v = (1, 1, 0, 0) every turn.
    lw = nb["lyapunov_multi_windows"]
    nv = I.norm(np.array([[1.0, 1.0, 0.0, 0.0]]))[0]
    for tag, k in (("5", 5), ("10", 10), ("15", 15)):
        raw = [sum(np.log(nv) / L for i in range(min(k, L))) for L in (5, 10, 15)]
        bw = [sum(np.log(nv) * O.birkhoff_weights(L)[i] for i in range(min(k, L)))
              for L in (5, 10, 15)]
        np.testing.assert_allclose(raw, lw[f"raw_after_{tag}"], rtol=1e-7, atol=5e-9)
        np.testing.assert_allclose(bw, lw[f"b_after_{tag}"], rtol=1e-7, atol=5e-9)
    # The loop runs and loses the large-amplitude particles.
    x, px, y, py = grid(0.6, 8)
    L = I.ConstructLoop(x, px, y, py, (sx, cx, sy, cy), 0.0, 10.0, [1, 0, 0, 0], [10, 50],
                        [10, 50], [20, 40]).run(100)
    assert np.isnan(L.m_l3).any() and np.isfinite(L.m_l3).any()


def test_tune_oracle_reproduces_notebook_values():
    from oracle import tunes as T

    nb = golden_json("notebook_values.json")["tunes_0p1_eps0"]
    tabs = O.tables(10000, *TUNES, "sps", epsilon=0.0)
    orb = T.remove_mean(T.orbit([0.1], [0.0], [0.1], [0.0], tabs, 10000, 0.0, 10.0))
    x, px, y, py = (orb[c, :, 0] for c in range(4))

    def window(key):
        a, b = (int(v) for v in key.split("-"))
        return slice(a, b + 1)

    for key, v in nb["birkhoff_x"].items():
        s = window(key)
        assert T.birkhoff_tune(x[s], px[s]) == v, key
    for key, v in nb["fft_x"].items():
        s = window(key)
        assert T.fft_tune(x[s], px[s]) == v, key
    for key, v in nb["fft_y"].items():
        s = window(key)
        assert T.fft_tune(y[s], py[s]) == v, key
    for key, v in nb["birkhoff_y_approx"].items():
        s = window(key)
        assert abs(T.birkhoff_tune(y[s], py[s]) - v) < 1e-10, key
    # windows + full orbit layout, NaN handling
    b = T.tune_vec(x, px, y, py, [0, 500], [500, 1000], "birkhoff")
    assert len(b) == 6 and b[0] == nb["birkhoff_x"]["0-500"]
    xn = x.copy()
    xn[700] = np.nan
    b = T.tune_vec(xn, px, y, py, [0, 500], [500, 1000], "fft")
    assert np.isnan(b[2]) and np.isnan(b[3]) and not np.isnan(b[0]) and np.isnan(b[4])


@pytest.mark.skipif(O.reference_module("fmad_off") is None, reason="reference build absent")
@pytest.mark.parametrize("eps,mu,nt", [(0.0, 0.0, 1500), (16.0, 0.2, 1500), (64.0, -0.3, 1200)])
def test_oracle_equals_reference_build_live(eps, mu, nt):
    R = O.reference_module("fmad_off")
    x, px, y, py = grid(0.55, 20, px0=0.001)
    t = R.henon_tracker(nt, *TUNES, "sps", NAN, eps, 0)
    p = R.particles_4d(x, px, y, py)
    t.track(p, nt, mu, 10.0)
    want = [np.asarray(p.get_x()), np.asarray(p.get_px()), np.asarray(p.get_y()),
            np.asarray(p.get_py()), np.asarray(p.get_steps())]
    got = O.track(x, px, y, py, np.zeros(x.size, np.uint32),
                  O.tables(nt, *TUNES, "sps", epsilon=eps), nt, mu, 10.0)
    for a, b in zip(got[:4], want[:4]):
        assert_bitwise(a, b)
    np.testing.assert_array_equal(got[4], want[4])


def test_philox_known_answers():
    # Philox4x32-10 known-answer vectors published with the generator
    # (Random123 kat_vectors: counter, key -> output).
    kat = [([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
           ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
           ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
            [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1])]
    for ctr, key, want in kat:
        np.testing.assert_array_equal(O.philox4x32_10(ctr, key), np.array(want, np.uint32))


def test_kick_directions_are_unit_and_isotropic():
    d = np.array([O.kick_direction(99, i, t) for i in range(2000) for t in (0, 1, 12345)])
    np.testing.assert_allclose(np.einsum("ij,ij->i", d, d), 1.0, rtol=0, atol=1e-15)
    assert np.abs(d.mean(axis=0)).max() < 0.02           # 6000 samples: sd 0.0065
    cov = d.T @ d / len(d)
    np.testing.assert_allclose(cov, np.eye(4) / 4, atol=0.015)
    # a function of (seed, particle, turn) only
    np.testing.assert_array_equal(O.kick_direction(99, 7, 3), O.kick_direction(99, 7, 3))
    assert not np.array_equal(O.kick_direction(99, 7, 3), O.kick_direction(98, 7, 3))
    assert not np.array_equal(O.kick_direction(99, 7, 3), O.kick_direction(99, 7, 4))


def test_kicked_oracle_moves_each_turn_by_the_kick():
    # With the rotation turned into the identity (omega = 0 tables) and a
    # particle at the origin, one kicked turn leaves kick * direction plus
    # the sextupole terms of that small displacement.
    tabs = (np.zeros(3), np.ones(3), np.zeros(3), np.ones(3))
    z = np.zeros(1)
    got = O.track_kicked(z, z, z, z, np.zeros(1, np.uint32), tabs, 1, 0.0, 10.0, 1e-6, 5)
    d = O.kick_direction(5, 0, 0)
    assert got[4][0] == 1
    np.testing.assert_allclose([got[0][0], got[2][0]], 1e-6 * d[[0, 2]], rtol=0, atol=1e-20)
    np.testing.assert_allclose([got[1][0], got[3][0]], 1e-6 * d[[1, 3]], rtol=0, atol=1e-11)
