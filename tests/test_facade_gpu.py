"""The drop-in Python API (henon_map_cpp_b200, mirroring henon_map_cpp)
driven the way the reference's notebooks drive it, checked against their
recorded answers, the oracle and the reference's own GPU engine."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, golden_json, grid
from oracle import oracle as O

pytestmark = pytest.mark.gpu

hm = pytest.importorskip("henon_map_cpp_b200")


def test_construct_notebook_flow(gpu):
    # tests/test_construct.ipynb, in the order its cells were executed.
    nb = golden_json("notebook_values.json")
    m1, m2 = hm.matrix_4d_vector(3), hm.matrix_4d_vector(3)
    t = hm.henon_tracker(1000, 0.168, 0.201, "sps")
    pp = np.array([0.1, 0.1, 0.1])
    p = hm.particles(pp, np.zeros(3), pp, np.zeros(3))
    m1.set_with_tracker(t, p, 0.0)
    t.track(p, 1, 0.0)
    m2.set_with_tracker(t, p, 0.0)
    np.testing.assert_allclose(m1.get_matrix()[2], nb["tangent_matrix_x0"]["matrix"], rtol=1e-7,
                               atol=1e-8)
    np.testing.assert_allclose(m2.get_matrix()[0], nb["tangent_matrix_x1"]["matrix"], rtol=1e-7,
                               atol=1e-8)
    np.testing.assert_allclose(p.get_x(), nb["x_after_one_turn"]["value"], rtol=1e-7)
    megno = hm.megno_construct(3)
    np.testing.assert_array_equal(megno.get_values(), 0.0)
    megno.add(m2, m1)
    want = np.log10(np.linalg.norm(m2.get_matrix()[0]) / np.linalg.norm(m1.get_matrix()[0]))
    np.testing.assert_allclose(megno.get_values(), want, rtol=1e-13)
    v = hm.vector_4d(np.array([[1.0, 1.0, 0.0, 0.0] for _ in range(3)]))
    construct = hm.lyapunov_birkhoff_construct_multi(3, [5, 10, 15])
    lw = nb["lyapunov_multi_windows"]
    for tag in ("5", "10", "15"):
        for _ in range(5):
            construct.add(v)
        np.testing.assert_allclose(construct.get_values_raw()[:, 0], lw[f"raw_after_{tag}"],
                                   rtol=1e-7, atol=5e-9)
        np.testing.assert_allclose(construct.get_values_b()[:, 0], lw[f"b_after_{tag}"],
                                   rtol=1e-7, atol=5e-9)
    c = hm.lyapunov_birkhoff_construct(3, 10)
    c.change_weights(10)
    np.testing.assert_allclose(c.get_weights(), nb["birkhoff_weights_10"]["value"], rtol=1e-7,
                               atol=1e-12)
    v.set_vectors(np.array([1.0, 0.0, 0.0, 0.0]))
    v.multiply(m1)
    vm = nb["vector_multiply_normalize"]
    np.testing.assert_allclose(v.get_vectors()[0], vm["multiplied"], rtol=1e-7)
    v.normalize()
    np.testing.assert_allclose(v.get_vectors()[1], vm["normalized"], rtol=1e-7)
    storage = hm.storage_gpu(3, 2)
    storage.store(p)
    t.track(p, 1, 0.0)
    storage.store(p)
    assert storage.get_x().shape == (2, 3)
    assert_bitwise(storage.get_x()[1], p.get_x())


def test_ghost_notebook_flow_and_reference_rng(gpu):
    # tests/test_new_standard.ipynb cells 44-54.
    x = np.ones(3)
    p = hm.particles(x, x.copy(), x.copy(), x.copy())
    for d in ("x", "px", "y", "py", "random"):
        p.add_ghost(1e-4, d)
    np.testing.assert_allclose(p.get_displacement_module(), 1e-4, rtol=1e-9)
    d = p.get_displacement_direction()
    assert d.shape == (4, 3, 5)
    np.testing.assert_allclose(d[:, :, 0], [[1, 1, 1], [0, 0, 0], [0, 0, 0], [0, 0, 0]], atol=1e-9)
    want_random = [[-0.64201979, -0.02533011, 0.21874217],
                   [0.73799688, -0.12804619, -0.80929451],
                   [0.18792332, -0.98280347, 0.06593186],
                   [0.08863419, 0.13061355, -0.54115362]]
    np.testing.assert_allclose(d[:, :, 4], want_random, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(np.sum(d[:, :, 1] ** 2, axis=0), 1.0, rtol=1e-12)
    p.renormalize(1.0)
    np.testing.assert_allclose(p.get_displacement_module(), 1.0, rtol=1e-12)
    R = O.reference_module("fmad_off")
    if R is not None:
        rp = R.particles_4d_gpu(x, x, x, x)
        for dd in ("x", "px", "y", "py", "random"):
            rp.add_ghost(1e-4, dd)
        rp.renormalize(1.0)
        assert_bitwise(p.get_x(), np.asarray(rp.get_x()))
        assert_bitwise(p.get_py(), np.asarray(rp.get_py()))
        assert_bitwise(p.get_displacement_direction(), np.asarray(rp.get_displacement_direction()))
        assert_bitwise(p.get_displacement_module(), np.asarray(rp.get_displacement_module()))


def test_ghost_lyapunov_loop_matches_reference_gpu(gpu):
    # The displacement Lyapunov loop of tests/test_new_standard.ipynb:477-479.
    v = np.linspace(0, 0.5, 6)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)
    p = hm.particles(x, z, y, z)
    p.add_ghost(1e-10, "x")
    t = hm.henon_tracker(1000, 0.168, 0.201, "sps", np.nan, 64.0, 0)
    lyap = np.zeros(x.size)
    for _ in range(50):
        t.track(p, 10, 0.0)
        lyap += np.log(p.get_displacement_module().flatten() / 1e-10)
        p.renormalize(1e-10)
    R = O.reference_module("fmad_off")
    if R is None:
        pytest.skip("reference build absent")
    rp = R.particles_4d_gpu(x, z, y, z)
    rp.add_ghost(1e-10, "x")
    rt = R.henon_tracker_gpu(1000, 0.168, 0.201, "sps", NAN, 64.0, 0)
    rl = np.zeros(x.size)
    for _ in range(50):
        rt.track(rp, 10, 0.0, 10.0)
        rl += np.log(np.asarray(rp.get_displacement_module()).flatten() / 1e-10)
        rp.renormalize(1e-10)
    assert_bitwise(lyap, rl)
    np.testing.assert_array_equal(p.get_steps(), np.asarray(rp.get_steps()))


def test_tracker_facade_semantics(gpu):
    x, px, y, py = grid(0.6, 20)
    t = hm.henon_tracker(2001, *TUNES, "sps", np.nan, 16.0, 0)
    p = hm.particles(x, px, y, py)
    t.track(p, 2000, 0.2)  # facade default barrier = 10.0
    want = O.track(x, px, y, py, np.zeros(x.size, np.uint32),
                   O.tables(2000, *TUNES, "sps", epsilon=16.0), 2000, 0.2, 10.0)
    np.testing.assert_array_equal(p.get_steps(), want[4])
    assert_bitwise(p.get_x(), want[0])
    with pytest.raises(RuntimeError, match="The number of turns is too large."):
        t.track(p, 2, 0.2)
    with pytest.raises(RuntimeError, match="Unknown modulation kind"):
        hm.henon_tracker(10, 0.1, 0.2, "nope")
    with pytest.raises(NotImplementedError):
        hm.particles(x, px, y, py, force_CPU=True)
    with pytest.raises(TypeError):
        hm.particles(list(x), px, y, py)
    tm = t.get_tangent_matrix(p, 0.2)
    assert tm.shape == (x.size, 4, 4)
    lost = ~np.isfinite(p.get_x())
    assert lost.any()
    # entries that depend on x, y are NaN for lost particles; sin/cos stay
    assert np.isnan(tm[lost][:, :, 0]).all() and np.isfinite(tm[lost][:, 0, 1]).all()
    sx, cx, sy, cy = O.tables(2001, *TUNES, "sps", epsilon=16.0)
    live = np.flatnonzero(~lost)[:5]
    for i in live:
        want = O.tangent_matrix(p.get_x()[i], 0.0, p.get_y()[i], 0.0, sx[2000], cx[2000],
                                sy[2000], cy[2000], 0.2)
        assert_bitwise(tm[i], want)
    np.testing.assert_allclose(p.get_radius_mean(), np.nanmean(p.get_radius()), rtol=1e-12)
    np.testing.assert_allclose(p.get_angle_x_std(), np.nanstd(p.get_angle_x()), rtol=1e-10)


def test_track_indicators_through_facade(gpu):
    x, px, y, py = grid(0.5, 8)
    n = x.size
    t = hm.henon_tracker(301, *TUNES, "sps", np.nan, 16.0, 0)
    p = hm.particles(x, px, y, py)
    M = hm.matrix_4d_vector(n)
    Mo = hm.matrix_4d_vector(n)
    mg = hm.megno_construct(n)
    tu = hm.tune_birkhoff_construct(n, [50, 100])
    tu.first_add(p)
    snaps = t.track_indicators(p, 300, 0.0, matrix=M, matrix_old=Mo, megno=mg, tune=tu,
                               megno_sample_turns=[10, 300])
    assert snaps.shape == (2, n)
    assert_bitwise(snaps[1], mg.get_values())
    # the same loop, call by call
    t2 = hm.henon_tracker(301, *TUNES, "sps", np.nan, 16.0, 0)
    p2 = hm.particles(x, px, y, py)
    M2, Mo2, mg2 = hm.matrix_4d_vector(n), hm.matrix_4d_vector(n), hm.megno_construct(n)
    tu2 = hm.tune_birkhoff_construct(n, [50, 100])
    tu2.first_add(p2)
    for _ in range(300):
        Mo2.explicit_copy(M2)
        t2.track(p2, 1, 0.0)
        M2.structured_multiply(t2, p2, 0.0)
        mg2.add(M2, Mo2)
        tu2.add(p2)
    assert_bitwise(mg.get_values(), mg2.get_values())
    assert_bitwise(np.asarray(tu.get_tune2_y()), np.asarray(tu2.get_tune2_y()))
    assert_bitwise(M.get_matrix(), M2.get_matrix())


def test_kicked_track_through_facade(gpu):
    x, px, y, py = grid(0.4, 12)
    p = hm.particles(x, px, y, py)
    assert p.kick_seed == 0
    p.kick_seed = 2024
    t = hm.henon_tracker(800, *TUNES, "sps", np.nan, 16.0, 0)
    t.track(p, 800, 0.2, kick_module=5e-4)
    want = O.track_kicked(x, px, y, py, np.zeros(x.size, np.uint32),
                          O.tables(800, *TUNES, "sps", epsilon=16.0), 800, 0.2, 10.0, 5e-4, 2024)
    np.testing.assert_array_equal(p.get_steps(), want[4])
    assert_bitwise(p.get_x(), want[0])
    assert_bitwise(p.get_py(), want[3])


@pytest.mark.parametrize("every,n_steps,mu,dirs", [(10, 60, 0.2, ("x", "y")),
                                                    (7, 700, 0.0, ("x", "py", "random")),
                                                    (1, 300, 0.2, ("px",))])
def test_fused_ghost_lyapunov_equals_the_loop(gpu, every, n_steps, mu, dirs):
    # track_ghost_lyapunov against the notebook loop run on the reference's
    # own GPU classes (or, without the reference build, on ours): the same
    # coordinates and steps bit for bit -- lost bases, lost ghosts and ghosts
    # of lost bases included -- and the same log sums to 1e-13.  700 steps
    # of 7 turns cross the fused call's launch boundaries.
    v = np.linspace(0, 0.6, 14)
    xx, yy = np.meshgrid(v, v)
    x, y = xx.ravel(), yy.ravel()
    z = np.zeros_like(x)
    module, eps = 1e-10, 64.0
    turns = every * n_steps
    p = hm.particles(x, z, y, z)
    for d in dirs:
        p.add_ghost(module, d)
    t = hm.henon_tracker(turns + 1, 0.168, 0.201, "sps", np.nan, eps, 0)
    got = t.track_ghost_lyapunov(p, n_steps, every, mu, module)
    assert got.shape == (x.size, len(dirs))

    R = O.reference_module("fmad_off")
    if R is not None:
        rp = R.particles_4d_gpu(x, z, y, z)
        for d in dirs:
            rp.add_ghost(module, d)
        rt = R.henon_tracker_gpu(turns + 1, 0.168, 0.201, "sps", NAN, eps, 0)
        step = lambda: rt.track(rp, every, mu, 10.0)  # noqa: E731
    else:
        rp = hm.particles(x, z, y, z)
        for d in dirs:
            rp.add_ghost(module, d)
        rt = hm.henon_tracker(turns + 1, 0.168, 0.201, "sps", np.nan, eps, 0)
        step = lambda: rt.track(rp, every, mu)  # noqa: E731
    want = np.zeros((x.size, len(dirs)))
    for _ in range(n_steps):
        step()
        want += np.log(np.asarray(rp.get_displacement_module()).reshape(x.size, len(dirs))
                       / module)
        rp.renormalize(module)
    for name in ("get_x", "get_px", "get_y", "get_py"):
        assert_bitwise(getattr(p, name)(), np.asarray(getattr(rp, name)()), name)
    np.testing.assert_array_equal(p.get_steps(), np.asarray(rp.get_steps()))
    assert np.array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    np.testing.assert_allclose(got[m], want[m], rtol=1e-13, atol=1e-12)
    steps = p.get_steps()
    assert np.any(steps[:x.size] < turns) and np.any(steps[:x.size] == turns)
    assert p.particles.get_global_steps() == turns
