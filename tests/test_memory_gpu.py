"""Device memory of particle sets: initial conditions kept on the device,
host mirrors built on first use, and buffers reused from the library's pool.

The reference keeps x0..py0, valid, ghost, idx and idx_base on the host
(particles_4d, src/henon.cu:699-735); here they live on the device and are
mirrored to the host only for add_ghost and the tangent matrices.  Every
path must give the results the eager host copies gave.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, grid

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")


def test_create_sets_default_metadata(gpu):
    x, px, y, py = grid(0.5, 33)  # 1089 particles: not a multiple of the block
    p = C.Particles(x, px, y, py)
    n = x.size
    np.testing.assert_array_equal(p.get(C.FIELD_STEPS), 0)
    np.testing.assert_array_equal(p.get(C.FIELD_VALID), 1)
    np.testing.assert_array_equal(p.get(C.FIELD_GHOST), 0)
    np.testing.assert_array_equal(p.get(C.FIELD_IDX), np.arange(n, dtype=np.uint64))
    np.testing.assert_array_equal(p.get(C.FIELD_IDX_BASE), np.arange(n, dtype=np.uint64))
    for f, a in zip((C.FIELD_X, C.FIELD_PX, C.FIELD_Y, C.FIELD_PY), (x, px, y, py)):
        assert_bitwise(p.get(f), a)


def test_reset_restores_initial_conditions_from_device(gpu):
    x, px, y, py = grid(0.6, 24)
    t = C.Tracker(3000, TUNES[0], TUNES[1], "sps", NAN, 64.0, 0)
    p = C.Particles(x, px, y, py)
    t.track(p, 3000, 0.2, 10.0)
    assert np.isnan(p.get(C.FIELD_X)).any()  # some particles were lost
    p.reset()
    for f, a in zip((C.FIELD_X, C.FIELD_PX, C.FIELD_Y, C.FIELD_PY), (x, px, y, py)):
        assert_bitwise(p.get(f), a)
    np.testing.assert_array_equal(p.get(C.FIELD_STEPS), 0)
    np.testing.assert_array_equal(p.get(C.FIELD_VALID), 1)


def test_ghosts_after_tracking_start_from_initial_conditions(gpu):
    # add_ghost builds its host mirror after the device state has moved:
    # the ghosts and the restarted base particles must come from x0, not
    # from the tracked coordinates.
    x, px, y, py = grid(0.3, 8)
    n = x.size
    t = C.Tracker(1000, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)  # add_ghost keeps global_steps
    p = C.Particles(x, px, y, py)
    t.track(p, 500, 0.0, 10.0)
    C.call("hm_particles_add_ghost", p.h, 1e-6, b"x")
    got_x = p.get(C.FIELD_X)
    assert got_x.size == 2 * n
    assert_bitwise(got_x[:n], x)
    assert_bitwise(got_x[n:], x + 1e-6)
    assert_bitwise(p.get(C.FIELD_PX), np.concatenate([px, px]))
    np.testing.assert_array_equal(p.get(C.FIELD_GHOST), np.repeat([0, 1], n))
    np.testing.assert_array_equal(p.get(C.FIELD_IDX_BASE),
                                  np.concatenate([np.arange(n), np.arange(n)]).astype(np.uint64))
    np.testing.assert_array_equal(p.get(C.FIELD_STEPS), 0)
    # A reset after add_ghost restores the whole extended set.
    t.track(p, 100, 0.0, 10.0)
    p.reset()
    assert_bitwise(p.get(C.FIELD_X), np.concatenate([x, x + 1e-6]))


def test_pool_reuse_is_bit_identical_and_trim_keeps_live_buffers(gpu):
    x, px, y, py = grid(0.6, 64)
    t = C.Tracker(4000, TUNES[0], TUNES[1], "sps", NAN, 16.0, 0)

    def run():
        p = C.Particles(x, px, y, py)
        t.track(p, 4000, 0.2, 10.0)
        return p.state()

    first = run()  # its buffers go back to the pool ...
    again = run()  # ... and are handed out again here
    for a, b in zip(first, again):
        assert_bitwise(a, b) if a.dtype == np.float64 else np.testing.assert_array_equal(a, b)
    live = C.Particles(x, px, y, py)
    C.release_cached_memory()  # trims free blocks only
    for f, a in zip((C.FIELD_X, C.FIELD_PX, C.FIELD_Y, C.FIELD_PY), (x, px, y, py)):
        assert_bitwise(live.get(f), a)
    t.track(live, 4000, 0.2, 10.0)
    for a, b in zip(first, live.state()):
        assert_bitwise(a, b) if a.dtype == np.float64 else np.testing.assert_array_equal(a, b)
    C.release_cached_memory()
