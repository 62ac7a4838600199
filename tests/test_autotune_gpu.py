"""The autotuner picks launch shapes from its search space by timing them;
the shape it leaves behind tracks bit-identically to any other."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import TUNES, assert_bitwise, grid

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")
from henon_map_cpp_b200 import autotune, sweep  # noqa: E402


def _track(x, px, y, py):
    t = C.Tracker(3000, *TUNES, "sps", float("nan"), 16.0, 0)
    p = C.Particles(x, px, y, py)
    t.track(p, 3000, 0.2, 10.0)
    return p.state()


def test_tune_track_returns_a_shape_of_the_space(gpu):
    saved, saved_stage = C.get_track_config(), C.get_track_staging()
    x, px, y, py = grid(0.6, 48)
    before = _track(x, px, y, py)
    try:
        data = autotune._calibration(side=128, turns=2000)
        shape, ms, timings = autotune.tune_track(C.ARITH_EXACT, budget_s=5.0, data=data)
        assert ms > 0 and len(timings) >= 2
        for k, values in autotune.TRACK_SPACE.items():
            assert shape[k] in values
        assert C.get_track_config() == (shape["threads"], shape["per_thread"], shape["chunk0"],
                                        shape["chunk_max"])
        assert C.get_track_staging() == shape["stage_turns"]
        after = _track(x, px, y, py)
        for a, b in zip(before, after):
            assert_bitwise(a, b) if a.dtype == np.float64 else np.testing.assert_array_equal(a, b)
    finally:
        C.set_track_config(*saved)
        C.set_track_staging(saved_stage)


def test_tune_batch_returns_a_configuration(gpu):
    sets, coords = sweep.heterogeneous_sets(seed=3, n_sets=5, n_range=(200, 2000),
                                            turn_range=(100, 2000))
    best, seconds, timings = autotune.tune_batch(sets, coords, budget_s=5.0)
    assert seconds > 0 and len(timings) >= 1
    for k, values in autotune.BATCH_SPACE.items():
        assert best[k] in values
