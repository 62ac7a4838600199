"""The drop-in package on a machine without a GPU: it imports, its host
numerics work, and every GPU class raises instead of falling back to a CPU
implementation."""
from __future__ import annotations

import inspect

import numpy as np
import pytest

from conftest import TUNES, assert_bitwise, golden_npz

hm = pytest.importorskip("henon_map_cpp_b200")


def test_engine_loaded_and_host_numerics():
    from henon_map_cpp_b200 import henon_map_engine as E

    g = golden_npz("ref_modulation.npz")
    assert_bitwise(hm.birkhoff_weights(1000), g["bw1000"])
    assert_bitwise(E.sps_modulation(TUNES[0], 16.0, 0, 4000), g["sps_x_eps16"])
    assert_bitwise(E.basic_modulation(0.31, 0.01, 0.5, 0, 2000), g["basic_x"])
    assert E.gaussian_modulation(0.3, 1e-3, 0, 10).shape == (10,)


def test_reference_signatures_are_kept():
    sig = inspect.signature(hm.henon_tracker.track)
    assert list(sig.parameters)[1:] == ["particles", "n_turns", "mu", "barrier", "kick_module",
                                        "inverse"]
    assert sig.parameters["barrier"].default == 10.0
    sig = inspect.signature(hm.henon_tracker.__init__)
    assert list(sig.parameters)[1:] == ["N", "omega_x", "omega_y", "modulation_kind", "omega_0",
                                        "epsilon", "offset", "force_CPU"]
    sig = inspect.signature(hm.henon_tracker.compute_a_modulation)
    assert list(sig.parameters)[1:5] == ["n_turns", "omega_x", "omega_y", "epsilon"]
    for cls in ("particles", "matrix_4d_vector", "vector_4d", "lyapunov_birkhoff_construct",
                "lyapunov_birkhoff_construct_multi", "megno_construct",
                "megno_birkhoff_construct", "tune_birkhoff_construct", "storage_gpu"):
        assert hasattr(hm, cls)


def test_no_silent_cpu_fallback():
    if hm.gpu_available():
        pytest.skip("a GPU is visible")
    x = np.zeros(3)
    with pytest.raises(RuntimeError, match="CUDA device"):
        hm.particles(x, x, x, x)
    with pytest.raises(RuntimeError, match="CUDA device"):
        hm.henon_tracker(10, 0.1, 0.2, "sps")
    with pytest.raises(NotImplementedError):
        hm.henon_tracker(10, 0.1, 0.2, "sps", force_CPU=True)
