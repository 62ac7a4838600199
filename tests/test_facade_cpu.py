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


def test_engine_has_every_name_the_reference_package_imports():
    # henon_map_cpp/__init__.py:5-17 imports these from its engine; the
    # module-level functions are those of src/bind.cpp:227-242.
    from henon_map_cpp_b200 import henon_map_engine as E

    for name in ("birkhoff_weights", "henon_tracker", "henon_tracker_gpu",
                 "lyapunov_birkhoff_construct", "lyapunov_birkhoff_construct_multi",
                 "matrix_4d_vector", "matrix_4d_vector_gpu", "megno_birkhoff_construct",
                 "megno_construct", "particles_4d", "particles_4d_gpu", "storage_4d",
                 "storage_4d_gpu", "tune_birkhoff_construct", "vector_4d_gpu",
                 "is_cuda_device_available", "basic_modulation", "sps_modulation",
                 "gaussian_modulation", "uniform_modulation", "get_tunes"):
        assert hasattr(E, name), name
    # The CPU classes exist by name only: this build is the GPU path.
    for cls, args in ((E.particles_4d, ([0.0], [0.0], [0.0], [0.0])),
                      (E.henon_tracker, (10, 0.1, 0.2, "sps", 0.0, 0.0, 0)),
                      (E.matrix_4d_vector, (4,)), (E.storage_4d, (4,))):
        with pytest.raises(NotImplementedError, match="_gpu"):
            cls(*args)
