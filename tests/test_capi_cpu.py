"""The C ABI on a machine without a GPU: the library loads, exports every
symbol that include/*.h declares, and its host-side numerics (modulation
tables, Birkhoff weights) are bit-identical to the reference fixtures."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import REPO, TUNES, assert_bitwise, golden_npz
from oracle import oracle as O

C = pytest.importorskip("henon_map_cpp_b200._capi")


def declared_symbols() -> list[str]:
    names = []
    for h in sorted((REPO / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(hm_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = C.load()
    names = declared_symbols()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declared_symbols():
    names = set(declared_symbols())
    assert names <= set(C._SIGNATURES) | {"hm_cancel_fn"}, sorted(names - set(C._SIGNATURES))


def test_version_and_device_count():
    lib = C.load()
    assert lib.hm_version() >= 10000
    assert lib.hm_device_count() >= 0


def test_host_modulation_bitwise_equal_reference():
    g = golden_npz("ref_modulation.npz")
    out = np.empty(4000)
    C.call("hm_sps_modulation", TUNES[0], 16.0, 0, 4000, C.dptr(out))
    assert_bitwise(out, g["sps_x_eps16"])
    out = np.empty(3000)
    C.call("hm_sps_modulation", TUNES[1], 64.0, 12345, 15345, C.dptr(out))
    assert_bitwise(out, g["sps_y_eps64_off"])
    out = np.empty(2000)
    C.call("hm_basic_modulation", 0.31, 0.01, 0.5, 0, 2000, C.dptr(out))
    assert_bitwise(out, g["basic_x"])
    for n, k in ((10, "bw10"), (1000, "bw1000")):
        w = np.empty(n)
        C.call("hm_birkhoff_weights", n, C.dptr(w))
        assert_bitwise(w, g[k])


def test_pick_a_modulation_kinds():
    wx, wy = np.empty(500), np.empty(500)
    C.call("hm_modulation", b"sps", 500, TUNES[0], TUNES[1], float("nan"), 32.0, 100,
           C.dptr(wx), C.dptr(wy))
    ox, oy = O.omegas(500, *TUNES, "sps", epsilon=32.0, offset=100)
    assert_bitwise(wx, ox)
    assert_bitwise(wy, oy)
    C.call("hm_modulation", b"none", 500, 1.1, 1.3, float("nan"), 0.0, 0, C.dptr(wx), C.dptr(wy))
    assert np.all(wx == 1.1) and np.all(wy == 1.3)
    C.call("hm_modulation", b"gaussian", 500, 0.3, 0.31, float("nan"), 1e-3, 0,
           C.dptr(wx), C.dptr(wy))
    assert abs(np.mean(wx) / (2 * np.pi) - 0.3) < 1e-3
    C.call("hm_modulation", b"uniform", 500, 0.3, 0.31, float("nan"), 0.32, 0,
           C.dptr(wx), C.dptr(wy))
    assert np.all(wx >= 2 * np.pi * 0.3) and np.all(wx <= 2 * np.pi * 0.32)


def test_host_errors_are_status_codes_not_exits():
    o = np.empty(4)
    with pytest.raises(C.HMError, match="Unknown modulation kind") as e:
        C.call("hm_modulation", b"foo", 4, 0.1, 0.2, float("nan"), 0.0, 0, C.dptr(o), C.dptr(o))
    assert e.value.status == C.HM_ERR_UNKNOWN_MODULATION
    with pytest.raises(ValueError):
        C.call("hm_sps_modulation", 0.1, 0.0, 5, 5, C.dptr(o))
    with pytest.raises(ValueError):
        C.call("hm_basic_modulation", 0.1, float("nan"), 0.0, 0, 4, None)
    with pytest.raises(ValueError):
        C.call("hm_modulation", b"basic", 4, 0.1, 0.2, float("nan"), 0.0, 0, C.dptr(o), C.dptr(o))
    with pytest.raises(ValueError):
        C.call("hm_set_track_config", 100, 2, 512, 1024)
    with pytest.raises(ValueError):
        C.call("hm_set_track_config", 128, 3, 512, 1024)
    with pytest.raises(ValueError):
        C.call("hm_tracker_create", 10, 0.1, 0.2, b"sps", 0.0, 0.0, 0, None)


def test_track_config_roundtrip():
    saved = C.get_track_config()
    try:
        C.set_track_config(64, 4, 256, 4096)
        assert C.get_track_config() == (64, 4, 256, 4096)
    finally:
        C.set_track_config(*saved)


def test_track_staging_roundtrip_and_validation():
    saved = C.get_track_staging()
    try:
        for ok in (0, 16, 128, 512):
            C.set_track_staging(ok)
            assert C.get_track_staging() == ok
        for bad in (1, 8, 48, 1024):
            with pytest.raises(C.HMError):
                C.set_track_staging(bad)
    finally:
        C.set_track_staging(saved)


def test_workspace_size_is_linear():
    lib = C.load()
    a = lib.hm_track_workspace_bytes(1000)
    b = lib.hm_track_workspace_bytes(2000)
    assert a > 1000 * 72 and b > a and lib.hm_track_workspace_bytes(0) >= 256


def test_device_calls_fail_cleanly_without_device():
    lib = C.load()
    if lib.hm_device_count() > 0:
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    x = np.zeros(4)
    with pytest.raises(C.HMError):
        C.call("hm_particles_create", C.dptr(x), C.dptr(x), C.dptr(x), C.dptr(x), 4,
               ctypes.byref(h))
    assert not h.value
