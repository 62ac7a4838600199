"""hm_track_device_noalloc: tracking for callers that cannot allocate.

Some hosts of the library may not call cudaMalloc/cudaFree (an application
that reserves all device memory at start-up, a framework whose allocator
owns every device byte, a loop that cannot take cudaFree's device-wide
synchronisation).  This entry point keeps its scratch in a fixed device
array built into the library instead of a caller workspace.  The test runs
it twice in a row through the C ABI and checks each result bit for bit
against hm_track_device (the allocating entry point, given a workspace) on
the same inputs -- exact arithmetic, so the tolerance is zero -- that the
device's free memory is the same before and after the second call (nothing
was allocated), and that a size above the fixed limit is refused.  The file name sorts last so that
pytest collects it after every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import NAN, TUNES, assert_bitwise, grid

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")
MAX_PARTICLES = 131072  # HM_NOALLOC_MAX_PARTICLES in include/henon_b200.h


def _device_state(torch, x, px, y, py):
    coords = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (x, px, y, py)]
    steps = torch.zeros(len(x), dtype=torch.int32, device="cuda")
    return coords, steps


def _host(torch, coords, steps):
    torch.cuda.synchronize()
    return [c.cpu().numpy() for c in coords], steps.cpu().numpy().view(np.uint32)


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    torch = pytest.importorskip("torch")
    # 256 x 256 = 65536 particles (within the fixed scratch), 3000 turns:
    # several chunks, so the survivor lists in the scratch are used.
    x, px, y, py = grid(0.6, 256)
    n, n_turns = x.size, 3000
    trackers = [C.Tracker(n_turns, TUNES[0], TUNES[1], "sps", NAN, eps, 0) for eps in (64.0, 16.0)]
    ws = torch.empty(C.load().hm_track_workspace_bytes(n), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call, (tr, mu) in enumerate(zip(trackers, (0.2, 0.0))):
        ref_c, ref_s = _device_state(torch, x, px, y, py)
        C.call("hm_track_device", *[c.data_ptr() for c in ref_c], ref_s.data_ptr(), n,
               tr.device_tables(), n_turns, 0, n_turns, mu, 10.0, 0, C.ARITH_EXACT,
               ws.data_ptr(), stream)
        got_c, got_s = _device_state(torch, x, px, y, py)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        C.call("hm_track_device_noalloc", *[c.data_ptr() for c in got_c], got_s.data_ptr(), n,
               tr.device_tables(), n_turns, 0, n_turns, mu, 10.0, 0, C.ARITH_EXACT, stream)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            # The first call did the per-device set-up; the second takes no
            # device memory at all.
            assert free_after == free_before, (free_before, free_after)
        want, want_steps = _host(torch, ref_c, ref_s)
        have, have_steps = _host(torch, got_c, got_s)
        np.testing.assert_array_equal(have_steps, want_steps, err_msg=f"call {call}")
        for a, b in zip(have, want):
            assert_bitwise(a, b, f"call {call}")
        assert 0 < np.sum(want_steps == n_turns) < n


def test_noalloc_refuses_sizes_beyond_its_scratch(gpu):
    torch = pytest.importorskip("torch")
    n = MAX_PARTICLES + 1
    coords = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    tr = C.Tracker(10, TUNES[0], TUNES[1], "sps", NAN, 0.0, 0)
    with pytest.raises(ValueError, match="fixed scratch"):
        C.call("hm_track_device_noalloc", *[c.data_ptr() for c in coords], steps.data_ptr(), n,
               tr.device_tables(), 10, 0, 10, 0.0, 10.0, 0, C.ARITH_EXACT, None)
