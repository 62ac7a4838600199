"""Host logic of bench.py that needs no GPU: each rank's slice of the scan
grid (weak scaling over N ranks) and the GPU naming of the clock sampler."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_rank_slices_tile_the_wide_grid(world):
    # Each of N ranks scans an interleaved side x side slice of a
    # side x (side N) grid on [0, 0.6]^2: together exactly that grid, once.
    side = 16
    pts = []
    for rank in range(world):
        x, px, y, py = bench.grid_slice(side, rank, world)
        assert x.size == side * side
        assert np.all(px == 0) and np.all(py == 0)
        assert x.min() >= 0.0 and x.max() <= 0.6 and y.min() >= 0.0 and y.max() <= 0.6
        pts.append(np.stack([x, y], axis=1))
    allp = np.concatenate(pts)
    xs = np.linspace(0.0, 0.6, side * world)
    ys = np.linspace(0.0, 0.6, side)
    want = np.stack(np.meshgrid(xs, ys), axis=-1).reshape(-1, 2)
    key = lambda a: a[np.lexsort((a[:, 1], a[:, 0]))]  # noqa: E731
    np.testing.assert_array_equal(key(allp), key(want))


def test_clock_sampler_names_the_visible_gpu(monkeypatch):
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES", raising=False)
    assert bench.smi_id(0) == "0"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "3,5")
    assert bench.smi_id(0) == "3" and bench.smi_id(1) == "5"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "GPU-aaaa, GPU-bbbb")
    assert bench.smi_id(1) == "GPU-bbbb"


def test_workload_config_names_the_scan():
    from types import SimpleNamespace

    args = SimpleNamespace(side=1024, turns=100_000, arith="exact", stage_turns=256)
    cfg = bench.workload_config(args, 4)
    assert cfg["particles_per_gpu"] == 1024 * 1024 and cfg["turns"] == 100_000
    assert cfg["parallelism"] == "particle shards x4"


def _bench_json(cmd, env=None):
    import json
    import os
    import subprocess

    out = subprocess.run(cmd, capture_output=True, text=True, timeout=240,
                         env={**os.environ, **(env or {})}, cwd=str(Path(bench.__file__).parent))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_gpus_flag_starts_that_many_ranks():
    # Without torchrun's environment, --gpus 2 re-executes bench.py under
    # torch.distributed.run with two ranks; with no GPU they join over gloo.
    line = _bench_json([sys.executable, "bench.py", "--gpus", "2", "--launch-check"],
                       env={"CUDA_VISIBLE_DEVICES": ""})
    assert line["n_gpus"] == 2 and line["backend"] == "gloo"
    assert sorted(r["rank"] for r in line["ranks"]) == [0, 1]


def test_world_size_must_match_gpus(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "2")
    with pytest.raises(SystemExit, match="WORLD_SIZE=2"):
        bench.check_world(type("A", (), {"gpus": 4})())


def test_cpu_sample_is_fixed():
    # Both the reference arm and the GPU arm's cpu_baseline leg time the
    # same fixed stride of the grid.
    import inspect

    assert bench.CPU_STRIDE == 24
    sig = inspect.signature(bench.reference_cpu_sample)
    assert sig.parameters["stride"].default == bench.CPU_STRIDE
