"""Host-side multi-GPU logic on CPU: shard arithmetic, set assignment and
the collectives, run as two gloo ranks (the GPU data path has no
collective inside the turn loop, so this is all of it)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from henon_map_cpp_b200 import sharding as S
from henon_map_cpp_b200 import sweep


def test_particle_shards_cover_exactly():
    for n in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            sl = [S.particle_shard(n, r, world) for r in range(world)]
            assert sl[0].start == 0 and sl[-1].stop == n
            assert all(a.stop == b.start for a, b in zip(sl, sl[1:]))
            sizes = [s.stop - s.start for s in sl]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        S.particle_shard(10, 2, 2)


def test_interleaved_grid_partitions_the_global_grid():
    side, world = 16, 4
    parts = [S.interleaved_grid(side, r, world) for r in range(world)]
    xs = np.sort(np.concatenate([p[0] for p in parts]))
    ys = np.sort(np.concatenate([p[2] for p in parts]))
    gx, gy = np.meshgrid(np.linspace(0, 0.6, side * world), np.linspace(0, 0.6, side))
    np.testing.assert_array_equal(xs, np.sort(gx.ravel()))
    np.testing.assert_array_equal(ys, np.sort(gy.ravel()))
    one = S.interleaved_grid(side, 0, 1)
    gx1, gy1 = np.meshgrid(np.linspace(0, 0.6, side), np.linspace(0, 0.6, side))
    np.testing.assert_array_equal(one[0], gx1.ravel())


def test_lpt_assignment_balances():
    sets, _ = sweep.heterogeneous_sets(seed=20261203, n_sets=64)
    for world in (1, 2, 4, 8):
        parts = S.assign_sets(sets, world)
        assert sorted(k for p in parts for k in p) == list(range(64))
        loads = [sum(sets[k]["n_particles"] * sets[k]["n_turns"] for k in p) for p in parts]
        biggest = max(s["n_particles"] * s["n_turns"] for s in sets)
        assert max(loads) - min(loads) <= biggest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r holds particles with losses 1..r+2 and r+1 survivors
        loss_sum = float(sum(range(1, rank + 3)))
        count = rank + 1
        g = np.full(4, float(rank + 1))
        mean, gmean = S.reduce_loss(loss_sum, count, g)
        steps = S.gather_steps(np.arange(rank * 10, rank * 10 + 3 + rank))
        out[rank] = (mean, gmean.tolist(), steps.tolist())
    finally:
        dist.destroy_process_group()


def test_collectives_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    total = (1 + 2) + (1 + 2 + 3)
    for r in range(2):
        mean, gmean, steps = res[r]
        assert mean == pytest.approx(total / 3)
        assert gmean == pytest.approx([(1 + 2) / 3] * 4)
        assert steps == [0, 1, 2, 10, 11, 12, 13]


def test_shard_sets_cut_the_concatenated_points():
    sets, coords = sweep.heterogeneous_sets(seed=7, n_sets=9, n_range=(3, 40),
                                            turn_range=(10, 1000))
    offsets = np.concatenate([[0], np.cumsum([s["n_particles"] for s in sets])])
    seen = []
    for world in (1, 2, 3):
        seen = []
        for rank in range(world):
            mine, sub, sub_coords = sweep.shard_sets(sets, coords, rank, world)
            seen += mine
            assert [sets[k] for k in mine] == sub
            want = [np.concatenate([c[offsets[k]:offsets[k + 1]] for k in mine]) for c in coords]
            for a, b in zip(sub_coords, want):
                np.testing.assert_array_equal(a, b)
        assert sorted(seen) == list(range(len(sets)))


def _sweep_worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sets, coords = sweep.heterogeneous_sets(seed=7, n_sets=9, n_range=(3, 40),
                                                turn_range=(10, 1000))
        ran = []

        def fake_local(sub, sub_coords, *args):
            # Stands in for the device batch: steps = the set's turn budget
            # minus its first x coordinate's rank in the set, so results are
            # tied to both the set and its points.
            ran.extend(s["n_turns"] for s in sub)
            out_l, o = [], 0
            for s in sub:
                n = s["n_particles"]
                out_l.append({"steps": np.full(n, s["n_turns"], np.uint32),
                              "x": np.asarray(sub_coords[0][o:o + n])})
                o += n
            return out_l

        sweep._local_sweep = fake_local
        res = sweep.run_sweep(sets, coords)
        out[rank] = ([r["steps"].tolist() for r in res], [r["x"].tolist() for r in res],
                     sorted(ran))
    finally:
        dist.destroy_process_group()


def test_sweep_spreads_sets_over_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_sweep_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    sets, coords = sweep.heterogeneous_sets(seed=7, n_sets=9, n_range=(3, 40),
                                            turn_range=(10, 1000))
    offsets = np.concatenate([[0], np.cumsum([s["n_particles"] for s in sets])])
    parts = S.assign_sets(sets, 2)
    for r in range(2):
        steps, xs, ran = res[r]
        # each rank tracked only its own sets ...
        assert ran == sorted(sets[k]["n_turns"] for k in parts[r])
        # ... and every rank returns every set's result, in set order
        for k, s in enumerate(sets):
            assert steps[k] == [s["n_turns"]] * s["n_particles"]
            np.testing.assert_array_equal(xs[k], coords[0][offsets[k]:offsets[k + 1]])
