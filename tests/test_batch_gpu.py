"""Batched heterogeneous tracking (hm_batch_*): every parameter set of the
batch must end exactly as a plain hm_track of that set alone -- same
coordinates bit for bit, same survival turns -- with and without the CUDA
graph, over replays, for both arithmetic modes."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu

C = pytest.importorskip("henon_map_cpp_b200._capi")
from henon_map_cpp_b200 import sweep  # noqa: E402


def plain(s, x, px, y, py, arith):
    t = C.Tracker(s["n_turns"], s["omega_x"], s["omega_y"], "sps", float("nan"), s["epsilon"], 0)
    t.arith = arith
    p = C.Particles(x, px, y, py)
    t.track(p, s["n_turns"], s["mu"], s["barrier"])
    return p.state()


@pytest.mark.parametrize("arith", [0, 1])
def test_batch_equals_plain_per_set(gpu, arith):
    sets, coords = sweep.heterogeneous_sets(seed=11, n_sets=9, n_range=(40, 3000),
                                            turn_range=(50, 6000))
    sets[3]["n_turns"] = 0          # a set with no turns
    sets[5]["n_particles"] = 1      # a one-particle set (keep coords in sync below)
    pts = [sweep.ball_points(np.random.default_rng(100 + k), s["n_particles"], 0.6)
           for k, s in enumerate(sets)]
    coords = tuple(np.concatenate([p[k] for p in pts]) for k in range(4))
    coords[0][7] = np.nan           # a particle lost before tracking
    res_graph = sweep.run_sweep(sets, coords, arith=arith, chunk0=64, chunk_max=1024)
    res_plain = sweep.run_sweep(sets, coords, arith=arith, chunk0=100, chunk_max=100,
                                per_thread=4, use_graph=False)
    res_two = sweep.run_sweep(sets, coords, arith=arith, chunk0=128, chunk_max=2048,
                              per_thread=2)
    o = 0
    for s, rg, rp, r2 in zip(sets, res_graph, res_plain, res_two):
        n = s["n_particles"]
        want = plain(s, *(c[o:o + n] for c in coords), arith)
        o += n
        for r in (rg, rp, r2):
            np.testing.assert_array_equal(r["steps"], want[4])
            for k, w in zip(("x", "px", "y", "py"), want[:4]):
                assert_bitwise(r[k], w, k)
    assert res_graph[0]["steps"][7] == 0 and np.isnan(res_graph[0]["x"][7])


def test_batch_graph_replays_identically(gpu):
    sets, coords = sweep.heterogeneous_sets(seed=5, n_sets=6, n_range=(500, 4000),
                                            turn_range=(200, 3000))
    b = C.Batch(sets)
    b.configure(C.ARITH_EXACT, 2, 128, 512)
    b.load(*coords)
    b.run(True)
    first = [b.get(f) for f in (C.FIELD_X, C.FIELD_STEPS)]
    b.run(True)
    second = [b.get(f) for f in (C.FIELD_X, C.FIELD_STEPS)]
    assert_bitwise(first[0], second[0])
    np.testing.assert_array_equal(first[1], second[1])
    max_turns = max(s["n_turns"] for s in sets)
    done, length, chunks = 0, 128, 0
    while done < max_turns:
        done += min(length, max_turns - done)
        length = min(2 * length, 512)
        chunks += 1
    assert b.n_chunks() == chunks


@pytest.mark.parametrize("arith", [0, 1])
def test_batch_barriers_at_the_last_bit(gpu, arith):
    # One set per barrier whose square lies within a few doubles of some
    # particle's largest radius: each set's loss decisions must be those of
    # a plain hm_track with that barrier (and, exact, of the oracle).
    from conftest import TUNES, edge_barriers, grid
    from oracle import oracle as O

    x, px, y, py = grid(0.5, 8)
    n_turns, eps, mu = 300, 16.0, 0.2
    barriers, _, _ = edge_barriers(x, px, y, py, n_turns, eps, mu)
    sets = [dict(omega_x=TUNES[0], omega_y=TUNES[1], epsilon=eps, mu=mu, n_particles=x.size,
                 n_turns=n_turns, barrier=b) for b in barriers]
    coords = tuple(np.tile(c, len(sets)) for c in (x, px, y, py))
    res = sweep.run_sweep(sets, coords, arith=arith, chunk0=64, chunk_max=128)
    tabs = O.tables(n_turns, *TUNES, "sps", epsilon=eps)
    for s, r in zip(sets, res):
        want = plain(s, x, px, y, py, arith)
        np.testing.assert_array_equal(r["steps"], want[4])
        for k, w in zip(("x", "px", "y", "py"), want[:4]):
            assert_bitwise(r[k], w, k)
        if arith == 0:
            o = O.track(x, px, y, py, np.zeros(x.size, np.uint32), tabs, n_turns, mu, s["barrier"])
            np.testing.assert_array_equal(r["steps"], o[4])


def test_batch_barrier_scales_match_oracle(gpu):
    # One set per barrier scale (subnormal square, small, large, overflowing
    # square, +inf, NaN) in one batch: exact decisions equal the oracle's.
    from conftest import TUNES, grid
    from oracle import oracle as O

    barriers = [1e-160, 1e-3, 0.2, 0.5, 3.0, 1e10, 1e200, np.inf, np.nan]
    x, px, y, py = grid(0.6, 16)
    n_turns, eps, mu = 300, 16.0, 0.2
    sets = [dict(omega_x=TUNES[0], omega_y=TUNES[1], epsilon=eps, mu=mu, n_particles=x.size,
                 n_turns=n_turns, barrier=b) for b in barriers]
    coords = tuple(np.tile(c, len(sets)) for c in (x, px, y, py))
    res = sweep.run_sweep(sets, coords, arith=0, chunk0=64, chunk_max=128)
    tabs = O.tables(n_turns, *TUNES, "sps", epsilon=eps)
    for s, r in zip(sets, res):
        o = O.track(x, px, y, py, np.zeros(x.size, np.uint32), tabs, n_turns, mu, s["barrier"])
        np.testing.assert_array_equal(r["steps"], o[4], err_msg=f"barrier {s['barrier']!r}")
        for k, w in zip(("x", "px", "y", "py"), o[:4]):
            assert_bitwise(r[k], w, k)


def test_batch_groups_do_not_change_results(gpu):
    # Sets split into 1..16 concurrently tracked groups, with grids from a
    # single block per group to the whole device: each set still ends
    # exactly as a plain hm_track of it alone.
    sets, coords = sweep.heterogeneous_sets(seed=23, n_sets=11, n_range=(40, 2000),
                                            turn_range=(50, 5000))
    b = C.Batch(sets)
    b.load(*coords)
    outs = []
    for g, share in ((1, 0.0), (3, 1.5), (8, 1.5), (16, 1e-9), (11, 0.0)):
        b.set_groups(g)
        b.set_grid_share(share)
        b.configure(C.ARITH_EXACT, 1, 128, 1024)
        b.run(True)
        outs.append([b.get(f) for f in (C.FIELD_X, C.FIELD_PY, C.FIELD_STEPS)])
    for o in outs[1:]:
        for a, w in zip(o, outs[0]):
            assert_bitwise(a, w) if a.dtype == np.float64 else np.testing.assert_array_equal(a, w)
    o = 0
    for s in sets:
        n = s["n_particles"]
        want = plain(s, *(c[o:o + n] for c in coords), 0)
        np.testing.assert_array_equal(outs[0][2][o:o + n], want[4])
        o += n
    with pytest.raises(C.HMError):
        b.set_groups(17)
    for bad in (-1.0, float("inf"), float("nan")):
        with pytest.raises(C.HMError):
            b.set_grid_share(bad)


def test_job_list_runs_as_one_batch_like_run_sim(gpu, tmp_path):
    # The reference runs each line of the job list as its own process
    # (htcondor_jobs/run_sim.py); one batch must give every job the
    # survival turns that script gets through the same facade calls.
    import henon_map_cpp_b200 as hm

    path = tmp_path / "all_jobs.txt"
    path.write_text("0.168 0.201 0.0 0.0 0.75\n0.168 0.201 16.0 0.5 0.75\n"
                    "0.31 0.32 64.0 0.25 0.25\n")
    jobs = sweep.read_jobs(path)
    n_points, n_iter = 12, 800
    steps = sweep.run_jobs(jobs, n_points, n_iter, out_dir=tmp_path / "out")
    for j, st in zip(jobs, steps):
        x, px, y, py = sweep.job_grid(j["max_radius"], n_points)
        p = hm.particles(x, px, y, py)
        t = hm.henon_tracker(n_iter, j["omega_x"], j["omega_y"], "sps", epsilon=j["epsilon"])
        t.track(p, n_iter, mu=j["mu"], barrier=10.0)
        want = np.asarray(p.get_steps())
        np.testing.assert_array_equal(st, want)
        base = tmp_path / "out" / sweep.job_file_name(j)
        h5, npz = base.with_suffix(".h5"), base.with_suffix(".npz")
        if h5.exists():
            import h5py

            with h5py.File(h5, "r") as f:
                np.testing.assert_array_equal(f["steps"][...], want)
        else:
            np.testing.assert_array_equal(np.load(npz)["steps"], want)


def test_batch_sets_equal_reference_gpu_tracker(gpu):
    # Each set of a batch against the reference's own GPU tracker built with
    # --fmad=false (henon_tracker_gpu::track, src/henon.cu:3155-3185), set by
    # set: coordinates bit for bit and survival turns.
    from oracle import oracle as O

    if not (O.REF_DIR / "fmad_off").exists():
        pytest.skip("reference build absent")
    sets, coords = sweep.heterogeneous_sets(seed=23, n_sets=5, n_range=(300, 5000),
                                            turn_range=(500, 20000))
    res = sweep.run_sweep(sets, coords, arith=C.ARITH_EXACT)
    o = 0
    for s, r in zip(sets, res):
        n = s["n_particles"]
        part = [c[o:o + n] for c in coords]
        o += n
        want = O.reference_track_subprocess("fmad_off", *part, s["n_turns"],
                                            (s["omega_x"], s["omega_y"]), s["epsilon"], s["mu"],
                                            s["barrier"], gpu=True)
        np.testing.assert_array_equal(r["steps"], want[4])
        for k, w in zip(("x", "px", "y", "py"), want[:4]):
            assert_bitwise(r[k], w, k)
