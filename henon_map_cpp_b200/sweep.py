"""Parameter sweeps as one batched launch.

The reference sweeps (omega_x, omega_y, epsilon, mu) grids with one process
and one GPU per parameter set (htcondor_jobs/compose_config.py:3-15,
run_sim.py:41-74).  Here a whole sweep is one hm_batch: every set keeps its
own particle count and turn budget, and the sets are tracked together as a
replayed CUDA graph of persistent chunk launches.

    sets = heterogeneous_sets(seed=20261203)           # or sweep_sets(...)
    result = run_sweep(sets, points)                   # steps per set

The reference's job list (configs/all_jobs.txt, one "omega_x omega_y
epsilon mu max_radius" line per job) runs as one batch too, writing one
result file per job as its run_sim.py does:

    python -m henon_map_cpp_b200.sweep --jobs configs/all_jobs.txt \
        --num_points 100 --num_iterations 100000 --out results/
"""
from __future__ import annotations

import math

import numpy as np

from . import _capi as C


def ball_points(rng: np.random.Generator, n: int, radius: float):
    """n points uniform in the 4D ball of the given radius."""
    g = rng.normal(size=(n, 4))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    r = radius * rng.uniform(size=n) ** 0.25
    p = g * r[:, None]
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), p[:, 3].copy()


def heterogeneous_sets(seed: int = 20261203, n_sets: int = 64, n_range=(1_000, 256_000),
                       turn_range=(1_000, 1_000_000), radius: float = 0.6):
    """The mixed-size workload: n_sets parameter sets with tunes
    U[0.15, 0.32], epsilon U[0, 64], mu U[-0.5, 0.5], log-uniform particle
    counts and turn budgets, points uniform in the 4D ball r < radius.

    Returns (sets, (x, px, y, py)) with the points of all sets concatenated
    in set order."""
    rng = np.random.default_rng(seed)
    sets = []
    for _ in range(n_sets):
        tx, ty = rng.uniform(0.15, 0.32, size=2)
        eps = rng.uniform(0.0, 64.0)
        mu = rng.uniform(-0.5, 0.5)
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        t = int(round(math.exp(rng.uniform(math.log(turn_range[0]), math.log(turn_range[1])))))
        sets.append(dict(omega_x=tx, omega_y=ty, epsilon=eps, mu=mu, n_particles=n, n_turns=t,
                         barrier=10.0))
    pts = [ball_points(rng, s["n_particles"], radius) for s in sets]
    coords = tuple(np.concatenate([p[k] for p in pts]) for k in range(4))
    return sets, coords


def sweep_sets(omega_pairs, epsilons, mus, n_particles: int, n_turns: int,
               barrier: float = 10.0):
    """The reference's sweep grid (compose_config.py): every combination of
    (omega_x, omega_y) pair, epsilon and mu, each on the same particles."""
    return [dict(omega_x=wx, omega_y=wy, epsilon=e, mu=m, n_particles=n_particles,
                 n_turns=n_turns, barrier=barrier)
            for (wx, wy) in omega_pairs for e in epsilons for m in mus]


def shard_sets(sets, coords, rank: int, world: int):
    """This rank's share of a sweep: the set indices that longest-processing-
    time assignment (sharding.assign_sets, on particles x turns) gives it,
    those sets, and their points cut out of the concatenated coords.  This
    replaces the reference's one-GPU-per-job HTCondor submission
    (htcondor_jobs/htcondor_gpu.sub, run_sim.py:41-74) with one batch per
    rank."""
    from .sharding import assign_sets

    offsets = np.concatenate([[0], np.cumsum([int(s["n_particles"]) for s in sets])])
    mine = assign_sets(sets, world)[rank] if sets else []
    sub = [sets[k] for k in mine]
    sub_coords = tuple(
        np.concatenate([np.asarray(c)[offsets[k]:offsets[k + 1]] for k in mine])
        if mine else np.zeros(0) for c in coords)
    return mine, sub, sub_coords


def run_sweep(sets, coords, arith: int = C.ARITH_EXACT, per_thread: int = 1,
              chunk0: int = 512, chunk_max: int = 4096, use_graph: bool = True,
              distributed: bool | None = None, group=None):
    """Tracks every set to its budget; returns a list with one dict per set:
    x, px, y, py (final) and steps (survival turns).

    With a torch.distributed process group (distributed=None: whenever one is
    initialised with more than one rank), each rank tracks the sets that
    shard_sets assigns it as one batch on its own GPU -- no exchange during
    tracking -- and the per-set results are then gathered so that every
    rank returns all of them."""
    if distributed is None:
        try:
            import torch.distributed as dist

            distributed = dist.is_available() and dist.is_initialized() and \
                dist.get_world_size(group) > 1
        except ImportError:
            distributed = False
    if not distributed:
        return _local_sweep(sets, coords, arith, per_thread, chunk0, chunk_max, use_graph)
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine, sub, sub_coords = shard_sets(sets, coords, rank, world)
    local = _local_sweep(sub, sub_coords, arith, per_thread, chunk0, chunk_max,
                         use_graph) if sub else []
    parts = [None] * world
    dist.all_gather_object(parts, list(zip(mine, local)), group=group)
    out = [None] * len(sets)
    for part in parts:
        for k, r in part:
            out[k] = r
    return out


def _local_sweep(sets, coords, arith, per_thread, chunk0, chunk_max, use_graph):
    """Every set in one batch on the current device."""
    b = C.Batch(sets)
    b.configure(arith, per_thread, chunk0, chunk_max)
    b.load(*coords)
    b.run(use_graph)
    fields = {k: b.get(f) for k, f in (("x", C.FIELD_X), ("px", C.FIELD_PX), ("y", C.FIELD_Y),
                                         ("py", C.FIELD_PY), ("steps", C.FIELD_STEPS))}
    out, o = [], 0
    for s in sets:
        n = int(s["n_particles"])
        out.append({k: v[o:o + n] for k, v in fields.items()})
        o += n
    return out


# ---- the reference's job list ------------------------------------------------------

def read_jobs(path):
    """Jobs of a compose_config.py list (htcondor_jobs/compose_config.py:12-15):
    one "omega_x omega_y epsilon mu max_radius" line each."""
    jobs = []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if len(parts) != 5:
                raise ValueError(f"{path}: expected 5 numbers per line, got {line.strip()!r}")
            ox, oy, eps, mu, rmax = (float(v) for v in parts)
            jobs.append(dict(omega_x=ox, omega_y=oy, epsilon=eps, mu=mu, max_radius=rmax))
    return jobs


def job_grid(max_radius: float, num_points: int):
    """run_sim.py's initial conditions (htcondor_jobs/run_sim.py:28-36): the
    num_points x num_points grid of (x, y) on [0, max_radius]^2, px = py = 0."""
    positions = np.linspace(0, max_radius, num_points)
    xx, yy = np.meshgrid(positions, positions)
    x, y = xx.flatten(), yy.flatten()
    return x, np.zeros_like(x), y, np.zeros_like(y)


def job_file_name(job) -> str:
    """run_sim.py's output name (:64-66), decimal points written as "d"."""
    f = lambda v: str(v).replace(".", "d")  # noqa: E731
    return (f"stability_henon_{f(job['omega_x'])}_{f(job['omega_y'])}_{f(job['epsilon'])}_"
            f"{f(job['mu'])}_{f(job['max_radius'])}")


def run_jobs(jobs, num_points: int = 100, num_iterations: int = 100_000, out_dir=None,
             arith: int = C.ARITH_EXACT):
    """Every job of the list in one batch: SPS modulation, barrier 10, each on
    its own grid (run_sim.py:40-47).  Returns the survival turns of each job;
    with out_dir, also writes one file per job holding `steps`: HDF5 as the
    reference does when h5py is importable, else .npz.  Under a
    torch.distributed process group the jobs are spread over the ranks
    (run_sweep) and rank 0 writes every file."""
    import os

    sets, pts = [], []
    for j in jobs:
        sets.append(dict(omega_x=j["omega_x"], omega_y=j["omega_y"], epsilon=j["epsilon"],
                         mu=j["mu"], n_particles=num_points * num_points,
                         n_turns=num_iterations, barrier=10.0))
        pts.append(job_grid(j["max_radius"], num_points))
    coords = tuple(np.concatenate([p[k] for p in pts]) for k in range(4)) if pts else \
        tuple(np.zeros(0) for _ in range(4))
    results = run_sweep(sets, coords, arith=arith) if sets else []
    steps = [r["steps"] for r in results]
    if out_dir is not None and _rank() == 0:
        os.makedirs(out_dir, exist_ok=True)
        try:
            import h5py  # noqa: PLC0415
        except ImportError:
            h5py = None
        for j, st in zip(jobs, steps):
            base = os.path.join(out_dir, job_file_name(j))
            if h5py is not None:
                with h5py.File(base + ".h5", "w") as f:
                    f.create_dataset("steps", data=st)
            else:
                np.savez(base + ".npz", steps=st)
    return steps


def _rank() -> int:
    try:
        import torch.distributed as dist

        return dist.get_rank() if dist.is_available() and dist.is_initialized() else 0
    except ImportError:
        return 0


def main(argv=None) -> None:
    import argparse
    import time

    ap = argparse.ArgumentParser(description="Run a job list of parameter sets as one batch.")
    ap.add_argument("--jobs", required=True, help="compose_config.py list: omega_x omega_y "
                                                  "epsilon mu max_radius per line")
    ap.add_argument("--num_points", type=int, default=100)
    ap.add_argument("--num_iterations", type=int, default=100_000)
    ap.add_argument("--out", default=".")
    args = ap.parse_args(argv)
    jobs = read_jobs(args.jobs)
    t0 = time.perf_counter()
    run_jobs(jobs, args.num_points, args.num_iterations, args.out)
    print(f"{len(jobs)} jobs in {time.perf_counter() - t0:.3f} s", flush=True)


if __name__ == "__main__":
    main()
