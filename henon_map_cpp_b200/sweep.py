"""Parameter sweeps as one batched launch.

The reference sweeps (omega_x, omega_y, epsilon, mu) grids with one process
and one GPU per parameter set (htcondor_jobs/compose_config.py:3-15,
run_sim.py:41-74).  Here a whole sweep is one hm_batch: every set keeps its
own particle count and turn budget, and the sets are tracked together as a
replayed CUDA graph of persistent chunk launches.

    sets = heterogeneous_sets(seed=20261203)           # or sweep_sets(...)
    result = run_sweep(sets, points)                   # steps per set
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


def run_sweep(sets, coords, arith: int = C.ARITH_EXACT, per_thread: int = 1,
              chunk0: int = 512, chunk_max: int = 16384, use_graph: bool = True):
    """Tracks every set to its budget in one batch; returns a list with one
    dict per set: x, px, y, py (final) and steps (survival turns)."""
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
