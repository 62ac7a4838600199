"""Multi-GPU partitioning: one process per GPU, no exchange inside the turn
loop (particles and parameter sets are independent).

* particle_shard / interleaved_grid: a rank's share of one ensemble;
* assign_sets: parameter sets of a sweep spread over ranks by
  longest-processing-time on (particles x turns);
* reduce_loss: the single collective of the differentiable loss, one
  all_reduce of [loss sum, survivor count, dL/dtheta (4)];
* gather_steps: survival turns of every shard, to rank 0.
"""
from __future__ import annotations

import heapq

import numpy as np


def particle_shard(n: int, rank: int, world: int) -> slice:
    """Contiguous slice of n particles for `rank` (sizes differ by <= 1)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def interleaved_grid(side: int, rank: int, world: int, extent: float = 0.6):
    """Rank's columns of a side x (side*world) grid on [0, extent]^2 (every
    world-th column), px0 = py0 = 0: equal-sized shards whose loss rates
    match, so a weak-scaling run keeps every GPU equally busy."""
    xs = np.linspace(0.0, extent, side * world)[rank::world]
    ys = np.linspace(0.0, extent, side)
    xx, yy = np.meshgrid(xs, ys)
    x = np.ascontiguousarray(xx.ravel())
    y = np.ascontiguousarray(yy.ravel())
    return x, np.zeros_like(x), y, np.zeros_like(y)


def assign_sets(sets, world: int):
    """Longest-processing-time assignment of parameter sets to ranks by
    n_particles * n_turns; returns one list of set indices per rank."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    order = sorted(range(len(sets)), key=lambda k: -float(sets[k]["n_particles"]) *
                   float(sets[k]["n_turns"]))
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + float(sets[k]["n_particles"]) * float(sets[k]["n_turns"]), r))
    for lst in out:
        lst.sort()
    return out


def reduce_loss(loss_sum, count, grad_theta, group=None):
    """Sums [loss_sum, count, grad_theta[0..3]] over the ranks of `group`
    (one all_reduce) and returns (mean loss, mean dL/dtheta)."""
    import torch
    import torch.distributed as dist

    t = torch.cat([torch.as_tensor([float(loss_sum), float(count)], dtype=torch.float64),
                   torch.as_tensor(grad_theta, dtype=torch.float64).reshape(4).cpu()])
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
    return float(t[0] / t[1]), (t[2:] / t[1]).numpy()


def gather_steps(steps, group=None):
    """All shards' survival turns concatenated in rank order (every rank
    gets the result)."""
    import torch
    import torch.distributed as dist

    s = torch.as_tensor(np.asarray(steps, dtype=np.int64))
    if not (dist.is_available() and dist.is_initialized()):
        return s.numpy()
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(dist.get_world_size(group))]
    dist.all_gather(sizes, torch.tensor([s.numel()], dtype=torch.int64), group=group)
    m = int(max(int(z) for z in sizes))
    pad = torch.full((m,), -1, dtype=torch.int64)
    pad[:s.numel()] = s
    parts = [torch.empty(m, dtype=torch.int64) for _ in sizes]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:int(z)] for p, z in zip(parts, sizes)]).numpy()
