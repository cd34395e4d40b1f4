"""Multi-GPU plumbing of the monodomain path: one process per GPU, no
data-path collective.

The reference advances one heart in one process; nothing in its time step
exchanges data between devices (simulation/functions/
purkinje_myocardium_pipeline.py:1347-1420).  Here the units that shard are
whole hearts: a single heart runs as one replica per rank, and an ensemble's
variants are dealt to ranks by longest-processing-time-first on their voxel
counts, each rank advancing its share as one batched ensemble.  The only
collectives are on the host side of the timed region: a barrier before it,
the maximum of the ranks' device times after it, and the gather of per-rank
results.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_assign(sizes, n_ranks):
    """Variant indices per rank, largest first onto the least-loaded rank
    (ties to the lower rank).  Every rank's list is in increasing order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    sizes = np.asarray(sizes, np.int64)
    heap = [(0, r) for r in range(n_ranks)]
    out = [[] for _ in range(n_ranks)]
    for v in sorted(range(len(sizes)), key=lambda q: (-int(sizes[q]), q)):
        load, r = heapq.heappop(heap)
        out[r].append(v)
        heapq.heappush(heap, (load + int(sizes[v]), r))
    return [sorted(o) for o in out]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank float over the default process group (the
    job's time is its slowest rank's); identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_all(obj):
    """Every rank's object, in rank order (host-side gather)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def shard_run_gather(sizes, run_share):
    """Deals the variants (expected work `sizes`) to the ranks of the
    default process group by longest-processing-time-first, runs
    run_share(indices) on each rank -- it returns one result per index, in
    the order given -- and returns every variant's result in variant order
    on every rank.  Without a process group the one rank runs them all."""
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if on else 1
    rank = dist.get_rank() if on else 0
    share = lpt_assign(sizes, world)[rank]
    res = list(run_share(share))
    if len(res) != len(share):
        raise ValueError(f"run_share returned {len(res)} results for {len(share)} variants")
    out = [None] * len(sizes)
    for g in gather_to_all({"variants": share, "results": res}):
        for v, r in zip(g["variants"], g["results"]):
            out[v] = r
    return out
