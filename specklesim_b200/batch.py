"""Many independent solves across the GPUs of one node.

The solve path has no data exchange: realisations (independent meshes) and their
right-hand sides are the unit of parallel work.  One process per GPU takes a share of
the realisations; nothing crosses NVLink during a solve.  The only collective is the
final gather of the far-field intensities and statistics to rank 0.

Realisations of uneven size are shared by a greedy bin-pack on the edge count: the
largest realisation goes to the least-loaded rank (the cost of a solve grows with M).
"""
import heapq

import numpy as np


def assign_realisations(sizes, world):
    """Indices of the realisations each rank solves: greedy longest-first bin-packing on
    `sizes` (e.g. RWG edge counts).  Deterministic, so every rank computes the same plan."""
    heap = [(0.0, r) for r in range(world)]
    plan = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-float(sizes[i]), i)):
        load, r = heapq.heappop(heap)
        plan[r].append(i)
        heapq.heappush(heap, (load + float(sizes[i]), r))
    return [sorted(p) for p in plan]


def gather_to_rank0(local, world, rank, group=None):
    """Gather one picklable object per rank to rank 0 (a list in rank order there, None
    elsewhere).  Uses torch.distributed when world > 1."""
    if world == 1:
        return [local]
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(local, out, dst=0, group=group)
    return out


def run_batch(realisations, solve_one, world=1, rank=0, group=None):
    """Solve every realisation of `realisations` (a list of dicts holding at least
    "n_edges") on this node's ranks.  `solve_one(realisation)` runs on the rank's own GPU
    and returns a dict (intensities, statistics).  Returns, on rank 0, the results in
    realisation order; on the other ranks None."""
    plan = assign_realisations([r["n_edges"] for r in realisations], world)
    mine = {i: solve_one(realisations[i]) for i in plan[rank]}
    parts = gather_to_rank0(mine, world, rank, group)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[i] for i in range(len(realisations))]


def balance(plan, sizes):
    """Largest / mean per-rank load of a plan (1.0 = perfect)."""
    loads = np.array([sum(sizes[i] for i in p) for p in plan], dtype=float)
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0
