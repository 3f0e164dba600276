"""Multi-GPU by replicas: one process per GPU, no data-path collective.

The lattice path does not shard in this implementation (halo exchange is
replaced by in-kernel periodic indexing).  What spreads over GPUs is
independent work: replicas of one lattice (Philox stream = rank) or the
lattices of an ensemble.  The only cross-GPU steps are host-side: a balanced
partition of the lattices, a gather of per-lattice observables to rank 0, and
the max over ranks of each timed region.  They run over any torch.distributed
process group (NCCL on the GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(sites, world: int):
    """Lattice indices per rank, balancing total sites (longest first onto the lightest rank).

    Deterministic: ties go to the lower rank and, among equal lattices, the lower index.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sites)), key=lambda i: (-int(sites[i]), i))
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sites[i]), r))
    return [sorted(p) for p in parts]


def gather_observables(local: dict, world: int, rank: int, group=None):
    """Rank 0 receives {lattice index: array} from every rank, merged and ordered by index.

    Other ranks receive None.  Every rank takes part (same collective steps in the
    same order on all ranks).
    """
    if world == 1:
        return dict(sorted(local.items()))
    import torch.distributed as dist

    payload = {int(k): np.asarray(v) for k, v in local.items()}
    out = [None] * world if rank == 0 else None
    dist.gather_object(payload, out, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"lattice {k} reported by two ranks")
            merged[k] = v
    return dict(sorted(merged.items()))


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a timing over ranks (all ranks call it)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_statistics(values: dict):
    """Mean over replicas and its standard error (replicas independent)."""
    v = np.array([np.asarray(x, np.float64) for _, x in sorted(values.items())])
    mean = v.mean(axis=0)
    err = v.std(axis=0, ddof=1) / np.sqrt(v.shape[0]) if v.shape[0] > 1 else np.zeros_like(mean)
    return mean, err
