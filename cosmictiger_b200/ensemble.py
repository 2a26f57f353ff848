"""Placement of independent periodic boxes on GPUs and the aggregation of their timings.

Boxes of an ensemble (or requests of the serving loop) never exchange data: each rank owns a
disjoint subset of whole boxes and the only collective is the final reduction of counters
(max of the timed region, sum of particle-steps).  The reference has no such layer (its
multi-node path is a domain decomposition of one box over HPX localities, out of scope here).
"""
import numpy as np


def shard_boxes(sizes, world, rank):
    """Indices of the boxes owned by `rank`: greedy largest-first onto the least-loaded rank,
    so that every rank gets a near-equal particle count.  Deterministic for given sizes."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(sizes), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += sizes[i]
    return np.nonzero(owner == rank)[0]


def aggregate(local_ms, local_particle_steps, dist=None, device=None):
    """Whole-job throughput: sum of particle-steps over ranks / max timed region over ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local_particle_steps / (local_ms / 1e3), local_ms
    import torch

    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    n = torch.tensor([float(local_particle_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(n.item()) / (float(t.item()) / 1e3), float(t.item())
