"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host side.

Photon histories are independent and depend only on (seed, photon id), so a
run shards by photon id ranges (or whole events) with no collective on the
data path. The only exchange is optional: summing the integer tallies of all
ranks (exact, order-independent) and taking the max of per-rank timings.
"""
from __future__ import annotations

import numpy as np


def shard_first_id(rank: int, photons_per_rank: int, base_first_id: int = 0) -> int:
    """First photon id of `rank` when every rank transports photons_per_rank photons."""
    return base_first_id + rank * photons_per_rank


def shard_events(counts, rank: int, world: int):
    """Splits events into `world` contiguous groups of about equal photon count.

    Returns (event index range [lo, hi), photon id offset of event lo) for `rank`;
    event i keeps the photon ids it has in the whole batch."""
    counts = np.asarray(counts, dtype=np.uint64)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    total = int(offs[-1])
    cuts = [int(np.searchsorted(offs, total * r // world, side="left")) for r in range(world + 1)]
    cuts[0], cuts[-1] = 0, len(counts)
    lo, hi = cuts[rank], cuts[rank + 1]
    return (lo, hi), int(offs[lo])


def max_over_ranks(value: float, dist, device=None) -> float:
    """Max of a per-rank scalar (e.g. ms per step) over the process group."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_tallies(tallies: np.ndarray, dist, device=None) -> np.ndarray:
    """Sum of the ranks' integer tallies (exact: 64-bit integer all-reduce)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(tallies).astype(np.int64))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy().astype(np.uint64)
