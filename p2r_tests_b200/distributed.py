"""Multi-GPU plumbing: one process per GPU over torch.distributed.

Tracks are independent, so the forward shards events across ranks with no data-path
collective (weak scaling: each rank owns a contiguous event range, which is one contiguous
byte range of the Matriplex arrays). The only exchange is in calibration: the per-layer
radius-offset and Bz gradients of the adjoint are summed over ranks with one all-reduce
(NCCL over NVLink on GPUs, gloo in the CPU tests). The reference has no multi-process code.
"""
from __future__ import annotations

import numpy as np


def shard_events(nevts: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous event range [e0, e1) of `rank`; sizes differ by at most one event."""
    if world < 1 or not 0 <= rank < world or nevts < 0:
        raise ValueError("bad world/rank/nevts")
    return nevts * rank // world, nevts * (rank + 1) // world


def shard_uneven(ntrk_event, world: int, rank: int) -> tuple[int, int]:
    """Contiguous event range balancing the TRACK count (prefix split of the cumulative
    counts at multiples of total/world), for batches with uneven events."""
    counts = np.asarray(ntrk_event, np.int64).reshape(-1)
    if world < 1 or not 0 <= rank < world or (counts < 0).any():
        raise ValueError("bad world/rank or negative track count")
    c = np.concatenate([[0], np.cumsum(counts)])
    total = c[-1]
    cut = lambda r: int(np.searchsorted(c, total * r / world, side="left")) if r < world else len(c) - 1
    return cut(rank), cut(rank + 1)


def event_slice(arr: np.ndarray, e0: int, e1: int, nevts: int) -> np.ndarray:
    """The rows of a Matriplex array (tracks or hits, event-major) that belong to [e0, e1)."""
    flat = np.ascontiguousarray(arr).reshape(-1)
    if nevts < 1 or flat.size % nevts or not 0 <= e0 <= e1 <= nevts:
        raise ValueError(f"event range [{e0}, {e1}) of {nevts} events over {flat.size} words")
    per = flat.size // nevts
    return flat[e0 * per:e1 * per]


def allreduce_calibration(grad_dr, grad_bz, group=None):
    """Sums the shared calibration gradients over ranks (in place; returns them)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return grad_dr, grad_bz
    buf = torch.cat([grad_dr.reshape(-1), grad_bz.reshape(-1)])
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    n = grad_dr.numel()
    grad_dr.copy_(buf[:n].reshape(grad_dr.shape))
    grad_bz.copy_(buf[n:].reshape(grad_bz.shape))
    return grad_dr, grad_bz
