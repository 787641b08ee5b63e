"""Particles split across ranks (one process per GPU): the partial-map sum.

The reference reconstructs with one partial map per thread and sums them in
thread order before weighing (img_reconstruction_sum_weigh,
bsoft/src/mg/mg_reconstruct.cpp:263-324; the threads' maps are made in
breconstruct.cpp:268-305).  Across GPUs the same step is one exchange at
the end: every rank's FP64 accumulators go to one rank, which adds them in
rank order, so the result depends only on the split and not on timing.

``shard_indices`` gives rank r the particles r, r + world, ... (the split
the benchmark uses).  ``gather_partials`` moves each rank's arrays to rank
`dst` in rank order over a torch.distributed group that carries CPU tensors
(gloo); ``reduce_partial_maps`` applies it to a Reconstructor's
accumulators and adds the other ranks' sums into rank `dst`'s context
(bsg_recon_add_partial), after which that context finishes the map.
"""
from __future__ import annotations

import numpy as np


def shard_indices(n: int, rank: int, world: int) -> np.ndarray:
    """Indices of the particles rank `rank` of `world` inserts."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return np.arange(rank, n, world)


def gather_partials(arrays, group=None, dst: int = 0):
    """Each rank's list of float64 arrays (the same shapes on every rank) to
    rank `dst`: returns, on `dst`, one list of arrays per rank in rank
    order, and None elsewhere.  Every rank of the group must call it."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    out = [] if rank == dst else None
    for a in arrays:
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
        bufs = [torch.empty_like(t) for _ in range(world)] if rank == dst else None
        dist.gather(t, gather_list=bufs, dst=dst, group=group)
        if rank == dst:
            out.append([b.numpy() for b in bufs])
    if rank != dst:
        return None
    return [[out[i][r] for i in range(len(arrays))] for r in range(world)]


def sum_in_rank_order(parts):
    """The partial sums of every rank added in rank order (FP64)."""
    total = [np.array(p, dtype=np.float64, copy=True) for p in parts[0]]
    for pr in parts[1:]:
        for t, p in zip(total, pr):
            t += p
    return total


def reduce_partial_maps(rec, half: int = 0, group=None, dst: int = 0) -> None:
    """Add every other rank's accumulators of half `half` into rank `dst`'s
    Reconstructor, in rank order after its own sums (exactly the rank-order
    sum for dst = 0); rank `dst` then finishes the map.  `rec` needs
    accumulators(half) -> (complex vol, weight) and add_partial(vol,
    weight, half), as Reconstructor has."""
    import torch.distributed as dist
    vol, w = rec.accumulators(half)
    v2 = np.stack([vol.real, vol.imag], axis=-1)
    parts = gather_partials([v2, w], group=group, dst=dst)
    if parts is None:
        return
    for r, (pv, pw) in enumerate(parts):
        if r == dist.get_rank(group):
            continue
        rec.add_partial(pv[..., 0] + 1j * pv[..., 1], pw, half)
