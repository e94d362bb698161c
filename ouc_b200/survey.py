"""A survey of many shots over one or several GPUs (one process per GPU).

The reference migrates its shots one after another in one process
(P-S-seperating.cu:2108-2400) and sums the per-shot Laplacian images on the
host afterwards (PS:2403-2443).  Nothing but that sum links two shots, so
shots shard across ranks with no collective on the data path: each rank
migrates its own share, ``max_batch`` shots per launch, into its context's
FP64 stack, and the single exchange is one all-reduce (sum) of the three FP64
stacks -- PP, PS and illumination -- at the end.

``partition`` assigns shots to ranks, round-robin or, given per-shot costs
(e.g. cell-updates of shots on sub-grids of different apertures), greedily
by longest cost first.  ``reduce_stack`` is the exchange; it works on any
``torch.distributed`` backend (NCCL on B200s, gloo on the host).
``migrate`` drives one rank's share through a ``Context``.
"""
from __future__ import annotations

import numpy as np


def partition(n_shots: int, world: int, rank: int, cost=None) -> list[int]:
    """Indices of the shots rank ``rank`` of ``world`` migrates, ascending.

    cost None: round-robin (shot k on rank k mod world).  Otherwise the
    shots are taken in order of decreasing cost (ties by index) and each goes
    to the rank with the least cost so far (ties to the lowest rank), so the
    ranks' totals differ by at most the largest single cost.  Every rank
    computes the same assignment from the same arguments; the union over the
    ranks is every shot exactly once."""
    if world < 1 or not 0 <= rank < world or n_shots < 0:
        raise ValueError(f"bad partition request: {n_shots} shots, rank {rank} of {world}")
    if cost is None:
        return list(range(rank, n_shots, world))
    cost = np.asarray(cost, dtype=np.float64)
    if cost.shape != (n_shots,) or not np.all(np.isfinite(cost)) or np.any(cost < 0):
        raise ValueError("cost must hold one finite, non-negative value per shot")
    load = np.zeros(world)
    owner = np.empty(n_shots, dtype=np.int64)
    for k in sorted(range(n_shots), key=lambda i: (-cost[i], i)):
        r = int(np.argmin(load))            # first minimum: lowest rank on ties
        owner[k] = r
        load[r] += cost[k]
    return [int(k) for k in np.nonzero(owner == rank)[0]]


def reduce_stack(pp, ps, illum, group=None):
    """Sum the ranks' FP64 stacks in place (all ranks end with the total).

    pp, ps, illum: float64 torch tensors of one shape on the backend's device
    (CUDA for NCCL, CPU for gloo).  One all-reduce carries all three."""
    import torch
    import torch.distributed as dist
    parts = (pp, ps, illum)
    for t in parts:
        if t.dtype != torch.float64 or t.shape != pp.shape:
            raise ValueError("stacks must be float64 tensors of one shape")
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return parts
    buf = torch.cat([t.reshape(-1) for t in parts])
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    n = pp.numel()
    for k, t in enumerate(parts):
        t.copy_(buf[k * n:(k + 1) * n].view_as(t))
    return parts


def migrate(ctx, shots, wavelet, recs=None, rank=0, world=1, cost=None, group=None):
    """Migrate this rank's share of ``shots`` and return the survey's FP64
    stacks (PP, PS, illumination) as numpy arrays, summed over all ranks.

    ctx: a ``Context`` on this rank's GPU whose stack holds nothing yet;
    recs: per-shot (rec_vx, rec_vz) host arrays, or None for self-modelled
    records.  Shots go through ``rtm_batch`` in groups of ``max_batch``."""
    import torch
    mine = partition(len(shots), world, rank, cost)
    b = max(1, ctx.cfg.max_batch)
    for k in range(0, len(mine), b):
        idx = mine[k:k + b]
        ctx.rtm_batch([shots[i] for i in idx], wavelet, None if recs is None else [recs[i] for i in idx])
    pp, ps, il = ctx.stack(reset=True)
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if (
        dist.is_initialized() and dist.get_backend(group) == "nccl") else torch.device("cpu")
    t = [torch.from_numpy(a).to(dev) for a in (pp, ps, il)]
    reduce_stack(*t, group=group)
    return tuple(x.cpu().numpy() for x in t)
