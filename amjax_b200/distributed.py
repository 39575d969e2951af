"""Multi-GPU solves: independent right-hand-side columns sharded across ranks.

The solve phase of one hierarchy does not shard by rows without a halo exchange per
SpMV and an all-reduce per CG dot; what does shard cleanly is the batch: every rank
holds a replica of the hierarchy and solves its own contiguous block of the k columns.
There is no collective on the data path; ``gather=True`` adds one all-gather of the
solutions at the end (for callers that want X on every rank).
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard_columns(k: int, world: int, rank: int):
    """Contiguous block [lo, hi) of k columns for ``rank`` (sizes differ by at most 1)."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world {world}")
    base, rem = divmod(k, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def solve_sharded(ml, B, method="pcg", group=None, gather=True, solve_fn=None, **kwargs):
    """Solve this rank's columns of B ([N, k]) with ``ml.<method>``; optionally all-gather.

    ``solve_fn(B_local, **kwargs) -> X_local`` overrides the per-rank solver."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    k = int(B.shape[1])
    lo, hi = shard_columns(k, world, rank)
    fn = solve_fn if solve_fn is not None else getattr(ml, method)
    B_local = B[:, lo:hi].contiguous()
    X_local = fn(B_local, **kwargs) if hi > lo else B_local.clone()
    X_local = torch.as_tensor(X_local).reshape(B.shape[0], hi - lo)
    if not gather:
        return X_local, (lo, hi)
    width = -(-k // world)
    pad = torch.zeros(B.shape[0], width, dtype=X_local.dtype, device=X_local.device)
    pad[:, : hi - lo] = X_local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    cols = []
    for r in range(world):
        a, b = shard_columns(k, world, r)
        cols.append(parts[r][:, : b - a])
    return torch.cat(cols, dim=1)
