"""One replica per GPU: CPIs are independent, so a stream of CPIs is sharded across ranks
with no data exchange; ranks meet only to agree on timing (barrier, max over ranks)."""
from __future__ import annotations

from typing import List, Sequence


def shard(items: Sequence, rank: int, world: int) -> List:
    """Round-robin share of `items` for `rank` (every item goes to exactly one rank)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    return list(items[rank::world])


def max_over_ranks(values, dist=None, device=None):
    """Element-wise maximum of per-rank timings (a list of floats) across the process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]
