"""Multi-GPU layout: one process per GPU, no data-path collective.

The assembly of one mesh runs on one GPU. Several GPUs either run independent replicas of the same workload
(the benchmark's weak scaling) or share the independent specimens of a batched calibration sweep, in
contiguous blocks by specimen index. The only collectives are the timing barrier and the max-over-ranks of the
timed region.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous block of items owned by `rank`: sizes differ by at most one, lower ranks take the extra."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def specimen_shard(scale: float, seed: int, rank: int, world: int):
    """(mesh, json_dict, state_fn) of this rank's specimens of the batched sweep."""
    from . import config as cf
    specs = cf.specimen_draws(scale, seed)
    mine = [specs[i] for i in shard(len(specs), rank, world)]
    return cf.batch_config(mine, seed)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar (the timed region's device time) over all ranks; identity without dist."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
