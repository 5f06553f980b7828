"""Multi-GPU plumbing of the renderer: ensembles are independent of each other, so N ranks (one
process per GPU) split the ensembles of every camera and need no collective on the data path.
The only exchange is optional: summing the ranks' accumulations into one history, a single
all-reduce of W*H*4 floats (NCCL over NVLink on GPUs, gloo in the CPU tests).
"""


def shard(count: int, world: int, rank: int):
    """(first ensemble offset, ensembles) of `rank` when `count` ensembles are split over `world`
    ranks: contiguous, sizes differing by at most one, in rank order."""
    base, extra = divmod(count, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def rank_first_seed(first_seed: int, count: int, world: int, rank: int) -> int:
    """Seed of the first ensemble of `rank` so that the union over ranks is exactly the seeds
    first_seed .. first_seed + count - 1 of a single-process render_ensembles call."""
    return (first_seed + shard(count, world, rank)[0]) & 0xFFFFFFFF


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of a per-rank number (the bench's timed milliseconds)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_accum(accum, dist=None):
    """Sums the ranks' (RGB sum, count) accumulation tensors in place (all ranks get the total)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return accum
    dist.all_reduce(accum, op=dist.ReduceOp.SUM)
    return accum
