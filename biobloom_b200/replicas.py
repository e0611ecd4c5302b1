"""Replica sharding across GPUs: one process per GPU holds every filter, the
reads are split into contiguous shards, and the only exchange is one sum of
the summary counters (and a max of the step times for reporting).

The reference has no multi-GPU path (its parallelism is OpenMP threads in one
process); the classification of each read does not depend on any other read,
so shards need no communication while they run.
"""


def shard_range(n, rank, world):
    """[lo, hi) of the reads rank `rank` of `world` classifies: contiguous,
    sizes differing by at most one, covering [0, n) exactly once."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(int(n), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def reduce_counts(counts, group=None):
    """Sum summary counters (a 1-D integer numpy array) over all ranks; returns
    the summed array (the input is left unchanged)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.asarray(counts, dtype=np.int64).copy())
    if dist.is_available() and dist.is_initialized():
        backend = dist.get_backend(group)
        if backend == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().astype(np.uint64)


def max_over_ranks(value, group=None):
    """The largest of one float per rank (step times are reported as the max)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.is_available() and dist.is_initialized():
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.cpu().item())
