"""Multi-GPU use of the path tracer: one process per GPU, independent units per rank.

Camera samples are independent given the scene, and so are whole images and batch jobs, so ranks
split the units among themselves and exchange nothing on the data path (the reference renders one
image per process with host threads, graphics_engine.cpp:42-57). Each rank keeps its own copy of
the read-only scene on its GPU. The only collectives are bookkeeping: the maximum device time
over ranks (the job's time) and sums of counts. Every rank calls them in the same order.
"""


def shard(n, rank, world):
    """[lo, hi) of n units owned by rank: contiguous blocks whose sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %r outside world of size %r" % (rank, world))
    base, extra = divmod(int(n), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def owned(units, rank, world):
    """The slice of a list of units (images, batch jobs, seeds) that rank renders."""
    lo, hi = shard(len(units), rank, world)
    return units[lo:hi]


def _reduce(values, op, device):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=op)
    return [float(v) for v in t.cpu()]


def _device():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_backend() == "nccl":
        import torch
        return torch.device("cuda", torch.cuda.current_device())
    return "cpu"


def max_over_ranks(values):
    """Element-wise maximum over ranks (list of floats); the identity without a process group."""
    import torch.distributed as dist
    return _reduce(values, dist.ReduceOp.MAX if dist.is_available() else None, _device())


def sum_over_ranks(values):
    """Element-wise sum over ranks (list of floats); the identity without a process group."""
    import torch.distributed as dist
    return _reduce(values, dist.ReduceOp.SUM if dist.is_available() else None, _device())
