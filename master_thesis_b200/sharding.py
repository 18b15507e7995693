"""Multi-GPU use of the path tracer: one process per GPU, independent units per rank.

Camera samples are independent given the scene, and so are whole images and batch jobs, so ranks
split the units among themselves (the reference renders one image per process with host threads,
graphics_engine.cpp:42-57). Each rank keeps its own copy of the read-only scene on its GPU.

  - Whole images or batch jobs per rank (owned): nothing is exchanged on the data path.
  - One image over all ranks (render_split): pixel tiles assembled by one all_gather (exact), or
    sample ranges added by one all_reduce of the float32 image.
  - One gradient over all ranks (adjoint_split): sample ranges, one all_reduce per gradient.

Bookkeeping collectives: the maximum device time over ranks (the job's time) and sums of counts.
Every rank makes the same collective calls in the same order. Collectives go through
torch.distributed (NCCL between GPUs, gloo on the CPU).
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


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1 else None


def render_split(render_part, width, height, spp, rank, world, split="spp", device="cpu"):
    """One image split over `world` ranks; every rank returns the whole image [height, width, 3].

    The reference's engine splits one image over host threads by pixel (an atomic pixel counter,
    graphics_engine.cpp:49-56,73-74); across GPUs the units are pixel tiles or sample ranges:

      split="tiles": rank r renders the pixels shard(width*height, r, world) with all samples. The
        tiles are exactly those pixels of a one-rank render (same random numbers, same per-pixel sum
        in sample order), and one all_gather assembles them: the result is bit-identical.
      split="spp": rank r renders the samples shard(spp, r, world) of every pixel, scaled by the
        whole image's 1/spp, and one all_reduce(sum) adds the ranks' images: the one-rank image up
        to the float summation order of the per-pixel sums.

    render_part(pixel_begin, pixel_count, sample_begin, sample_count) returns that part as a float32
    tensor [pixel_count, 3] on `device` (for a Scene: scene_part_renderer). A rank whose share is
    empty contributes zeros and does not call it. Every rank makes the same collective calls."""
    import torch
    npix = width * height
    if split == "tiles":
        lo, hi = shard(npix, rank, world)
        size = -(-npix // world)  # tiles padded to the largest share for the all_gather
        tile = torch.zeros((size, 3), dtype=torch.float32, device=device)
        if hi > lo:
            tile[:hi - lo] = render_part(lo, hi - lo, 0, spp)
        d = _dist()
        if d is None:
            parts = [tile]
        else:
            parts = [torch.empty_like(tile) for _ in range(world)]
            d.all_gather(parts, tile)
        img = torch.cat([p[:shard(npix, r, world)[1] - shard(npix, r, world)[0]] for r, p in enumerate(parts)])
        return img.reshape(height, width, 3)
    if split == "spp":
        s0, s1 = shard(spp, rank, world)
        img = torch.zeros((npix, 3), dtype=torch.float32, device=device)
        if s1 > s0:
            img += render_part(0, npix, s0, s1 - s0)
        d = _dist()
        if d is not None:
            d.all_reduce(img)
        return img.reshape(height, width, 3)
    raise ValueError("split must be 'tiles' or 'spp', not %r" % (split,))


def adjoint_split(adjoint_part, spp, rank, world, shapes, device="cpu", dtype=None):
    """The gradient of one image split over ranks by sample range: rank r computes the share of
    the samples shard(spp, r, world) (each weighted by the whole image's 1/spp), and one
    all_reduce(sum) per gradient tensor gives every rank the whole image's gradient.
    adjoint_part(sample_begin, sample_count) returns a tuple of tensors of `shapes` (float32 unless
    dtype says otherwise)."""
    import torch
    s0, s1 = shard(spp, rank, world)
    if s1 > s0:
        grads = [g.contiguous() for g in adjoint_part(s0, s1 - s0)]
    else:
        grads = [torch.zeros(sh, dtype=dtype or torch.float32, device=device) for sh in shapes]
    d = _dist()
    if d is not None:
        for g in grads:
            d.all_reduce(g)
    return tuple(grads)


def scene_part_renderer(scene, cam, width, height, spp, depth, seed=0, stream=None, **render_kw):
    """render_part for render_split over a master_thesis_b200.Scene on this rank's GPU: the
    library renders the requested pixels and samples of the image (swr_render_opts pixel_begin,
    pixel_count, sample_begin, spp_total)."""
    def part(pixel_begin, pixel_count, sample_begin, sample_count):
        return scene.render(cam, width, height, sample_count, depth, seed=seed, stream=stream,
                            pixel_begin=pixel_begin, pixel_count=pixel_count, sample_begin=sample_begin,
                            spp_total=spp, **render_kw).reshape(pixel_count, 3)
    return part
