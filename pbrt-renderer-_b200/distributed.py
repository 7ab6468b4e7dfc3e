"""Multi-GPU rendering of one frame: sample-range sharding and the film reduce.

Paths are independent, so a frame shards by sample index: with N ranks, rank
r renders every pixel with samples [(f*N + r)*spp, (f*N + r + 1)*spp) of frame
f, which together cover [f*N*spp, (f+1)*N*spp) exactly once.  The reference
renders one sample per pixel per DispatchRays and advances the frame counter
(src/gpu/DXRApp.cpp:84-118, the Sobol sample index of shaders/RNG.hlsli);
the ranks here split that counter between them.

A rank's film is one contiguous float32 buffer of shape (2, H, W, 4): [0] the
running sum of (L, 1) per pixel, [1] its Kahan compensation (the value is
sum - comp).  Keeping both halves in one buffer makes the reduce a single
collective; the ranks' corrected sums add linearly.
"""

from __future__ import annotations


def sample_offset(frame: int, rank: int, world: int, spp: int) -> int:
    """First sample index of `rank` for `frame` (spp samples per rank)."""
    if not (0 <= rank < world) or spp <= 0 or frame < 0:
        raise ValueError(f"bad shard: frame={frame} rank={rank} world={world} spp={spp}")
    return (frame * world + rank) * spp


def new_film(height: int, width: int, device=None):
    """A zeroed (2, H, W, 4) float32 film buffer (sum, compensation)."""
    import torch

    return torch.zeros((2, height, width, 4), dtype=torch.float32, device=device)


def all_reduce_film(film, group=None):
    """Sum the films of all ranks in place (one collective: sum and
    compensation travel together)."""
    import torch.distributed as dist

    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    return film


def resolve(film):
    """Per-pixel mean radiance (H, W, 3) of a (2, H, W, 4) film: the Kahan-
    corrected sum divided by its sample count (the reference's accum.xyz /
    accum.w, src/gpu/DXRApp_Camera.cpp:334-399)."""
    v = film[0] - film[1]
    w = v[..., 3:4]
    return v[..., :3] / w.clamp_min(1.0)


def render_shard(ctx, params_for_offset, film, frame: int, rank: int, world: int, spp: int):
    """Render this rank's share of `frame` into the device film (2, H, W, 4)
    through the C ABI (added to what the film holds); `params_for_offset(offset)`
    builds pt_render_params."""
    P = params_for_offset(sample_offset(frame, rank, world, spp))
    mem_device = 1  # PT_MEM_DEVICE
    return ctx.render(P, film[0].data_ptr(), film[1].data_ptr(), mem_device)


def device_renderer(ctx):
    """`render_into(params, film)` for render_frame: libpt renders into a
    device film (2, H, W, 4), adding to it."""
    mem_device = 1  # PT_MEM_DEVICE

    def render_into(P, film):
        return ctx.render(P, film[0].data_ptr(), film[1].data_ptr(), mem_device)

    return render_into


def render_frame(render_into, params_for_offset, acc, frame: int, rank: int, world: int, spp: int,
                 shard=None, group=None, host_acc=None):
    """One frame of world x spp samples per pixel, added to the accumulated
    film `acc` (2, H, W, 4) exactly once.

    With one rank the samples are rendered straight into `acc`.  With more,
    each rank renders its sample range into its own film `shard` (same shape
    as acc), the shards are summed over the ranks with one all-reduce (the
    path's only exchange step), and the frame's sum is added to `acc`, so
    after F frames every rank's acc holds samples [0, F x world x spp) once
    each.  (Reducing an accumulating film in place would count the earlier
    frames again at every step.)

    `host_acc` (optional, pinned host memory of acc's shape) makes the step
    end to end: the accumulated film is copied host -> device into the
    rank-0 shard before the render and the reduced result device -> host
    after it (rank 0; the other ranks' shards start at zero), which leaves
    host_acc = host_acc + the frame and `acc` unused.

    `render_into(params, film)` renders into `film` (adding to it) and
    returns the render's statistics."""
    P = params_for_offset(sample_offset(frame, rank, world, spp))
    if world == 1 and host_acc is None:
        return render_into(P, acc)
    if shard is None:
        raise ValueError("render_frame: world > 1 (or a host film) needs a shard film")
    if host_acc is not None and rank == 0:
        shard.copy_(host_acc, non_blocking=True)
    else:
        shard.zero_()
    st = render_into(P, shard)
    all_reduce_film(shard, group)
    if host_acc is not None:
        if rank == 0:
            host_acc.copy_(shard, non_blocking=True)
    else:
        acc.add_(shard)
    return st
