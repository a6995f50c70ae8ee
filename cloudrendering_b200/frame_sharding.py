"""One image on several GPUs: frame (spp) sharding.

The reference renders on one GPU.  Here each rank (one process per GPU, torch.distributed) renders a
disjoint range of the image's frame indices (vpt_set_frame_index), so all ranks together trace
exactly the paths of one run over all frames: the seed of a path depends only on its frame index and
pixel (Clouds.glsl:80-84).  The ranks' FP64 films are summed by one all_reduce and divided by the
total frame count.  No data moves between ranks while tracing; the final reduction is 3 doubles per
pixel (24 MiB at 1024^2).
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import torch
import torch.distributed as dist


def frame_range(rank: int, world: int, total_frames: int) -> Tuple[int, int]:
    """(first frame, frame count) of `rank`: a balanced split of [0, total_frames)."""
    if world <= 0 or not 0 <= rank < world or total_frames < 0:
        raise ValueError("frame_range: bad rank, world size or frame count")
    base, extra = divmod(total_frames, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def combine_films(film_sum: torch.Tensor, total_frames: int, group=None) -> torch.Tensor:
    """Sums the ranks' FP64 films (in place) and returns the mean image."""
    if film_sum.dtype != torch.float64:
        raise TypeError("combine_films: the film must be float64")
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(film_sum, op=dist.ReduceOp.SUM, group=group)
    return film_sum / float(total_frames)


def render_sharded(total_frames: int, width: int, height: int,
                   render_fn: Optional[Callable[[int, int], torch.Tensor]] = None, group=None) -> torch.Tensor:
    """Mean image [3, H, W] (float64) of `total_frames` frames rendered by all ranks of `group`.
    `render_fn(first, count)` returns this rank's FP64 film sum; by default the vpt module renders it
    on this rank's GPU (the film is moved to the device for an NCCL group)."""
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    first, count = frame_range(rank, world, total_frames)
    if render_fn is None:
        from . import vpt

        def render_fn(first_frame: int, frames: int) -> torch.Tensor:
            vpt.set_frame_index(first_frame)
            out = torch.zeros((3, height, width), dtype=torch.float32, device="cuda")
            if frames > 0:
                vpt.render_frame(out, frames)
            else:
                return torch.zeros((3, height, width), dtype=torch.float64)
            return vpt.get_film_sum(width, height)

    film = render_fn(first, count)
    if dist.is_initialized() and dist.get_backend(group) == "nccl":
        film = film.cuda()
    return combine_films(film, total_frames, group).cpu()
