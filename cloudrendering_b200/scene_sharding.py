"""Many independent scenes on several GPUs: scene sharding with longest-processing-time assignment.

Each scene (its own grid, camera, image size, spp and medium) is traced on exactly one rank; nothing
moves between ranks while tracing.  Scenes are assigned by the longest-processing-time rule: in order
of decreasing estimated cost, each goes to the rank with the least assigned cost so far, which keeps
the largest per-rank load within 4/3 of the optimum.  The cost estimate is the expected number of
density lookups: camera paths times (1 + extinction x the mean chord through the unit-extent volume x
the mean normalised density), the work of delta tracking with a global majorant.

`render_scenes_sharded` runs one rank's share through a caller-supplied renderer (for example the
batched persistent launch of `vpt_batch_render` over this rank's contexts) and, if asked, gathers the
results on rank 0 (the only collective, after all tracing is done).
"""
from __future__ import annotations

import heapq
from typing import Callable, Dict, List, Optional, Sequence

import torch.distributed as dist

# mean chord length through the unit cube for uniformly distributed lines (isotropic: 2/3 of the side)
MEAN_CHORD = 2.0 / 3.0


def scene_cost(width: int, height: int, spp: int, extinction: float, mean_density: float = 0.5,
               extent: float = 1.0) -> float:
    """Estimated density lookups of one scene's frames (delta tracking with a global majorant)."""
    if width <= 0 or height <= 0 or spp < 0 or extinction < 0.0:
        raise ValueError("scene_cost: bad image size, spp or extinction")
    return float(width) * float(height) * float(spp) * (1.0 + extinction * MEAN_CHORD * extent * mean_density)


def assign_lpt(costs: Sequence[float], world: int) -> List[List[int]]:
    """Scene indices per rank: longest processing time first, each to the least-loaded rank (ties to
    the lower rank).  Deterministic, so every rank computes the same assignment."""
    if world <= 0:
        raise ValueError("assign_lpt: world size must be > 0")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for lst in out:
        lst.sort()
    return out


def rank_loads(costs: Sequence[float], assignment: Sequence[Sequence[int]]) -> List[float]:
    return [sum(float(costs[i]) for i in lst) for lst in assignment]


def render_scenes_sharded(costs: Sequence[float], render_fn: Callable[[List[int]], Dict[int, object]],
                          group=None, gather: bool = False) -> Optional[Dict[int, object]]:
    """Renders this rank's scenes: `render_fn(indices)` returns {scene index: result}.  With `gather`,
    rank 0 receives every scene's result (all_gather_object after the tracing) and the others None;
    without it, each rank returns its own results."""
    rank = dist.get_rank(group) if dist.is_available() and dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    mine = assign_lpt(costs, world)[rank]
    results = render_fn(mine) if mine else {}
    if not gather or world == 1:
        return results
    parts: List[Optional[Dict[int, object]]] = [None] * world
    dist.all_gather_object(parts, results, group=group)
    if rank != 0:
        return None
    merged: Dict[int, object] = {}
    for p in parts:
        merged.update(p or {})
    return merged
