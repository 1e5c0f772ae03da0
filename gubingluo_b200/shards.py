"""Shot sharding for runs on several GPUs (one process per GPU, torch.distributed).

Shots are independent (the reference loops over them one at a time, rtm_model.cu:117-488),
so a multi-GPU run needs no halo exchange and no domain split: each rank migrates its own
shots into its own image accumulators, and the only collective is one sum of the stacked
images (image1, image2s, illum; image2m equals image1) after the last shot.

The partition is longest-processing-time first on the cost of each shot, nt * X * Z
cell-updates of its padded grid: with layout 1 and per-shot apertures the shot grids differ,
with a fixed spread they are all equal and the partition is round robin.
"""
from __future__ import annotations

from . import SurveyConfig, geometry


def shot_costs(survey: SurveyConfig, shots, geometries=None) -> list:
    """nt * nxpad * nzpad of each shot's padded grid (geometries[k] of shot k when given, as
    for rtm_session_open_geometry; else the survey's layout)."""
    out = []
    for k, ishot in enumerate(shots):
        g = geometry(survey, int(ishot)) if geometries is None else geometries[k]
        out.append(float(survey.nt) * g.nxpad * g.nzpad)
    return out


def lpt_shards(costs, world: int) -> list:
    """Partition shot indices 0..len(costs)-1 over `world` ranks, longest processing time
    first: shots in decreasing cost (ties: lower index first) go one at a time to the rank
    with the least cost so far (ties: lower rank).  Returns one ascending index list per rank;
    the result depends only on the costs and `world`, so every rank computes the same one."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def allreduce_images(tensors, dist) -> None:
    """Sum each rank's accumulated images in place (torch tensors on the rank's device, or on
    the host with gloo).  Call once, after every rank has migrated all of its shots: each
    rank's accumulators must hold only its own shots' contributions, so calling it between
    batches and then accumulating more would count the earlier shots again."""
    if dist is None:
        return
    for t in tensors:
        dist.all_reduce(t)
