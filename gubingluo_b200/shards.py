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


def migrate_sharded(survey: SurveyConfig, options, shots, vp, rho, gathers=None, vp_mig=None, rho_mig=None,
                    dist=None, migrate_fn=None) -> dict:
    """Migrate `shots` over the ranks of the default torch.distributed process group, one
    process per GPU (`options.device` = the rank's GPU): every rank computes the same
    longest-processing-time partition, migrates its own shots, and one all-reduce per image
    sums the stacked images, which every rank then returns.  `gathers` (mode 1) lists every
    shot's gather in the order of `shots`, on every rank (each rank uploads only its own).
    With `dist` None, or a world of one, it is `migrate` on all the shots.

    The images travel through the rank's GPU for an NCCL group and stay on the host for gloo;
    in mode 0 each rank returns the gathers of its own shots (`shots_of_rank`, in that order).
    The sums over ranks add the ranks' stacked images in rank order, not shot by shot, so the
    result equals a single-process run's to within the images' rounding, not bit for bit.
    `migrate_fn(survey, options, shots, vp, rho, gathers, vp_mig, rho_mig)` replaces the
    library's `migrate` (the CPU tests pass the oracle there).  Every rank must call this with
    the same arguments; a rank that fails before the reduction makes the others' reduction
    fail with an error (or time out with the process group's timeout) rather than wait."""
    import numpy as np

    if migrate_fn is None:
        from . import migrate as migrate_fn
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    parts = lpt_shards(shot_costs(survey, shots), world)
    idx = parts[rank]
    mine = [shots[i] for i in idx]
    if mine:
        out = dict(migrate_fn(survey, options, mine, vp, rho, None if gathers is None else [gathers[i] for i in idx],
                              vp_mig, rho_mig))
    else:   # more ranks than shots: this rank adds zeros
        z = np.zeros((survey.nz, survey.nx), np.float32)
        out = {k: z.copy() for k in ("image1", "image2s", "image2m", "illum")}
        if getattr(options, "accum_fp64", 0):
            out["f64"] = {k: np.zeros((survey.nz, survey.nx)) for k in ("image1", "image2s", "illum")}
        if getattr(options, "extra_images", 0):
            for k in ("image3s", "image4s", "image5s", "image3m", "image4m", "image5m", "imagetrue"):
                out[k] = z.copy()
        if survey.mode == 0:
            out["gathers"] = []
    out["shots_of_rank"] = mine
    if world == 1:
        return out
    import torch

    dev = f"cuda:{options.device}" if dist.get_backend() == "nccl" else "cpu"

    def reduced(a):   # on a copy: the caller's arrays (which may alias each other) stay as they were
        t = torch.tensor(np.asarray(a), device=dev)
        dist.all_reduce(t)
        return t.cpu().numpy()

    # the same keys in the same order on every rank: every image is a sum over shots
    for k in sorted(k for k, v in out.items() if k.startswith(("image", "illum")) and isinstance(v, np.ndarray)):
        out[k] = reduced(out[k])
    if "f64" in out:
        out["f64"] = {k: reduced(out["f64"][k]) for k in sorted(out["f64"])}
    return out
