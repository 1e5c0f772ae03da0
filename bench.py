#!/usr/bin/env python
"""Benchmark of the B200 RTM path: shots/s (and Gcell-updates/s) of 2-D acoustic prestack
reverse-time migration on the 64-shot full-spread survey of benchmark configuration 2
(1701 x 351 grid, dx = dz = 12.5 m, 50-cell PML, nt = 4000, 15 Hz Ricker,
source-illumination-normalised imaging), synthetic seeded model.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step migrates --shots-per-step shots per GPU as one batch (default 64: the whole survey;
mode 1: recorded gathers in, stacked images out).  `value` times K steps with the gathers already resident in device memory; `e2e` times
K steps through the same public C-ABI with each step's gathers copied from pinned host memory
and the stacked image read back.  Under torchrun each rank migrates its own shots (weak
scaling); the ranks' partial images are summed with one NCCL all-reduce after the timed
steps (inside the timed region).

--impl reference times the reference's CPU path on the host cores.  The reference has no CPU
implementation of the stencil or imaging (its host code is serial model preparation and file
I/O), so this arm runs the CPU restatement of its algorithm (oracle/, FP32, OpenMP on all host
threads) on a bounded sample: the survey's shot of median cell-updates, for
--cpu-sample-steps time steps, scaled to shots/s of the full nt at the survey's mean
cell-updates per shot.  --config N (1-5) selects another benchmark configuration; its
per-shot windows (configuration 4 draws each shot's aperture) are used by both arms.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = ("config 2: 1701x351 grid (X x Z = 1801 x 451 padded), dx=dz=12.5 m, 50-cell PML, nt=4000, "
            "dt=1 ms, 15 Hz Ricker, 64 full-spread shots every 25 grid points, source-illumination-"
            "normalised imaging, FP32 stencil/strips/gathers/accumulators")

MODEL_TEXT = {1: "four flat layers and a dipping 3500 m/s wedge",
              2: "gradient + random-field + thrust-fault",
              3: "gradient + random-field + thrust-fault",
              4: "gradient + random-field",
              5: "gradient + salt body + water layer"}


# per-shot image accumulation (rtm_options.accum_fp64) chosen by the flags, and its description
ACCUM_TEXT = {0: "FP32", 1: "FP64", 2: "compensated FP32 pair (Kahan)",
              3: "FP64 totals of 32-step FP32 partial sums"}


def accum_mode(args) -> int:
    return 2 if args.accum_kahan else 3 if args.accum_blocked else 1 if args.accum_fp64 else 0


def workload_text(args, s, shots, meta):
    """The workload of a --config run (configuration 2's text is WORKLOAD)."""
    fp32 = args.strips == "fp32" and args.gathers == "fp32" and accum_mode(args) == 0
    if args.config == 2 and s.nt == 4000 and fp32:
        return WORKLOAD
    X, Z = s.nx + 2 * s.npml, s.nz + 2 * s.npml
    if "apertures" in meta:
        ap = meta["apertures"].values()
        spread = (f"layout {s.layout}, each shot's aperture drawn from {min(ap)}-{max(ap)} columns and cut at "
                  f"the model's edges")
    else:
        spread = "full spread" if s.layout == 2 else f"layout {s.layout}"
    form = "FP32 stencil/strips/gathers/accumulators" if fp32 else (
        f"FP32 stencil, {args.strips} strips, {args.gathers} gathers, "
        f"{ACCUM_TEXT[accum_mode(args)]} accumulators")
    return (f"config {args.config}: {s.nx}x{s.nz} grid (X x Z = {X} x {Z} padded), dx=dz={s.dx:g} m, "
            f"{s.npml}-cell PML, nt={s.nt}, dt={s.dt * 1e3:g} ms, {s.fdom:g} Hz Ricker, {len(shots)} shots "
            f"({spread}), source-illumination-normalised imaging, {form}")


def data_text(n, meta):
    return (f"synthetic (seeded {MODEL_TEXT[n]} model of configuration {n}; gathers modelled in the true model "
            f"by this library before timing; migration in the {meta['smooth_m']:g} m-smoothed model)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--shots-per-step", type=int, default=64,
                    help="shots per step and GPU, run as one batch (default: the whole 64-shot survey)")
    ap.add_argument("--batch", type=int, default=0, help="shots per launch (0: all shots of a step)")
    ap.add_argument("--nt", type=int, default=0, help="override nt (quick runs only)")
    ap.add_argument("--strips", default="fp32", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--gathers", default="fp32", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--accum-fp64", action="store_true")
    ap.add_argument("--accum-kahan", action="store_true",
                    help="per-shot accumulation in compensated fp32 pairs, stacked in fp64")
    ap.add_argument("--accum-blocked", action="store_true",
                    help="per-shot accumulation in fp64 totals of 32-step fp32 partial sums, stacked in fp64")
    ap.add_argument("--cpu-sample-steps", type=int, default=500)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="model", choices=["model", "real"],
                    help="real: the recorded-data path (SU file -> resampling -> mute -> migration), one GPU")
    ap.add_argument("--profile-only", action="store_true",
                    help="run --steps steps and exit (for ncu launch lists)")
    ap.add_argument("--no-headline", action="store_true",
                    help="skip the configuration-4 comparison (batched mixed precision against plain "
                         "FP32 one shot per launch) that the N=1 line carries")
    ap.add_argument("--headline-only", action="store_true", help="run only the configuration-4 comparison")
    ap.add_argument("--headline-sample", type=int, default=8,
                    help="plain per-shot arm: every k-th shot of the 256 (default 8: 32 shots)")
    ap.add_argument("--headline-arms", default="batched,plain,graph",
                    help="which arms of the configuration-4 comparison to run (comma-separated)")
    ap.add_argument("--headline-accum", type=int, default=3, choices=[1, 2, 3],
                    help="image accumulation of the batched arm (rtm_options.accum_fp64; default 3: fp64 "
                         "totals of 32-step fp32 partial sums)")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd[1:1] = ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        load = [r for r in rows if r["power"] > 250.0] or rows
        reasons = set()
        for r in load:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(load)}


def measured_hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_per_unit(kernel: str, X: int, Z: int):
    """DRAM bytes per padded cell of one launch of `kernel` on an X x Z grid from the committed
    ncu summary (profiles/ncu_<kernel>_<X>x<Z>.txt, line 'dram_bytes_per_cell=<float>'), or
    None when no capture of that kernel on that grid is committed."""
    path = os.path.join(ROOT, "profiles", f"ncu_{kernel}_{X}x{Z}.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_cell="):
            return float(line.split("=", 1)[1])
    return None


# ------------------------------------------------------------------------------------------
# kernel families timed by the session (split kernels; whole-step kernel)
KERNEL_FAMILIES = ("vel_fwd", "pres_fwd", "vel_recon", "pres_recon", "vel_recv", "pres_recv", "step_fwd", "step_recon",
                   "step_recv", "pass_fwd", "pass_bwd")
# the other kernels of a step, timed the same way and reported beside the stencil families
# (strip_pack runs once per 32 source-pass steps, image_flush once per 32 backward steps)
AUX_FAMILIES = ("strip_save", "strip_pack", "image_flush")


def kernel_bytes(kind: str, X: int, Z: int, nxi: int, nzi: int, nrec: int, accum_bytes: int, nt: int = 1) -> float:
    """Algorithmic DRAM bytes of one launch of `kind` for one shot: every array the kernel
    must read or write, once (4-byte fields).
      vel_fwd, vel_recv:   read p, 1/rho; read+write vx, vz            24 B per padded cell
      pres_fwd, pres_recv: read vx, vz, kappa; read+write p            20 B per padded cell
                           + in the PML band (padded minus interior cells) the split parts
                           sx, sz read and written, the old p not read: +12 B per band cell
      vel_recon:  read ps, 1/rho; read+write vxs, vzs on the interior  24 B per interior cell
      pres_recon: read vxs, vzs, kappa; read+write ps on the interior  20 B per interior cell
      pres_recv adds the imaging: read ps, read+write g1 and illum     4 + 4*accum B per interior cell
      step_fwd, step_recv (whole step): read p, vx, vz, 1/rho, kappa; write p, vx, vz   32 B per padded cell
                           + sx, sz read and written in the band       +16 B per band cell
      step_recon: the same on the interior, with both strip sets       32 B per interior cell
    plus the boundary strips the reconstruction kernels read (the forward strips are written
    by a separate copy kernel).  pass_fwd / pass_bwd (persistent passes, one launch per pass of
    nt steps): the per-step kernels' bytes times the steps, with the strip saves."""
    cells, inner = X * Z, nxi * nzi
    band = cells - inner
    strips = 80 * (nxi + nzi)   # vx+vz or p strips of one step, fp32
    table = {
        "vel_fwd": 24 * cells,
        "pres_fwd": 20 * cells + 12 * band,
        "vel_recon": 24 * inner + strips,
        "pres_recon": 20 * inner + strips,
        "vel_recv": 24 * cells,
        "pres_recv": 20 * cells + 12 * band + (4 + 4 * accum_bytes) * inner + 4 * nrec,
        # whole-step kernel: read p, vx, vz, 1/rho, kappa; write p, vx, vz once per cell
        "step_fwd": 32 * cells + 16 * band,
        "step_recon": 32 * inner + 2 * strips,
        "step_recv": 32 * cells + 16 * band + (4 + 4 * accum_bytes) * inner + 4 * nrec,
    }
    # persistent passes (one launch per pass): the per-step kernels' bytes times the steps
    table["pass_fwd"] = nt * (table["vel_fwd"] + table["pres_fwd"] + 8 * 40 * (nxi + nzi))
    table["pass_bwd"] = (nt - 1) * (table["vel_recon"] + table["pres_recon"] + table["vel_recv"] + table["pres_recv"])
    return table[kind]


class _CudaArray:
    """__cuda_array_interface__ view of a device pointer (for torch.distributed)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def run_ours(args, rank, world, local_rank):
    import torch
    import gubingluo_b200 as G
    from gubingluo_b200 import synthetic

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    s, all_shots, v_true, v_mig, rho, meta = synthetic.config(args.config, nt=args.nt or None)
    B = args.shots_per_step
    K, W = args.steps, args.warmup
    # per-shot windows when the configuration draws each shot's aperture (else the layout's)
    s_mig = G.SurveyConfig(**{**s.__dict__, "mode": 1})
    geo_list = synthetic.shot_geometries(s_mig, all_shots, meta)
    geo_of = None if geo_list is None else dict(zip(all_shots, geo_list))

    def geoms_for(shots):
        return None if geo_of is None else [geo_of[sh] for sh in shots]
    # this rank's shots: longest-processing-time partition of the survey by shot cost
    # (nt * X * Z), repeated as needed to fill the steps
    from gubingluo_b200 import shards
    parts = shards.lpt_shards(shards.shot_costs(s_mig, all_shots, geo_list), world)
    mine = [all_shots[i] for i in parts[rank]] or all_shots[:1]
    need = B * (K + W)
    uniq = mine[: min(len(mine), need)]
    step_shots = [uniq[(i * B + j) % len(uniq)] for i in range(K + W) for j in range(B)]
    opts = G.RunOptions(device=local_rank, strip_precision=args.strips, gather_precision=args.gathers,
                        accum_fp64=accum_mode(args), batch=args.batch or B)
    # ---- synthetic data: model this rank's gathers in the true model (untimed setup)
    t0 = time.time()
    s_model = G.SurveyConfig(**{**s.__dict__, "mode": 0})
    with G.Session(s_model, G.RunOptions(device=local_rank, batch=min(len(uniq), 32)), uniq, v_true, rho,
                   geometries=geoms_for(uniq)) as ms:
        ms.model()
        gathers = {sh: ms.gather(k) for k, sh in enumerate(uniq)}
    t_data = time.time() - t0
    # ---- migration session: the session holds every shot the steps use (inputs resident)
    ss = G.Session(s_mig, opts, step_shots, v_mig, rho, geometries=geoms_for(step_shots))
    for k, sh in enumerate(step_shots):
        ss.set_gather(k, gathers[sh])
    # shot windows differ in layouts 1, 3, 4 and with per-shot apertures
    geos = {sh: (G.geometry(s_mig, sh) if geo_of is None else geo_of[sh]) for sh in set(step_shots)}
    geo = geos[step_shots[0]]
    X, Z, nxi, nzi, nrec = geo.nxpad, geo.nzpad, geo.nxlength, s.nz, geo.nrec

    def w_of(sh):   # cell-updates of one shot: source pass, reconstruction, receiver pass
        g = geos[sh]
        return s.nt * (2.0 * g.nxpad * g.nzpad + g.nxlength * s.nz)
    stream = torch.cuda.ExternalStream(ss.stream())
    ptrs = ss.image_ptrs()
    npix = s.nx * s.nz
    typestr = "<f8" if accum_mode(args) else "<f4"
    img_views = [torch.as_tensor(_CudaArray(ptrs[k], npix, typestr), device=f"cuda:{local_rank}")
                 for k in ("image1", "image2s", "illum")] if dist else []

    def reduce_images():
        # the one exchange step: sum of the ranks' stacked images, after all of their shots
        if dist:
            with torch.cuda.stream(stream):
                shards.allreduce_images(img_views, dist)

    def step(i):
        return ss.run_range(i * B, B)

    for i in range(W):
        step(i)
    ss.reset_images()   # the images of the timed run hold the timed shots only
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    batches = 1
    for i in range(W, W + K):
        st = step(i)
        launches += st.kernel_launches
        batches = max(batches, st.batches)
    reduce_images()
    e1.record(stream)
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    if dist:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    kern = {k: ss.kernel_ms(k) for k in KERNEL_FAMILIES}
    aux = {k: round(v[0], 4) for k, v in ((k, ss.kernel_ms(k)) for k in AUX_FAMILIES) if v[0] > 0}
    tiles = ss.tile_heights()
    if args.profile_only:
        ss.close()
        return None
    t_max = torch.tensor([ms_total], dtype=torch.float64, device=f"cuda:{local_rank}")
    if dist:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_total = float(t_max.item())
    shots_done = K * B * world
    value = shots_done / (ms_total * 1e-3)
    w_timed = sum(w_of(sh) for sh in step_shots[W * B:(W + K) * B])   # this rank's timed shots
    gcell = world * w_timed / (ms_total * 1e-3) * 1e-9

    # ---- e2e: the same steps through the public API with host-resident inputs
    e2e = None
    if not args.no_e2e:
        host = {}
        for sh in set(step_shots):
            t = torch.empty((s.nt, geos[sh].nrec), dtype=torch.float32, pin_memory=True)
            t.numpy()[:] = gathers[sh]
            host[sh] = t
        img_host = torch.empty((s.nz, s.nx), dtype=torch.float32, pin_memory=True)
        # bytes per step: the timed steps' gathers (their receiver counts differ with the window)
        h2d = sum(host[sh].numel() * 4 for sh in step_shots[W * B:(W + K) * B]) // K
        d2h = s.nz * s.nx * 4
        ss.reset_images()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(W, W + K):
            for j in range(B):
                k = i * B + j
                G._check(G.lib().rtm_session_set_gather(ss.h, k, host[step_shots[k]].data_ptr()))
            step(i)
            G._check(G.lib().rtm_session_get_images(ss.h, None, img_host.data_ptr(), None, None))
        reduce_images()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1)
        t_max = torch.tensor([ms_e2e], dtype=torch.float64, device=f"cuda:{local_rank}")
        if dist:
            dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        ms_e2e = float(t_max.item())
        e2e = {"value": shots_done / (ms_e2e * 1e-3), "unit": "shots/s", "h2d_bytes_per_step": h2d * world,
               "d2h_bytes_per_step": d2h * world, "ms_per_step": ms_e2e / K}
    ss.close()

    # ---- roofline of the dominant kernel
    # bytes per accumulator cell that the receiver pressure kernel reads and writes (the blocked
    # form's kernel updates fp32 partials; its flush is a launch of its own)
    accum_bytes = 8 if accum_mode(args) in (1, 2) else 4
    sampled = {k: v for k, v in kern.items() if v[0] > 0}
    dom = max(sampled, key=lambda k: sampled[k][0])
    launch_ms = sampled[dom][0]
    nshots_launch = -(-B // batches)   # the step's shots run in `batches` launches per kernel and step
    # algorithmic bytes of the first launch of a timed step: each shot's own window
    first = step_shots[W * B:W * B + nshots_launch]
    bytes_launch = sum(kernel_bytes(dom, geos[sh].nxpad, geos[sh].nzpad, geos[sh].nxlength, s.nz, geos[sh].nrec,
                                    accum_bytes, s.nt) for sh in first)
    achieved = bytes_launch / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    per_cell = ncu_traffic_per_unit(dom, X, Z)
    roofline = {"kernel": f"k_{dom}", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": None if per_cell is None else round(per_cell * sum(geos[sh].nxpad * geos[sh].nzpad
                                                                              for sh in first)),
                "algorithmic_bytes_per_launch": int(bytes_launch), "launch_ms": round(launch_ms, 4),
                "launches_sampled": sampled[dom][1],
                "kernel_ms": {k: round(v[0], 4) for k, v in sampled.items()},
                # every family's algorithmic bytes per launch / its mean event time, of the same peak
                "kernel_frac": {k: round(sum(kernel_bytes(k, geos[sh].nxpad, geos[sh].nzpad, geos[sh].nxlength, s.nz,
                                                          geos[sh].nrec, accum_bytes, s.nt) for sh in first)
                                         / (v[0] * 1e-3) / 1e9 / peak, 4) for k, v in sampled.items()},
                "aux_kernel_ms": aux}
    return dict(value=value, gcell=gcell, ms_total=ms_total, launches=launches, e2e=e2e, roofline=roofline, tiles=tiles,
                clocks=clock_info, shots_done=shots_done, t_data=t_data, X=X, Z=Z, nxi=nxi, nzi=nzi, nrec=nrec,
                w_shot=w_timed / (K * B), s=s, shots_per_launch=nshots_launch, meta=meta, all_shots=all_shots)


# ------------------------------------------------------------------------------------------
def run_headline(args, local_rank):
    """Configuration 4 (3201 x 801 grid, 10 m, 40-cell PML, nt = 5000 at 0.8 ms, 20 Hz; 256
    shots whose apertures are drawn from 201-801 columns), two arms on the same GPU:

      batched: all 256 shots in one session, as many per launch as device memory holds,
               fp16 boundary strips and gathers, fp64 image accumulation;
      plain per-shot: plain FP32 (strips, gathers, accumulators), one shot per launch, on
               every k-th shot of the survey (--headline-sample; the apertures are drawn
               independently of the shot number, so the sample has the survey's spread),
               timed with direct launches and with each pass's time loop replayed as a CUDA
               graph.

    Both are timed with CUDA events on the session stream, gathers resident.  The ratio is
    taken at equal work per shot: Gcell-updates/s of the batched arm over that of the faster
    per-shot arm, direct launches or graph replays (= shots/s over shots/s when both arms'
    shots have the same mean size).
    The image error of both forms against the FP64 oracle is tested in
    tests/test_gpu_configs.py (narrowest and widest aperture, full nt)."""
    import torch
    import gubingluo_b200 as G
    from gubingluo_b200 import synthetic

    torch.cuda.set_device(local_rank)
    s, shots, v_true, v_mig, rho, meta = synthetic.config(4, nt=args.nt or None)
    s_mig = G.SurveyConfig(**{**s.__dict__, "mode": 1})
    geo_of = dict(zip(shots, synthetic.shot_geometries(s_mig, shots, meta)))

    def w_of(sh):
        g = geo_of[sh]
        return s.nt * (2.0 * g.nxpad * g.nzpad + g.nxlength * s.nz)
    t0 = time.time()
    s_model = G.SurveyConfig(**{**s.__dict__, "mode": 0})
    gathers = {}
    for k0 in range(0, len(shots), 64):
        part = shots[k0:k0 + 64]
        with G.Session(s_model, G.RunOptions(device=local_rank, batch=64), part, v_true, rho,
                       geometries=[geo_of[sh] for sh in part]) as ms:
            ms.model()
            for k, sh in enumerate(part):
                gathers[sh] = ms.gather(k)
    t_data = time.time() - t0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(opts, arm_shots, warm):
        ss = G.Session(s_mig, opts, arm_shots, v_mig, rho, geometries=[geo_of[sh] for sh in arm_shots])
        for k, sh in enumerate(arm_shots):
            ss.set_gather(k, gathers[sh])
        stream = torch.cuda.ExternalStream(ss.stream())
        # the tuner's trials for the launch shapes of the timed run, then a short warm-up
        ss.prepare(0, len(arm_shots))
        ss.run_range(0, warm)
        ss.reset_images()
        torch.cuda.synchronize()
        e0.record(stream)
        st = ss.run_range(0, len(arm_shots))
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        kern = {k: round(v[0], 4) for k, v in ((k, ss.kernel_ms(k)) for k in KERNEL_FAMILIES + AUX_FAMILIES)
                if v[0] > 0}
        tiles = ss.tile_heights()
        ss.close()
        w = sum(w_of(sh) for sh in arm_shots)
        return {"shots": len(arm_shots), "seconds": round(ms * 1e-3, 3),
                "shots_per_s": round(len(arm_shots) / (ms * 1e-3), 4),
                "gcell_updates_per_s": round(w / (ms * 1e-3) * 1e-9, 3),
                "mean_cell_updates_per_shot": w / len(arm_shots), "batches": st.batches,
                "kernel_launches": st.kernel_launches, "kernel_ms": kern, "tile_rows": tiles}

    arms = set(args.headline_arms.split(","))
    empty = {"shots": 0, "shots_per_s": None, "gcell_updates_per_s": None}
    batched = timed(G.RunOptions(device=local_rank, strip_precision="fp16", gather_precision="fp16",
                                 accum_fp64=args.headline_accum), shots, 4) if "batched" in arms else empty
    sample = shots[args.headline_sample // 2::args.headline_sample]
    # plain FP32, one shot per launch: direct launches, and each pass replayed as a CUDA graph
    # (rounded grids, so that shots of nearby windows share a graph; every shot here has its
    # own window, and a graph per exact shape would be captured once per shot)
    plain = timed(G.RunOptions(device=local_rank, batch=1), sample, 1) if "plain" in arms else empty
    plain_graph = timed(G.RunOptions(device=local_rank, batch=1, use_graph=2), sample, 1) \
        if "graph" in arms else empty
    best = max((a for a in (plain, plain_graph) if a["shots"]), key=lambda a: a["gcell_updates_per_s"],
               default=None)
    ap = meta["apertures"]
    return {"workload": ("config 4: 3201x801 grid (10 m), 40-cell PML, nt=%d, dt=0.8 ms, 20 Hz Ricker, 256 shots, "
                         "apertures drawn from %d-%d columns (layout-1 windows cut at the model's edges), "
                         "gradient + random-field model, gathers modelled by this library before timing"
                         % (s.nt, min(ap.values()), max(ap.values()))),
            "batched_mixed": {**batched, "form": "fp16 strips + fp16 gathers + %s images, all 256 shots, "
                                                   "in equal launches of as many as fit"
                                                   % ACCUM_TEXT[args.headline_accum]},
            "plain_fp32_per_shot": {**plain, "form": "fp32, one shot per launch, direct launches",
                                    "sample": f"every {args.headline_sample}th shot ({len(sample)} shots)"},
            "plain_fp32_per_shot_graph": {**plain_graph, "form": "fp32, one shot per launch, each pass replayed as "
                                                               "a CUDA graph (rounded grids)",
                                          "sample": "the same shots"},
            "ratio": (round(batched["gcell_updates_per_s"] / best["gcell_updates_per_s"], 3)
                      if batched["shots"] and best else None),
            "ratio_denominator": "the faster of the two plain per-shot arms",
            "ratio_basis": "Gcell-updates/s (shots/s at equal work per shot)",
            "target": 3.0, "setup_seconds_data_modelling": round(t_data, 2)}


# ------------------------------------------------------------------------------------------
REAL_WORKLOAD = ("recorded-data path on the configuration-2 model (1701x351, dx=dz=12.5 m, 50-cell PML, nt=4000 at "
                 "1 ms): 64 off-end shots every 200 m, 241 receivers from 0 to 6000 m every 25 m, 2000 samples at "
                 "2 ms, one SU file; per shot F-K (x2) + windowed-sinc (x2) resampling to 481 traces x 4000 samples, "
                 "direct-wave mute in the migration model, migration in a 481-cell window (581 x 451 padded)")


def run_real(args, rank, world, local_rank):
    """--workload real: `value` = migration of the resampled gathers (resident in device
    memory); `e2e` = the whole recorded-data flow per step through the public API: scan of the
    SU file, trace reading, upload + resampling + mute (rtm_session_set_gather_raw),
    migration, stacked image read back."""
    if rank != 0:
        return
    import torch
    import gubingluo_b200 as G
    from gubingluo_b200 import synthetic

    torch.cuda.set_device(local_rank)
    s, _, v_true, v_mig, rho, _ = synthetic.config(args.config, nt=args.nt or None)
    B, K, W = args.shots_per_step, args.steps, args.warmup
    dx0, dt0, nt0, ntr, spacing = 2 * s.dx, float(np.float32(2 * s.dt)), s.nt // 2, 241, 200.0
    if (B - 1) * spacing + (ntr - 1) * dx0 > (s.nx - 1) * s.dx:
        raise SystemExit("--workload real: the shots do not fit in the model")
    # recorded data (untimed): gathers modelled in the true model on the 12.5 m / 1 ms grid, kept
    # every other receiver and sample, written as one SU file
    t0 = time.time()
    s_mod = G.SurveyConfig(**{**s.__dict__, "mode": 0, "layout": 3, "spx0": 0.0, "dspx": spacing, "offset": 0.0,
                              "offsetmax": (ntr - 1) * dx0})
    ids = list(range(1, B + 1))
    with G.Session(s_mod, G.RunOptions(device=local_rank, batch=min(B, 32)), ids, v_true, rho) as ms:
        ms.model()
        recs = [(spacing * (i - 1), 0, ms.gather(k)[::2, ::2][:nt0]) for k, i in enumerate(ids)]
    tmpd = tempfile.mkdtemp(prefix="rtm_real_bench_")
    path = os.path.join(tmpd, "shots.su")
    synthetic.write_shot_file(path, recs, nt0, dt0, dx0)
    t_data = time.time() - t0
    s_mig = G.SurveyConfig(**{**s.__dict__, "mode": 1, "layout": 3, "mute": 2})
    prof, endian = G.scan_shotgather(path, 0)
    geoms, cols = [], []
    for k in range(B):
        g, nc = G.real_geometry(s_mig, int(prof[0][k]), int(prof[3][k]), int(prof[1][k]), dx0)
        geoms.append(g)
        cols.append(nc)
    X, Z, nxi, nzi, nrec = geoms[0].nxpad, geoms[0].nzpad, geoms[0].nxlength, s.nz, geoms[0].nrec
    w_shot = s.nt * (2.0 * X * Z + nxi * nzi)
    opts = G.RunOptions(device=local_rank, batch=args.batch or B)
    ss = G.Session(s_mig, opts, ids, v_mig, rho, geometries=geoms)
    stream = torch.cuda.ExternalStream(ss.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def load_all():
        p, e = G.scan_shotgather(path, 0)
        for k in range(B):
            obs = G.read_shot_traces(path, 0, e, nt0, int(p[2][k]), int(p[1][k]), cols[k])
            ss.set_gather_raw(k, obs, dt0)

    load_all()
    for _ in range(W):
        ss.run()
    ss.reset_images()
    # resampling alone: upload + F-K + sinc + mute of every shot, CUDA events on the session stream
    obs_all = [G.read_shot_traces(path, 0, endian, nt0, int(prof[2][k]), int(prof[1][k]), cols[k]) for k in range(B)]
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(B):
        ss.set_gather_raw(k, obs_all[k], dt0)
    e1.record(stream)
    torch.cuda.synchronize()
    interp_ms = e0.elapsed_time(e1) / B
    clocks = ClockSampler("GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid))
    torch.cuda.synchronize()
    clocks.start()
    e0.record(stream)
    launches = 0
    for _ in range(K):
        launches += ss.run().kernel_launches
    e1.record(stream)
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    kern = {k: ss.kernel_ms(k) for k in KERNEL_FAMILIES}
    # e2e: file -> images, every step
    img_host = torch.empty((s.nz, s.nx), dtype=torch.float32, pin_memory=True)
    ss.reset_images()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        load_all()
        ss.run()
        G._check(G.lib().rtm_session_get_images(ss.h, None, img_host.data_ptr(), None, None))
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ss.close()
    os.remove(path)
    os.rmdir(tmpd)
    sampled = {k: v for k, v in kern.items() if v[0] > 0}
    dom = max(sampled, key=lambda k: sampled[k][0])
    nsl = min(B, args.batch or B)
    bytes_launch = nsl * kernel_bytes(dom, X, Z, nxi, nzi, nrec, 4)
    achieved = bytes_launch / (sampled[dom][0] * 1e-3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    line = {"metric": "shots/s", "value": K * B / (ms_total * 1e-3), "unit": "shots/s", "n_gpus": 1, "steps": K,
            "warmup": W, "ms_per_step": ms_total / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (configuration-2 model; gathers modelled by this library, decimated "
                                    "to the 25 m / 2 ms data grid and written as an SU file before timing)",
            "config": {"workload": REAL_WORKLOAD, "shots_per_step": B, "shots_per_launch": nsl, "nt": s.nt,
                       "parallelism": "one GPU"},
            "gcell_updates_per_s": K * B * w_shot / (ms_total * 1e-3) * 1e-9,
            "resample_ms_per_shot": round(interp_ms, 3),
            "roofline": {"kernel": f"k_{dom}", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": None, "kernel_ms": {k: round(v[0], 4) for k, v in sampled.items()}},
            "e2e": {"value": K * B / (ms_e2e * 1e-3), "unit": "shots/s",
                    "h2d_bytes_per_step": B * nt0 * max(cols) * 4, "d2h_bytes_per_step": s.nz * s.nx * 4,
                    "ms_per_step": ms_e2e / K},
            "gpu_launches": launches, "clocks": clock_info, "setup_seconds_data_modelling": round(t_data, 2)}
    print(json.dumps(line), flush=True)


def survey_shot_work(s, shots, meta):
    """Oracle geometry of every shot (with its own aperture where the configuration draws
    one) and its cell-updates nt (2 X Z + nxi nzi); shot windows differ in layouts 1, 3, 4."""
    from oracle import oracle as O

    out = []
    for ish in shots:
        om = (meta["apertures"][ish] - 1) * s.dx if "apertures" in meta else s.offsetmax
        g = O.geometry(s.layout, ish, s.nx, s.nz, s.nt, s.dx, s.dz, s.dt, s.npml, s.spx0, s.spz0, s.dspx,
                       s.offset, om)
        out.append((ish, om, s.nt * (2.0 * g.nxpad * g.nzpad + g.nxlength * s.nz)))
    return out


def cpu_sample(args, s, v_mig, rho, shots, meta, w_shot):
    """The CPU restatement of the reference's path (oracle, FP32, OpenMP) on one shot of the
    survey (the one of median cell-updates) for --cpu-sample-steps steps; returns shots/s of
    the full nt at w_shot cell-updates per shot, and the sample."""
    from oracle import oracle as O

    nt_s = args.cpu_sample_steps
    work = sorted(survey_shot_work(s, shots, meta), key=lambda t: (t[2], t[0]))
    ish, om, _ = work[len(work) // 2]
    g = O.geometry(s.layout, ish, s.nx, s.nz, nt_s, s.dx, s.dz, s.dt, s.npml, s.spx0, s.spz0, s.dspx, s.offset,
                   om)
    vp2 = O.pad_model(v_mig, g.nx1, g.nx2, s.npml, True)
    rp = O.pad_model(rho, g.nx1, g.nx2, s.npml, False)
    vpmax = float(np.sqrt(np.float32(vp2.max()), dtype=np.float32))
    sh = O.shot_struct(g.nxpad, g.nzpad, s.npml, nt_s, s.dx, s.dz, s.dt, g.nsx, g.nsz, s.amp, s.alp, s.fdom,
                       s.npml + s.receiver_depth, g.rx0, g.nrec, vpmax)
    data = np.random.default_rng(1).standard_normal((nt_s, g.nrec)).astype(np.float32) * 1e-6
    t0 = time.time()
    O.shot(sh, vp2, rp, mode=1, gather=data, mute=1, nw=int(np.float32(1.5) / (s.fdom * s.dt)), tlength=0)
    sec = time.time() - t0
    cells = nt_s * (2.0 * g.nxpad * g.nzpad + g.nxlength * s.nz)
    gcell = cells / sec * 1e-9
    return {"value": gcell * 1e9 / w_shot, "unit": "shots/s", "cores": O.num_threads(), "kind": "port",
            "gcell_updates_per_s": round(gcell, 4), "seconds": round(sec, 2),
            "sample": f"shot {ish} ({g.nxpad}x{g.nzpad} padded grid) for {nt_s} of {s.nt} time steps (source "
                      f"pass, reconstruction, receiver pass, imaging), scaled to the full nt"}


def run_reference(args, rank):
    if rank != 0:
        return
    from gubingluo_b200 import synthetic

    s, shots, v_true, v_mig, rho, meta = synthetic.config(args.config, nt=args.nt or None)
    # mean cell-updates per shot of the survey
    ws = [w for _, _, w in survey_shot_work(s, shots, meta)]
    w_shot = sum(ws) / len(ws)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_sample(args, s, v_mig, rho, shots, meta, w_shot)
        if i >= args.warmup:
            vals.append(r)
    value = statistics.mean(r["value"] for r in vals)
    sec = statistics.mean(r["seconds"] for r in vals)
    line = {"metric": "shots/s", "value": value, "unit": "shots/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "impl": "reference",
            "data": f"synthetic (seeded model of benchmark configuration {args.config})",
            "config": {"workload": workload_text(args, s, shots, meta), "shots_per_step": "bounded CPU sample"},
            "gcell_updates_per_s": statistics.mean(r["gcell_updates_per_s"] for r in vals),
            "cpu_baseline": {**vals[-1], "value": value},
            "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "real":
        run_real(args, rank, world, local_rank)
        return
    if args.headline_only:
        if rank == 0:
            print(json.dumps({"headline": run_headline(args, local_rank)}), flush=True)
        return
    r = run_ours(args, rank, world, local_rank)
    if r is None or rank != 0:
        return
    s = r["s"]
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from gubingluo_b200 import synthetic

        _, _, _, v_mig, rho, _ = synthetic.config(args.config, nt=args.nt or None)
        cpu = cpu_sample(args, s, v_mig, rho, r["all_shots"], r["meta"], r["w_shot"])
    headline = None
    if world == 1 and not args.no_headline and args.config == 2 and not args.profile_only:
        headline = run_headline(args, local_rank)
    acc_txt = {0: "f32 images", 1: "f64 images", 2: "kahan-f32 images", 3: "f64 images of f32 32-step partials"}[
        accum_mode(args)]
    dtype = "f32" if acc_txt == "f32 images" and args.strips == "fp32" and args.gathers == "fp32" else \
        f"f32 stencil, {args.strips} strips, {args.gathers} gathers, {acc_txt}"
    ws_gb = r["shots_per_launch"] * 12 * r["X"] * r["Z"] * 4 / 1e9
    line = {"metric": "shots/s", "value": r["value"], "unit": "shots/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_total"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": data_text(args.config, r["meta"]),
            "config": {"workload": workload_text(args, s, r["all_shots"], r["meta"]),
                       "shots_per_step_per_gpu": args.shots_per_step,
                       "shots_per_launch": r["shots_per_launch"], "nt": s.nt,
                       "parallelism": f"shots sharded over {world} GPU(s)",
                       "tile_rows": r["tiles"],
                       "l2": f"inputs larger than L2: per-launch wavefield+model working set {ws_gb:.1f} GB vs 126 MB L2"},
            "gcell_updates_per_s": r["gcell"],
            "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "gpu_launches": r["launches"],
            "clocks": r["clocks"], "setup_seconds_data_modelling": round(r["t_data"], 2)}
    if headline is not None:
        line["headline"] = headline
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
