"""One rank of the two-rank CPU check of the shot-sharded migration (run by test_shards.py).

Each rank migrates its longest-processing-time shard of the shots with the oracle (FP64 CPU
restatement; the GPU library is not needed here), then the ranks sum their stacked images
over gloo, exactly as the multi-GPU run sums its device images over NCCL.  Rank 0 writes
the reduced images to the output file.

    python tests/_gloo_rank.py <rank> <world> <port> <out.npz> [fail]

With `fail`, the last rank stops after migrating its shots, before the reduction, as a
rank whose process died would; the other ranks' reduction must then end with an error (the
peer's closed connection, at the latest the process group's timeout), not wait for ever.
They exit with status 4 after writing the error to <out.npz>.failed.
"""
import os
import sys
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def survey():
    s = dict(nx=72, nz=36, nt=160, dx=10.0, dz=10.0, dt=1e-3, npml=12, fdom=25.0, amp=1.0, alp=0.1,
             layout=1, spx0=60.0, spz0=10.0, dspx=110.0, offset=0.0, offsetmax=300.0, mode=0,
             medium_flag=0, ismth=0, direct=1.5, direct0=0.0, mute=1, receiver_depth=1)
    zz = np.arange(s["nz"])[:, None] * s["dz"]
    vp = (1500.0 + 1.2 * zz + 0.0 * np.arange(s["nx"])[None, :]).astype(np.float32)
    vp[20:, 30:50] = 2600.0
    rho = np.full_like(vp, 2000.0)
    return s, [1, 2, 3, 4, 5], vp, rho


def main():
    rank, world, port, out = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
    fail = len(sys.argv) > 5 and sys.argv[5] == "fail"
    import torch
    import torch.distributed as dist
    from gubingluo_b200 import SurveyConfig, shards
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = port
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20 if fail else 60))
    s, shots, vp, rho = survey()
    cfg = SurveyConfig(**{k: s[k] for k in SurveyConfig.__dataclass_fields__})
    parts = shards.lpt_shards(shards.shot_costs(cfg, shots), world)
    mine = [shots[i] for i in parts[rank]]
    if mine:
        r = O.rtm_model(s, mine, vp, rho, precision="f64")
        imgs = [r["image1"], r["image2s"], r["illum"]]
    else:
        imgs = [np.zeros((s["nz"], s["nx"])) for _ in range(3)]
    ts = [torch.from_numpy(np.ascontiguousarray(a, np.float64)) for a in imgs]
    if fail and rank == world - 1:
        os._exit(3)   # ends without leaving the process group, like a crashed rank
    try:
        shards.allreduce_images(ts, dist)
    except Exception as e:   # the peer is gone: report and stop
        with open(out + ".failed", "w") as f:
            f.write(f"rank {rank}: {type(e).__name__}: {e}")
        os._exit(4)
    if rank == 0:
        np.savez(out, image1=ts[0].numpy(), image2s=ts[1].numpy(), illum=ts[2].numpy(),
                 parts=np.array([len(p) for p in parts]))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
