"""One rank of the two-rank CPU check of the shot-sharded migration (run by test_shards.py).

Each rank calls the library's `shards.migrate_sharded` over gloo, with the oracle (FP64 CPU
restatement; the GPU library is not needed here) in place of the GPU migration: the
function partitions the shots, the rank migrates its longest-processing-time share, and the
ranks sum their stacked images, as a multi-GPU run sums them over NCCL.  Rank 0 writes the
reduced images to the output file.

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
    import torch.distributed as dist
    from gubingluo_b200 import RunOptions, SurveyConfig, shards
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = port
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20 if fail else 60))
    s, shots, vp, rho = survey()
    cfg = SurveyConfig(**{k: s[k] for k in SurveyConfig.__dataclass_fields__})

    def oracle_migrate(survey_, options, mine, vp_, rho_, gathers, vp_mig, rho_mig):
        r = O.rtm_model(s, mine, vp_, rho_, precision="f64")
        if fail and rank == world - 1:
            os._exit(3)   # after its shots, before the reduction; leaves without a word, like a crash
        return {"image1": r["image1"], "image2s": r["image2s"], "image2m": r["image1"], "illum": r["illum"]}

    try:
        red = shards.migrate_sharded(cfg, RunOptions(), shots, vp, rho, dist=dist, migrate_fn=oracle_migrate)
    except Exception as e:   # the peer is gone: report and stop
        with open(out + ".failed", "w") as f:
            f.write(f"rank {rank}: {type(e).__name__}: {e}")
        os._exit(4)
    parts = shards.lpt_shards(shards.shot_costs(cfg, shots), world)
    assert red["shots_of_rank"] == [shots[i] for i in parts[rank]]
    if rank == 0:
        np.savez(out, image1=red["image1"], image2s=red["image2s"], illum=red["illum"],
                 parts=np.array([len(p) for p in parts]))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
