"""Shot sharding for several GPUs: the longest-processing-time partition, and a two-rank
gloo run on the CPU whose summed images must equal the single-process images."""
import os
import socket
import subprocess
import sys

import numpy as np

from conftest import ROOT, rel_l2


def test_lpt_partition_is_complete_balanced_and_deterministic(rtmlib):
    from gubingluo_b200.shards import lpt_shards
    rng = np.random.default_rng(5)
    costs = list(rng.uniform(1.0, 10.0, 37))
    for world in (1, 2, 3, 8):
        parts = lpt_shards(costs, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert parts == lpt_shards(costs, world)
    # equal costs: round robin
    assert lpt_shards([1.0] * 7, 3) == [[0, 3, 6], [1, 4], [2, 5]]
    # more ranks than shots: the extra ranks get nothing
    assert lpt_shards([3.0, 2.0], 4) == [[0], [1], [], []]


def test_lpt_uses_each_shots_padded_grid(rtmlib):
    from gubingluo_b200 import SurveyConfig
    from gubingluo_b200.shards import lpt_shards, shot_costs
    # layout 1 with a bounded aperture: shots near the left edge have narrower grids
    s = SurveyConfig(nx=401, nz=101, nt=1000, dx=10.0, dz=10.0, dt=1e-3, npml=20, layout=1, spx0=20.0,
                     spz0=10.0, dspx=180.0, offsetmax=900.0)
    costs = shot_costs(s, [1, 2, 3, 12, 13])
    assert costs[0] < costs[1] < costs[2] < costs[3] == costs[4]
    parts = lpt_shards(costs, 2)
    loads = [sum(costs[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= max(costs)


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_two_gloo_ranks_sum_to_the_single_process_images(tmp_path, oracle):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _gloo_rank as W
    out = str(tmp_path / "reduced.npz")
    port = str(_free_port())
    env = dict(os.environ, PYTHONPATH=ROOT)
    procs = [subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "_gloo_rank.py"), str(r), "2", port, out],
                              env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT) for r in range(2)]
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=300)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
    assert all(p.returncode == 0 for p in procs), "\n".join(logs)
    red = np.load(out)
    assert list(red["parts"]) in ([3, 2], [2, 3])
    s, shots, vp, rho = W.survey()
    ref = oracle.rtm_model(s, shots, vp, rho, precision="f64")
    for k in ("image1", "image2s", "illum"):
        assert np.abs(ref[k]).max() > 0
        assert rel_l2(red[k], ref[k]) < 1e-12, k


def test_a_rank_that_dies_before_the_reduction_ends_the_others(tmp_path):
    """Failure detection on the host: the second of two gloo ranks exits after its shots and
    before the image reduction.  The first rank's reduction fails with an error instead of
    waiting, and it exits with its own status; both end well inside the test's time limit."""
    import time
    out = str(tmp_path / "reduced.npz")
    port = str(_free_port())
    env = dict(os.environ, PYTHONPATH=ROOT)
    t0 = time.time()
    procs = [subprocess.Popen([sys.executable, os.path.join(ROOT, "tests", "_gloo_rank.py"), str(r), "2", port, out,
                               "fail"], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT) for r in range(2)]
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=240)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
    assert [p.returncode for p in procs] == [4, 3], "\n".join(logs)
    assert os.path.exists(out + ".failed") and not os.path.exists(out)
    assert "rank 0" in open(out + ".failed").read()
    assert time.time() - t0 < 200


class _RecordingDist:
    """Stands in for torch.distributed in one process: records the all-reduce calls (shape,
    dtype) without reducing, so that ranks with and without shots can be compared."""

    def __init__(self, world, rank):
        self.world, self.rank, self.calls = world, rank, []

    def get_world_size(self):
        return self.world

    def get_rank(self):
        return self.rank

    def get_backend(self):
        return "gloo"

    def all_reduce(self, t):
        self.calls.append((tuple(t.shape), str(t.dtype)))


def test_sharded_migration_ranks_take_the_same_collective_steps(rtmlib):
    """Every rank of migrate_sharded makes the same all-reduce calls in the same order, also a
    rank left without shots (more ranks than shots, which adds zeros), with fp64 and the other
    imaging conditions on; world 1 runs the migration on all the shots."""
    from gubingluo_b200 import RunOptions, SurveyConfig
    from gubingluo_b200.shards import migrate_sharded
    s = SurveyConfig(nx=40, nz=20, nt=50, dx=10.0, dz=10.0, dt=1e-3, npml=10, layout=2, spx0=100.0, spz0=10.0,
                     dspx=100.0, mode=1)
    opts = RunOptions(accum_fp64=3, extra_images=1)
    seen = []

    def fake(survey, options, shots, vp, rho, gathers, vp_mig, rho_mig):
        seen.append((list(shots), None if gathers is None else len(gathers)))
        one = np.ones((survey.nz, survey.nx), np.float32)
        out = {k: one * len(shots) for k in ("image1", "image2s", "image2m", "illum")}
        out["f64"] = {k: np.ones((survey.nz, survey.nx)) for k in ("image1", "image2s", "illum")}
        for k in ("image3s", "image4s", "image5s", "image3m", "image4m", "image5m", "imagetrue"):
            out[k] = one.copy()
        out["stats"] = object()
        return out

    shots = [1, 2]
    gathers = [np.zeros((50, 40), np.float32) for _ in shots]
    calls = []
    for rank in range(3):
        d = _RecordingDist(3, rank)
        out = migrate_sharded(s, opts, shots, None, None, gathers=gathers, dist=d, migrate_fn=fake)
        calls.append(d.calls)
        assert out["shots_of_rank"] == ([1], [2], [])[rank]
        assert out["image1"].shape == (20, 40)
    assert calls[0] == calls[1] == calls[2] and len(calls[0]) == 11 + 3
    assert seen == [([1], 1), ([2], 1)]   # rank 2 migrated nothing
    out = migrate_sharded(s, opts, shots, None, None, gathers=gathers, migrate_fn=fake)
    assert out["shots_of_rank"] == shots and float(out["image1"][0, 0]) == 2.0
