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
