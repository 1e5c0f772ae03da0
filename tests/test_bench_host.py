"""bench.py's host side, without a GPU: the reference arm's JSON line (it runs the CPU
restatement on the host cores) and the per-shot work that converts a CPU sample to shots/s."""
import importlib.util
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("config", [2, 4])
def test_reference_arm_prints_one_contract_line(config):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", str(config),
           "--steps", "1", "--warmup", "1", "--cpu-sample-steps", "8"]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True, cwd=ROOT, timeout=600).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "shots/s" and d["unit"] == "shots/s"
    assert d["higher_is_better"] is True and d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith(f"config {config}:")


def test_survey_shot_work_follows_each_shots_window():
    b = _bench()
    from gubingluo_b200 import synthetic
    s, shots, _, _, _, meta = synthetic.config(2)
    work = b.survey_shot_work(s, shots, meta)
    X, Z = s.nx + 2 * s.npml, s.nz + 2 * s.npml
    assert {w for _, _, w in work} == {s.nt * (2.0 * X * Z + s.nx * s.nz)}   # full spread: one window
    s4, shots4, _, _, _, meta4 = synthetic.config(4)
    work4 = b.survey_shot_work(s4, shots4, meta4)
    assert len({w for _, _, w in work4}) > 100                  # drawn apertures: windows differ
    for ish, om, w in work4:
        assert om == (meta4["apertures"][ish] - 1) * s4.dx
        assert w <= s4.nt * (2.0 * (801 + 2 * s4.npml) * (s4.nz + 2 * s4.npml) + 801 * s4.nz)


def test_default_workload_label_is_the_configuration_2_text():
    b = _bench()
    from gubingluo_b200 import synthetic
    saved = sys.argv
    sys.argv = ["bench.py"]
    try:
        args = b.parse()          # the defaults
    finally:
        sys.argv = saved
    s, shots, _, _, _, meta = synthetic.config(2)
    assert b.workload_text(args, s, shots, meta) == b.WORKLOAD
    args.strips = "fp16"
    assert "fp16 strips" in b.workload_text(args, s, shots, meta)
