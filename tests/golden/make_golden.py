"""Convert the raw output of the reference's own CUDA code into the committed golden fixtures.

The raw output comes from ``oracle/_ref/ref_harness`` (built by ``make -C oracle/ref gpu``
from the reference sources and run once on a B200):

    oracle/_ref/ref_harness units <raw>     # unit kernels, 300 forward + 20 backward steps
    oracle/_ref/ref_harness rtm <raw>       # rtm_model() cases B, C, D

    python tests/golden/make_golden.py <raw-units-dir> [<raw-rtm-dir>]

Writes tests/golden/ref_units.npz and tests/golden/ref_case{B,C,D}.npz.  Every array is the
reference's own output, stored verbatim (float32 / int32), plus the SU/SEG-Y trace-header
bytes the reference wrote, for byte-exact comparison of our file writers.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Parameters of the harness cases (oracle/ref/ref_harness.cu, run_rtm()).
CASES = {
    "caseB": dict(layout=2, mode=0, medium_flag=0, ismth=0, nshot=2, nx=96, nz=64, nt=600, npml=32,
                  smooth_model=0, dx=10.0, dt=1e-3, fdom=25.0, spx0=300.0, spz0=20.0, dspx=360.0,
                  offset=0.0, offsetmax=0.0, amp=1.0, alp=0.1, direct=1.5, direct0=0.05),
    "caseC": dict(layout=2, mode=1, medium_flag=0, ismth=0, nshot=2, nx=96, nz=64, nt=600, npml=32,
                  smooth_model=4, dx=10.0, dt=1e-3, fdom=25.0, spx0=300.0, spz0=20.0, dspx=360.0,
                  offset=0.0, offsetmax=0.0, amp=1.0, alp=0.1, direct=1.5, direct0=0.05,
                  data_from="caseB"),
    "caseD": dict(layout=1, mode=0, medium_flag=1, ismth=2, nshot=2, nx=96, nz=64, nt=500, npml=32,
                  smooth_model=0, dx=10.0, dt=1e-3, fdom=25.0, spx0=200.0, spz0=20.0, dspx=550.0,
                  offset=0.0, offsetmax=860.0, amp=1.0, alp=0.07, direct=1.5, direct0=0.0),
}


def read_su(path, nt):
    raw = np.fromfile(path, dtype=np.uint8)
    tb = 240 + 4 * nt
    ntr = raw.size // tb
    tr = raw.reshape(ntr, tb)
    headers = tr[:, :240].copy()
    data = tr[:, 240:].copy().view(np.float32).reshape(ntr, nt).T.copy()   # [nt][ntr]
    return headers, data


def units(raw):
    out = {}
    for f in sorted(os.listdir(raw)):
        p = os.path.join(raw, f)
        if os.path.isdir(p):
            continue
        name, ext = os.path.splitext(f)
        out[name] = np.fromfile(p, dtype=np.int32 if ext == ".i32" else np.float32)
    np.savez_compressed(os.path.join(HERE, "ref_units.npz"), **out)
    print("ref_units.npz:", len(out), "arrays")


def case(raw, name):
    d = os.path.join(raw, name)
    prm = CASES[name]
    nx, nz, nt = prm["nx"], prm["nz"], prm["nt"]
    out = {"params": np.frombuffer(json.dumps(prm).encode(), dtype=np.uint8)}
    for img in ("vp0", "rho0", "image1", "image2s", "image3s", "image4s", "image5s", "image2m",
                "image3m", "image4m", "image5m", "illum"):
        out[img] = np.fromfile(os.path.join(d, img + ".f32"), dtype=np.float32).reshape(nz, nx)
    if prm["mode"] == 0:
        for s in range(1, prm["nshot"] + 1):
            h, g = read_su(os.path.join(d, "seisReal", f"{s}seisreal.su"), nt)
            out[f"gather{s}"] = g
            out[f"gather{s}_headers"] = h
    # header bytes of the first trace of an image file written by Output1d
    t = np.fromfile(os.path.join(d, "output", "Image1temp.su"), dtype=np.uint8)
    out["image_su_header0"] = t[:240].copy()
    out["image_su_bytes"] = np.array([t.size], np.int64)
    np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **out)
    print(f"ref_{name}.npz:", len(out), "arrays")


if __name__ == "__main__":
    units(sys.argv[1])
    rtm_raw = sys.argv[2] if len(sys.argv) > 2 else sys.argv[1]
    for name in CASES:
        if os.path.isdir(os.path.join(rtm_raw, name)):
            case(rtm_raw, name)
