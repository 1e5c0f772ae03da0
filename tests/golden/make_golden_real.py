"""Golden fixtures of the real-data path, made from the reference's own code.

1. End to end.  ``oracle/_ref/ref_harness real <raw>`` (built by ``make -C oracle/ref gpu``
   from the reference sources and run once on a B200) writes a 3-shot SEG-Y file, runs the
   reference's scanshotgather() and rtm_real() on it and dumps what they produced; this
   script packs ``<raw>/real`` into ref_real.npz: the file's bytes, the models, the shot
   table, the ten images rtm_real() returns and the Imagetrue image it writes.
2. Units.  The reference's scanshotgather() on little- and big-endian SU and SEG-Y files, and
   its Interpseis2d / GeneralFKinterp / Sincinterp on seeded gathers, run here through
   ``oracle/_ref/libref_host.so`` (the reference host C++ built from its sources, its
   Interp_function.cpp compiled against an FFTW-interface shim over the oracle's DFT), into
   ref_real_units.npz.

    python tests/golden/make_golden_real.py <raw-dir>
"""
import ctypes as C
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gubingluo_b200.synthetic import write_shot_file  # noqa: E402

# Parameters of the harness's real-data case (oracle/ref/ref_harness.cu, run_real()).
REAL = dict(nx=192, nz=64, nt=600, dx=10.0, dz=10.0, dt=1e-3, npml=32, nx0=96, nz0=32, nt0=300, dx0=20.0,
            dz0=20.0, dt0=2e-3, lx=2, lz=2, fdom=20.0, spz0=20.0, amp=1.0, alp=0.1, direct=1.5, direct0=0.05,
            medium_flag=1, ismth=2, sgyflag=1, nshot=3, filename="real.sgy")

# Scan cases: (sx, offset, traces) per shot, nt0, sgyflag, big-endian.
SCANS = {
    "le_su": ([(100, 30, 5), (350, 30, 7), (600, 60, 4)], 40, 0, False),
    "le_segy": ([(100, 30, 5), (350, 30, 7), (600, 60, 4)], 40, 1, False),
    "be_su": ([(100, 30, 5), (350, 30, 7), (600, 60, 4)], 40, 0, True),
    "be_segy_one": ([(2500, 0, 9)], 24, 1, True),
}

# Interpolation cases: nx0, nt0, nx, nt, dt0, dt (x and t / x only / t only / neither).
INTERP = {
    "xt_lx3": (9, 64, 25, 160, 0.005, 0.002),
    "xt_lx2": (12, 80, 23, 200, 0.004, 0.0016),
    "x_only": (10, 50, 19, 50, 0.004, 0.004),
    "t_only": (11, 60, 11, 150, 0.004, 0.0016),
    "t_narrow": (11, 60, 8, 150, 0.004, 0.0016),
}


def real(raw):
    d = os.path.join(raw, "real")
    p = REAL
    nx, nz = p["nx"], p["nz"]
    out = {"params": np.frombuffer(json.dumps(p).encode(), dtype=np.uint8)}
    for k in ("vp0", "rho0", "image1", "image2s", "image3s", "image4s", "image5s", "image2m", "image3m", "image4m",
              "image5m", "illum"):
        out[k] = np.fromfile(os.path.join(d, k + ".f32"), dtype=np.float32).reshape(nz, nx)
    out["profile"] = np.fromfile(os.path.join(d, "profile.i32"), dtype=np.int32).reshape(4, -1)
    out["endianflag"] = np.fromfile(os.path.join(d, "endianflag.i32"), dtype=np.int32)
    out["sgy_bytes"] = np.fromfile(os.path.join(d, "seisReal", p["filename"]), dtype=np.uint8)
    t = np.fromfile(os.path.join(d, "output", "0Imagetrue.su"), dtype=np.uint8).reshape(nx, 240 + 4 * nz)
    out["imagetrue"] = t[:, 240:].copy().view(np.float32).reshape(nx, nz).T.copy()
    np.savez_compressed(os.path.join(HERE, "ref_real.npz"), **out)
    print("ref_real.npz:", len(out), "arrays")


def units():
    R = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_host.so"))
    vp = C.c_void_p
    R.ref_scanshotgather.argtypes = [C.c_char_p, C.c_int, vp, vp, C.c_int]
    R.ref_Interpseis2d.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float]
    R.ref_GeneralFKinterp.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int]
    out = {}
    rng = np.random.default_rng(20260900)
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "seisReal"))
        cwd = os.getcwd()
        os.chdir(tmp)
        try:
            for name, (shots, nt0, sgy, be) in SCANS.items():
                g = [(sx, off, rng.standard_normal((nt0, n)).astype(np.float32)) for sx, off, n in shots]
                path = os.path.join(tmp, "seisReal", name + ".sgy")
                write_shot_file(path, g, nt0, 0.002, 10.0, sgyflag=sgy, big_endian=be)
                cap = len(shots) + 2
                prof = np.full((4, cap), -7, np.int32)
                endian = np.array([-1], np.int32)
                R.ref_scanshotgather((name + ".sgy").encode(), sgy, endian.ctypes.data, prof.ctypes.data, cap)
                out[f"scan_{name}_bytes"] = np.fromfile(path, dtype=np.uint8)
                out[f"scan_{name}_profile"] = prof
                out[f"scan_{name}_endian"] = endian
                out[f"scan_{name}_meta"] = np.array([sgy, nt0, len(shots)], np.int32)
        finally:
            os.chdir(cwd)
    for name, (nx0, nt0, nx, nt, dt0, dt) in INTERP.items():
        obs = rng.standard_normal((nt0, nx0)).astype(np.float32)
        res = np.zeros((nt, nx), np.float32)
        R.ref_Interpseis2d(res.ctypes.data, obs.ctypes.data, nx, nx0, nt, nt0, np.float32(dt), np.float32(dt0))
        out[f"interp_{name}_in"] = obs
        out[f"interp_{name}_out"] = res
        out[f"interp_{name}_dt"] = np.array([dt0, dt], np.float32)
    obs = rng.standard_normal((64, 9)).astype(np.float32)
    res = np.zeros((64, 25), np.float32)
    R.ref_GeneralFKinterp(obs.ctypes.data, res.ctypes.data, 25, 9, 64, 3)
    out["fk_lx3_in"], out["fk_lx3_out"] = obs, res
    np.savez_compressed(os.path.join(HERE, "ref_real_units.npz"), **out)
    print("ref_real_units.npz:", len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        real(sys.argv[1])
    units()
