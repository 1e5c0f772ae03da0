"""Run control around the migration: checkpoint / resume, detection of a diverging run
(NaN or infinite images), the reference's progress snapshots and the JSON-lines log.

The reference has no checkpoint (it dumps partial images every 50 shots, rtm_model.cu:490-538,
and is resumed by hand from a new startshot without them), no numeric checks and prints
max |p| every tsnap from a full-grid copy (rtm_model.cu:271-273, 324-326, 415-417).
Failures are made on the host: an unstable time step, a NaN in the model, a foreign or
truncated checkpoint file; no GPU fault is involved."""
import ctypes as C
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_l2


def _model(nz, nx, seed):
    rng = np.random.default_rng(seed)
    v = (1800 + 12 * np.arange(nz)[:, None] + 120 * rng.random((nz, nx))).astype(np.float32)
    return v, np.full((nz, nx), 2000.0, np.float32)


def _survey(G, **kw):
    s = dict(nx=96, nz=40, nt=300, dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=16, fdom=25.0, amp=1.0,
             alp=0.1, layout=2, spx0=100.0, spz0=20.0, dspx=150.0, mode=0, direct=1.5, direct0=0.0)
    s.update(kw)
    return G.SurveyConfig(**s)


def _header(nx, nz, nshots, done, elem=4, nimages=4, h=0x1234):
    return (b"RTMB200C" + struct.pack("<IIQ", 1, elem, h) + struct.pack("<6i", nx, nz, nshots, done, nimages, 2))


def test_checkpoint_info_and_refusals(rtmlib, tmp_path):
    p = tmp_path / "c.bin"
    p.write_bytes(_header(3, 2, 5, 2) + np.arange(24, dtype=np.float32).tobytes())
    info = rtmlib.checkpoint_info(str(p))
    assert info == dict(nx=3, nz=2, nshots=5, shots_done=2, elem_bytes=4, config_hash=0x1234)
    p.write_bytes(_header(3, 2, 5, 2) + bytes(20))                       # truncated
    with pytest.raises(rtmlib.RtmError, match="truncated"):
        rtmlib.checkpoint_info(str(p))
    p.write_bytes(b"NOTACKPT" + bytes(100))
    with pytest.raises(rtmlib.RtmError, match="not a checkpoint"):
        rtmlib.checkpoint_info(str(p))
    p.write_bytes(_header(3, 2, 5, 6) + bytes(96))                       # more shots done than shots
    with pytest.raises(rtmlib.RtmError):
        rtmlib.checkpoint_info(str(p))


@pytest.mark.gpu
@pytest.mark.parametrize("fp64,extra", [(False, 0), (True, 1)])
def test_resume_from_checkpoint_is_bitwise(rtmlib, tmp_path, fp64, extra):
    """Shots 1-2 in one session, a checkpoint, then shots 3-5 in a new session resumed from
    it: the same images, bit for bit, as one uninterrupted session (batches of 2, so the
    resume point also splits the batching differently)."""
    G = rtmlib
    v, rho = _model(40, 96, 1)
    s = _survey(G)
    shots = [1, 2, 3, 4, 5]
    opts = G.RunOptions(device=0, batch=2, accum_fp64=fp64, extra_images=extra)
    path = str(tmp_path / "run.ckpt")
    with G.Session(s, opts, shots, v, rho) as a:
        a.run_range(0, 2)
        a.save_checkpoint(path, 2)
        h = a.config_hash()
    assert G.checkpoint_info(path)["shots_done"] == 2 and G.checkpoint_info(path)["config_hash"] == h
    with G.Session(s, opts, shots, v, rho) as b:
        done = b.load_checkpoint(path)
        assert done == 2
        b.run_range(2, 1)
        b.run_range(3, 2)
        got = b.images()
        got_x = b.images_extra() if extra else {}
    with G.Session(s, opts, shots, v, rho) as c:
        c.run()
        want = c.images()
        want_x = c.images_extra() if extra else {}
    for k in ("image1", "image2s", "illum"):
        assert np.abs(want[k]).max() > 0
        assert np.array_equal(got[k], want[k]), k
    for k in want_x:
        assert np.array_equal(got_x[k], want_x[k]), k


@pytest.mark.gpu
def test_checkpoint_of_another_run_is_refused(rtmlib, tmp_path):
    G = rtmlib
    v, rho = _model(40, 96, 1)
    s = _survey(G)
    path = str(tmp_path / "run.ckpt")
    with G.Session(s, G.RunOptions(device=0), [1, 2], v, rho) as a:
        a.run_range(0, 1)
        a.save_checkpoint(path, 1)
    v2 = v.copy()
    v2[10, 10] += 1.0
    for args in (([1, 2], v2, rho, s), ([1, 3], v, rho, s), ([1, 2], v, rho, _survey(G, fdom=24.0))):
        with G.Session(args[3], G.RunOptions(device=0), args[0], args[1], args[2]) as b:
            with pytest.raises(G.RtmError, match="another survey"):
                b.load_checkpoint(path)
            assert np.abs(b.images()["image1"]).max() == 0      # untouched


@pytest.mark.gpu
def test_dropin_rtm_model_resumes(rtmlib, tmp_path, monkeypatch):
    """rtm_model() with RTM_B200_CHECKPOINT / RTM_B200_RESUME: a checkpoint after shot 1 (made
    by a session of the same configuration) is picked up and the remaining shots are added;
    the images equal those of a run from scratch."""
    G = rtmlib
    nx, nz, nt = 96, 40, 300
    v, rho = _model(nz, nx, 2)
    prm = dict(nshot=3, mode=0, medium_flag=0, layout=2, ismth=0, dt=float(np.float32(1e-3)), npml=16, direct=1.5,
               direct0=0.0, fdom=25.0, spx0=100.0, spz0=20.0, dspx=150.0, amp=1.0, alp=0.1)
    L = G.lib()
    f = lambda x: C.c_float(float(x))
    coef = G.coef_table()
    wl = np.zeros(nt, np.float32)

    def call():
        imgs = [np.zeros((nz, nx), np.float32) for _ in range(10)]
        L.rtm_model(0, prm["nshot"], 1, 1, prm["mode"], prm["medium_flag"], prm["layout"], 0, 0, prm["ismth"], nx, nz,
                    nt, f(10.0), f(10.0), f(prm["dt"]), prm["npml"], f(prm["direct"]), f(prm["direct0"]), f(0.0),
                    f(prm["fdom"]), f(prm["spx0"]), f(prm["spz0"]), f(prm["dspx"]), f(0.0), f(0.0), f(prm["amp"]),
                    f(prm["alp"]), v.ctypes.data_as(C.c_void_p), rho.ctypes.data_as(C.c_void_p),
                    coef.ctypes.data_as(C.c_void_p), wl.ctypes.data_as(C.c_void_p),
                    *[a.ctypes.data_as(C.c_void_p) for a in imgs])
        assert L.rtm_last_error() == b""
        return imgs

    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        os.makedirs("seisReal")
        os.makedirs("output")
        monkeypatch.setenv("RTM_B200_EXTRA_IMAGES", "0")
        monkeypatch.setenv("RTM_B200_BATCH", "1")
        clean = call()
        ck = str(tmp_path / "m.ckpt")
        s = _survey(G, nt=nt, mute=1, receiver_depth=0)
        with G.Session(s, G.RunOptions(device=0, batch=1), [1, 2, 3], v, rho) as a:
            a.run_range(0, 1)
            a.save_checkpoint(ck, 1)
        monkeypatch.setenv("RTM_B200_CHECKPOINT", ck)
        monkeypatch.setenv("RTM_B200_RESUME", "1")
        monkeypatch.setenv("RTM_B200_LOG", str(tmp_path / "run.jsonl"))
        resumed = call()
        assert rtmlib.checkpoint_info(ck)["shots_done"] == 3
        for a, b in zip(resumed, clean):
            assert np.array_equal(a, b)
        import json
        lines = [json.loads(x) for x in open(tmp_path / "run.jsonl")]
        assert [x["first_shot"] for x in lines] == [2, 3] and lines[-1]["shots_done"] == 3
    finally:
        os.chdir(cwd)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["unstable_dt", "nan_model"])
def test_diverging_run_is_reported(rtmlib, case):
    """A time step far above the stability limit, or a NaN in the velocity model, makes the
    wavefield non-finite; the run returns RTM_ERR_NUMERIC naming the shot instead of images
    full of NaN."""
    G = rtmlib
    v, rho = _model(40, 96, 3)
    kw = {}
    if case == "unstable_dt":
        kw["dt"] = float(np.float32(8e-3))
    else:
        v[20, 50] = np.nan
    s = _survey(G, **kw)
    with G.Session(s, G.RunOptions(device=0), [1, 2], v, rho) as ss:
        with pytest.raises(G.RtmError, match="NaN or infinite") as e:
            ss.run()
        assert "-5" in str(e.value) and "shot 1" in str(e.value)


@pytest.mark.gpu
def test_progress_snapshots(rtmlib, oracle, tmp_path):
    """verbose + tsnap prints the reference's progress lines, max |p| from an on-device
    reduction: the modelled (fused) source pass and the receiver pass, every tsnap; against
    the oracle's wavefield after the same number of forward steps."""
    code = f"""
import sys; sys.path.insert(0, {ROOT!r})
import numpy as np, gubingluo_b200 as G
rng = np.random.default_rng(3)
v = (1800 + 12 * np.arange(40)[:, None] + 120 * rng.random((40, 96))).astype(np.float32)
rho = np.full((40, 96), 2000.0, np.float32)
s = G.SurveyConfig(nx=96, nz=40, nt=300, dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=16, fdom=25.0,
                   amp=1.0, alp=0.1, layout=2, spx0=100.0, spz0=20.0, dspx=150.0, mode=0, direct=1.5, direct0=0.0)
with G.Session(s, G.RunOptions(device=0, verbose=True, tsnap=0.1), [1, 2], v, rho) as ss:
    ss.run()
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    src = [ln for ln in r.stdout.splitlines() if ln.startswith("source-the current shot")]
    bwd = [ln for ln in r.stdout.splitlines() if ln.startswith("backward-the current shot")]
    assert len(src) == 2 * 3 and len(bwd) == 2 * 3          # it = 0, 100, 200 (forward); 200, 100, 0 (backward)
    vals = {(int(ln.split()[3]), round(float(ln.split("time:")[1].split()[0]), 4)): float(ln.split("wavefield:")[1])
            for ln in src}
    assert vals[(1, 0.0)] == 0.0 and vals[(2, 0.0)] == 0.0
    G = rtmlib
    rng = np.random.default_rng(3)
    v = (1800 + 12 * np.arange(40)[:, None] + 120 * rng.random((40, 96))).astype(np.float32)
    rho = np.full((40, 96), 2000.0, np.float32)
    s = _survey(G)
    for ishot in (1, 2):
        for it in (100, 200):
            p, _, _, _ = G.forward(s, G.RunOptions(device=0), ishot, v, rho, it)
            want = float(np.abs(p).max())
            assert abs(vals[(ishot, round(it * 1e-3, 4))] - want) <= 1e-5 * want


@pytest.mark.gpu
@pytest.mark.parametrize("opt", ["fp32", "fp16_extra_fp64", "bz8_bz64"])
def test_guard_bands_hold(rtmlib, monkeypatch, opt):
    """Checking mode (RTM_B200_GUARDS=1): every device buffer is followed by a guard band,
    verified after setup and after every batch; the general cases (partial tiles, layouts
    1-4, receivers below z = 0, PML smoothing) in modes 0 and 1 with packed strips and
    gathers, fp64 images, the other imaging conditions and other tile heights leave every
    band intact, and give the same images as without the mode."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_gpu_parity import GENERAL, _random_model as rmodel, _survey as gsurvey, cfg_from
    G = rtmlib
    kw = dict(device=0, batch=2)
    if opt == "fp16_extra_fp64":
        kw.update(strip_precision="fp16", gather_precision="fp16", accum_fp64=True, extra_images=1)
    if opt == "bz8_bz64":
        monkeypatch.setenv("RTM_B200_BZ_VEL", "8")
        monkeypatch.setenv("RTM_B200_BZ_PRES", "64")
    for ci, c in enumerate(GENERAL):
        v, rho = rmodel(c["nz"], c["nx"], ci)
        shots = list(range(1, c["nshot"] + 1))
        monkeypatch.delenv("RTM_B200_GUARDS", raising=False)
        plain = G.migrate(cfg_from(G, gsurvey(c, 0)), G.RunOptions(**kw), shots, v, rho)
        monkeypatch.setenv("RTM_B200_GUARDS", "1")
        for mode in (0, 1):
            s = cfg_from(G, gsurvey(c, mode))
            with G.Session(s, G.RunOptions(**kw), shots, v, rho) as ss:
                assert ss.guard_count() > 20
                if mode == 1:
                    for k in range(len(shots)):
                        ss.set_gather(k, plain["gathers"][k])
                ss.run()
                got = ss.images()
            if mode == 0:
                for k in ("image1", "image2s", "illum"):
                    assert np.array_equal(got[k], plain[k]), (ci, k)


@pytest.mark.gpu
def test_guard_bands_hold_on_recorded_data(rtmlib, monkeypatch, tmp_path):
    """The same checking mode on the recorded-data path: resampling workspace (F-K and sinc)
    and the session's buffers."""
    from gubingluo_b200.synthetic import write_shot_file
    G = rtmlib
    monkeypatch.setenv("RTM_B200_GUARDS", "1")
    rng = np.random.default_rng(12)
    nz, nx = 37, 141
    v = (1800 + 200 * rng.random((nz, nx))).astype(np.float32)
    rho = np.full((nz, nx), 2000.0, np.float32)
    nt0, dt0, dx0 = 151, float(np.float32(2e-3)), 20.0
    shots = [(0, 20, 25), (240, 40, 30), (600, 0, 19)]
    write_shot_file(str(tmp_path / "d.su"), [(sx, off, rng.standard_normal((nt0, n)).astype(np.float32))
                                             for sx, off, n in shots], nt0, dt0, dx0, big_endian=True)
    prof, endian = G.scan_shotgather(str(tmp_path / "d.su"))
    s = G.SurveyConfig(nx=nx, nz=nz, nt=301, dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=17, fdom=20.0,
                       amp=1.0, alp=0.1, spz0=10.0, layout=3, mode=1, mute=2, ismth=1, direct=1.2)
    for mirror in (0, 1):
        out = G.migrate_real(s, G.RunOptions(device=0, batch=2), str(tmp_path / "d.su"), prof, [1, 2, 3], v, rho,
                             nt0, dt0, dx0, endianflag=endian, mirror=mirror)
        assert np.isfinite(out["image1"]).all() and np.abs(out["image1"]).max() > 0
    obs = rng.standard_normal((nt0, 24)).astype(np.float32)
    G.interp_gather(obs, 47, 301, float(np.float32(1e-3)), dt0)   # standalone entry, odd nt0
