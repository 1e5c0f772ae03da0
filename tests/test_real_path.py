"""The real-data path (reference rtm_real.cu, scanshotgather RTM_GPU_velstr.cpp:363-454,
Interp_function.cpp): shot-table scan, per-shot geometry, trace reading, F-K / sinc
resampling, the mute in the migration model and the migration.

Fixtures (tests/golden/make_golden_real.py): ref_real_units.npz holds the reference's own
scanshotgather() tables and Interpseis2d / GeneralFKinterp outputs (its host C++ built from
its sources, FFTW's DFT restated); ref_real.npz holds a 3-shot SEG-Y file and the images the
reference's rtm_real() produced from it on a B200.

Tolerances: FP32 results within 1e-4 relative L2 (the path's stated bound) unless a test says
why not; integer tables and geometry exact."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

TOL_FP32 = 1e-4
# image3 (wavefield decomposition) switches on the signs of products near zero; image4 bins
# Poynting angles, and at these data amplitudes the float Poynting products underflow only in
# part, so rounding moves contributions between angle bins in many cells (the oracle's f32
# and f64 forms differ by 0.2 there; the f32 oracle and the reference by 0.03); Imagetrue
# divides by the sine of that angle and is the least stable of all.
TOL_DECOMP = 3e-3
TOL_ANGLE = 5e-2
TOL_TRUE = 0.5


def _units():
    path = os.path.join(GOLDEN, "ref_real_units.npz")
    if not os.path.exists(path):
        pytest.skip("ref_real_units.npz not present")
    return np.load(path)


def _real_case():
    path = os.path.join(GOLDEN, "ref_real.npz")
    if not os.path.exists(path):
        pytest.skip("ref_real.npz not present")
    z = np.load(path)
    p = json.loads(bytes(z["params"]).decode())
    f = lambda v: float(np.float32(v))
    s = dict(nx=p["nx"], nz=p["nz"], nt=p["nt"], dx=f(p["dx"]), dz=f(p["dz"]), dt=f(p["dt"]), npml=p["npml"],
             fdom=f(p["fdom"]), amp=f(p["amp"]), alp=f(p["alp"]), spz0=f(p["spz0"]), medium_flag=p["medium_flag"],
             ismth=p["ismth"], direct=f(p["direct"]), direct0=f(p["direct0"]), mute=1, receiver_depth=0)
    return z, p, s


def _survey_cfg(G, s, mode=1, mute=2):
    keys = ("nx", "nz", "nt", "dx", "dz", "dt", "npml", "fdom", "amp", "alp", "spz0", "medium_flag", "ismth",
            "direct", "direct0", "receiver_depth")
    return G.SurveyConfig(**{k: s[k] for k in keys}, layout=3, mode=mode, mute=mute)


INTERP = ("xt_lx3", "xt_lx2", "x_only", "t_only", "t_narrow")
SCANS = ("le_su", "le_segy", "be_su", "be_segy_one")


# ---- oracle against the reference ---------------------------------------------------------
@pytest.mark.parametrize("name", INTERP)
def test_oracle_interp_matches_reference(oracle, name):
    """Interpseis2d restated (orc_interp.c) against the reference's, branch by branch; with the
    same DFT underneath the two agree to the bit, the bound allows for compilers."""
    z = _units()
    obs, ref = z[f"interp_{name}_in"], z[f"interp_{name}_out"]
    dt0, dt = (float(v) for v in z[f"interp_{name}_dt"])
    got = oracle.interp_gather(obs, ref.shape[1], ref.shape[0], dt, dt0)
    assert np.abs(ref).max() > 0
    assert rel_l2(got, ref) < 1e-6


def test_oracle_fk_matches_reference(oracle):
    z = _units()
    got = oracle.fk_interp(z["fk_lx3_in"], z["fk_lx3_out"].shape[1], 3)
    assert rel_l2(got, z["fk_lx3_out"]) < 1e-6


def test_fk_negative_frequency_indexing(oracle):
    """The reference builds the negative frequencies one row off the Hermitian partner: its F-K
    output of a dipping band-limited event is far from the event.  The Hermitian form (mirror
    1) interpolates it.  Odd nt0 (where the reference reads one row past its array) is
    defined: that row is zero."""
    nt0, nx0, dt0 = 120, 16, 0.004
    t = np.arange(nt0) * dt0

    def ricker(tt):
        a = (np.pi * 20.0 * tt) ** 2
        return (1 - 2 * a) * np.exp(-a)

    obs = np.stack([ricker(t - 0.15 - 0.01 * ix) for ix in range(nx0)], axis=1).astype(np.float32)
    nx = 2 * (nx0 - 1) + 1
    mid = ricker(t - 0.155)
    good = oracle.fk_interp(obs, nx, 2, mirror=1)
    bad = oracle.fk_interp(obs, nx, 2, mirror=0)
    assert np.corrcoef(good[:, 1], mid)[0, 1] > 0.9999
    assert np.corrcoef(bad[:, 1], mid)[0, 1] < 0.9
    odd = oracle.fk_interp(obs[:119], nx, 2, mirror=0)
    assert np.isfinite(odd).all() and np.abs(odd).max() > 0


def test_oracle_rtm_real_matches_reference(oracle, tmp_path):
    """The whole real-data shot loop restated (oracle.rtm_real) against the reference's
    rtm_real() images."""
    z, p, s = _real_case()
    path = tmp_path / "real.sgy"
    path.write_bytes(z["sgy_bytes"].tobytes())
    out = oracle.rtm_real(s, str(path), z["profile"], [1, 2, 3], z["vp0"], z["rho0"], p["nt0"],
                          float(np.float32(p["dt0"])), p["dx0"], sgyflag=1, endianflag=0, extra=2)
    for k in ("image1", "image2s", "image2m", "illum", "image5s", "image5m"):
        assert rel_l2(out[k], z[k]) < 1e-5, k
    for k in ("image3s", "image3m"):
        assert rel_l2(out[k], z[k]) < TOL_DECOMP, k
    for k in ("image4s", "image4m"):
        assert rel_l2(out[k], z[k]) < TOL_ANGLE, k
    assert rel_l2(out["imagetrue"], z["imagetrue"]) < TOL_TRUE


# ---- host layer of the product against the reference -----------------------------------------
@pytest.mark.parametrize("name", SCANS)
def test_scan_matches_reference(rtmlib, tmp_path, name):
    """rtm_scan_shotgather against the reference's scanshotgather().  For byte-swapped files
    the reference adds a trailing shot of zero traces (its end-of-file read swaps the last
    keys back); the product does not."""
    z = _units()
    sgy, nt0, nshots = (int(v) for v in z[f"scan_{name}_meta"])
    path = tmp_path / f"{name}.sgy"
    path.write_bytes(z[f"scan_{name}_bytes"].tobytes())
    prof, endian = rtmlib.scan_shotgather(str(path), sgy, max_shots=16)
    ref = z[f"scan_{name}_profile"]
    assert endian == int(z[f"scan_{name}_endian"][0])
    assert prof.shape == (4, nshots)
    assert np.array_equal(prof, ref[:, :nshots])
    if endian:
        assert ref[1][nshots] == 0            # the reference's trailing zero-trace entry
    else:
        assert ref[2][nshots] == -7           # untouched


def test_scan_edge_cases(rtmlib, tmp_path):
    from gubingluo_b200.synthetic import write_shot_file
    rng = np.random.default_rng(4)
    path = str(tmp_path / "a.su")
    # a partial trailing trace is not counted; a shot returning to an earlier sx is a new shot
    shots = [(0, 10, rng.standard_normal((16, 3))), (50, 10, rng.standard_normal((16, 2))),
             (0, 10, rng.standard_normal((16, 1)))]
    write_shot_file(path, shots, 16, 0.004, 10.0)
    with open(path, "ab") as f:
        f.write(b"\0" * 100)
    prof, e = rtmlib.scan_shotgather(path, 0)
    assert prof.tolist() == [[0, 50, 0], [3, 2, 1], [1, 4, 6], [10, 10, 10]] and e == 0
    with pytest.raises(rtmlib.RtmError):
        rtmlib.scan_shotgather(path, 0, max_shots=2)
    with open(path, "wb") as f:
        f.write(b"\0" * 200)
    with pytest.raises(rtmlib.RtmError):
        rtmlib.scan_shotgather(path, 0)


def test_real_geometry_matches_restatement(rtmlib, oracle):
    s = dict(nx=400, nz=80, nt=500, dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=24, spz0=15.0,
             receiver_depth=0, fdom=20.0, amp=1.0, alp=0.1, medium_flag=0, ismth=0, direct=1.5, direct0=0.0)
    cfg = _survey_cfg(rtmlib, s)
    n = 0
    for sx in (0, 7, 250, 1234):
        for off in (0, 5, 50, 133):
            for ntr in (1, 2, 17, 46):
                for dx0 in (10.0, 20.0, 12.5, 25.0):
                    want, nc_w = oracle.real_geometry(s, sx, off, ntr, dx0)
                    if want.nx2 > s["nx"] - 1 or want.nrec < 1 or want.nxlength < 2:
                        with pytest.raises(rtmlib.RtmError):
                            rtmlib.real_geometry(cfg, sx, off, ntr, dx0)
                        continue
                    g, nc = rtmlib.real_geometry(cfg, sx, off, ntr, dx0)
                    for k in ("nx1", "nx2", "nxlength", "noffset", "nsx", "nsz", "nxpad", "nzpad", "rx0", "nrec"):
                        assert getattr(g, k) == getattr(want, k), (sx, off, ntr, dx0, k)
                    assert nc == nc_w and g.rz == s["npml"]
                    n += 1
    assert n > 100


@pytest.mark.parametrize("name", SCANS)
def test_read_shot_traces(rtmlib, oracle, tmp_path, name):
    z = _units()
    sgy, nt0, nshots = (int(v) for v in z[f"scan_{name}_meta"])
    path = str(tmp_path / f"{name}.sgy")
    with open(path, "wb") as f:
        f.write(z[f"scan_{name}_bytes"].tobytes())
    prof = z[f"scan_{name}_profile"]
    endian = int(z[f"scan_{name}_endian"][0])
    for k in range(nshots):
        ntr, itr = int(prof[1][k]), int(prof[2][k])
        for ncols in (ntr, ntr + 1):
            got = rtmlib.read_shot_traces(path, sgy, endian, nt0, itr, ntr, ncols)
            want = oracle.read_traces(path, sgy, endian, nt0, itr, ntr, ncols)
            assert np.array_equal(got, want)
            assert not got[:, ntr:].any()
    with pytest.raises(rtmlib.RtmError):   # past the end of the file
        rtmlib.read_shot_traces(path, sgy, endian, nt0, int(prof[2][nshots - 1]), 50, 50)
    with pytest.raises(rtmlib.RtmError):   # trace length that is not the file's
        rtmlib.read_shot_traces(path, sgy, endian, nt0 - 1, 1, 1, 1)


def test_interp_refuses_bad_shapes_before_the_device(rtmlib):
    obs = np.zeros((20, 5), np.float32)
    with pytest.raises(rtmlib.RtmError, match="exceed"):
        rtmlib.interp_gather(obs, 11, 40, 0.001, 0.002)   # lx = 2, lx*nx0 = 10 < 11
    with pytest.raises(rtmlib.RtmError, match="two recorded traces"):
        rtmlib.interp_gather(np.zeros((20, 1), np.float32), 3, 40, 0.001, 0.002)


# ---- GPU ---------------------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", INTERP)
def test_gpu_interp_matches_reference(rtmlib, oracle, name):
    z = _units()
    obs, ref = z[f"interp_{name}_in"], z[f"interp_{name}_out"]
    dt0, dt = (float(v) for v in z[f"interp_{name}_dt"])
    got = rtmlib.interp_gather(obs, ref.shape[1], ref.shape[0], dt, dt0)
    assert rel_l2(got, ref) < TOL_FP32


@pytest.mark.gpu
@pytest.mark.parametrize("nx0,nt0,nx,nt,mirror", [(120, 1000, 239, 2000, 0), (120, 1000, 239, 2000, 1),
                                                  (61, 751, 181, 1502, 0), (61, 751, 181, 1502, 1),
                                                  (33, 400, 33, 999, 0), (40, 500, 79, 500, 1)])
def test_gpu_interp_matches_oracle(rtmlib, oracle, nx0, nt0, nx, nt, mirror):
    """Larger seeded gathers, odd nt0, both negative-frequency forms; cuFFT against the
    oracle's DFT."""
    rng = np.random.default_rng(nx0 * 1000 + nt0)
    obs = rng.standard_normal((nt0, nx0)).astype(np.float32)
    dt0 = float(np.float32(0.004))
    dt = float(np.float32(dt0 * nt0 / nt))
    want = oracle.interp_gather(obs, nx, nt, dt, dt0, mirror)
    got = rtmlib.interp_gather(obs, nx, nt, dt, dt0, mirror)
    assert rel_l2(got, want) < TOL_FP32


def _profile_rows(prof):
    rows = [np.ascontiguousarray(prof[r], dtype=np.int32) for r in range(4)]
    arr = (C.POINTER(C.c_int) * 4)(*[r.ctypes.data_as(C.POINTER(C.c_int)) for r in rows])
    return arr, rows


@pytest.mark.gpu
def test_gpu_rtm_real_dropin_matches_reference(rtmlib, tmp_path, monkeypatch):
    """rtm_real() with the argument list of its definition (rtm_real.cu:17-22) on the file the
    reference migrated: images against the reference's, Imagetrue and temp files written."""
    monkeypatch.setenv("RTM_B200_EXTRA_IMAGES", "2")
    z, p, s = _real_case()
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        os.makedirs("seisReal")
        os.makedirs("output")
        with open("seisReal/real.sgy", "wb") as f:
            f.write(z["sgy_bytes"].tobytes())
        nx, nz = p["nx"], p["nz"]
        imgs = [np.zeros((nz, nx), np.float32) for _ in range(10)]
        coef = rtmlib.coef_table()
        wl = np.zeros(p["nt"], np.float32)
        rows, keep = _profile_rows(z["profile"])
        vp, rho = np.ascontiguousarray(z["vp0"]), np.ascontiguousarray(z["rho0"])
        L = rtmlib.lib()
        f = lambda x: C.c_float(float(x))
        name = C.create_string_buffer(b"real.sgy", 40)
        L.rtm_real(0, p["nshot"], 1, 1, p["medium_flag"], 3, p["sgyflag"], int(z["endianflag"][0]), p["ismth"], nx,
                   nz, p["nt"], f(p["dx"]), f(p["dz"]), f(p["dt"]), p["nx0"], p["nz0"], p["nt0"], f(p["dx0"]),
                   f(p["dz0"]), f(p["dt0"]), p["npml"], p["lx"], p["lz"], f(1.0), f(p["fdom"]), f(p["spz0"]),
                   f(p["amp"]), f(p["alp"]), f(p["direct"]), f(p["direct0"]), vp.ctypes.data_as(C.c_void_p),
                   rho.ctypes.data_as(C.c_void_p), coef.ctypes.data_as(C.c_void_p), wl.ctypes.data_as(C.c_void_p),
                   name, rows, *[a.ctypes.data_as(C.c_void_p) for a in imgs])
        assert L.rtm_last_error() == b""
        names = ("image1", "image2s", "image3s", "image4s", "image5s", "image2m", "image3m", "image4m", "image5m",
                 "illum")
        got = dict(zip(names, imgs))
        for k in ("image1", "image2s", "image2m", "illum", "image5s", "image5m"):
            assert rel_l2(got[k], z[k]) < TOL_FP32, k
        for k in ("image3s", "image3m"):
            assert rel_l2(got[k], z[k]) < TOL_DECOMP, k
        for k in ("image4s", "image4m"):
            assert rel_l2(got[k], z[k]) < TOL_ANGLE, k
        t = np.fromfile("output/0Imagetrue.su", np.uint8).reshape(nx, 240 + 4 * nz)
        true = t[:, 240:].copy().view(np.float32).reshape(nx, nz).T
        assert rel_l2(true, z["imagetrue"]) < TOL_TRUE
        for n in ("Image1temp", "Image2stemp", "Illumtemp", "Imagetruetemp"):
            assert os.path.getsize(f"output/{n}.su") == nx * (240 + 4 * nz)
    finally:
        os.chdir(cwd)


@pytest.mark.gpu
@pytest.mark.parametrize("mirror,extra,big_endian", [(0, 0, True), (1, 1, False)])
def test_gpu_migrate_real_matches_oracle(rtmlib, oracle, tmp_path, mirror, extra, big_endian):
    """The session API on recorded data at sizes that are no multiple of anything (odd
    windows, 5 shots in batches of 2, a byte-swapped SU file), against the oracle."""
    from gubingluo_b200.synthetic import write_shot_file
    rng = np.random.default_rng(77 + mirror)
    nz, nx = 45, 173
    v = (1800 + 15 * np.arange(nz)[:, None] + 150 * rng.random((nz, nx))).astype(np.float32)
    rho = (1900 + 200 * rng.random((nz, nx))).astype(np.float32)
    s = dict(nx=nx, nz=nz, nt=500, dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=20, fdom=22.0, amp=1.0,
             alp=0.1, spz0=12.0, medium_flag=1, ismth=1, direct=1.2, direct0=0.02, mute=1, receiver_depth=0)
    nt0, dt0, dx0 = 250, float(np.float32(2e-3)), 20.0
    shots = []
    for i, (sx, off, ntr) in enumerate([(0, 30, 31), (160, 30, 29), (300, 50, 40), (660, 10, 22), (900, 30, 28)]):
        t = np.arange(nt0) * dt0
        h = off + dx0 * np.arange(ntr)
        tt = np.sqrt(0.2 ** 2 + (h / 2000.0) ** 2)
        a = (np.pi * 20.0 * (t[:, None] - tt[None, :])) ** 2
        shots.append((sx, off, ((1 - 2 * a) * np.exp(-a) + 0.05 * rng.standard_normal((nt0, ntr))).astype(np.float32)))
    path = str(tmp_path / "shots.su")
    write_shot_file(path, shots, nt0, dt0, dx0, sgyflag=0, big_endian=big_endian)
    prof, endian = rtmlib.scan_shotgather(path, 0)
    assert prof.shape[1] == 5 and endian == int(big_endian)
    ids = [1, 2, 3, 4, 5]
    want = oracle.rtm_real(s, path, prof, ids, v, rho, nt0, dt0, dx0, sgyflag=0, endianflag=endian, extra=extra,
                           mirror=mirror)
    cfg = _survey_cfg(rtmlib, s)
    got = rtmlib.migrate_real(cfg, rtmlib.RunOptions(device=0, batch=2, extra_images=extra), path, prof, ids, v, rho,
                              nt0, dt0, dx0, sgyflag=0, endianflag=endian, mirror=mirror)
    for k in ("image1", "image2s", "illum"):
        assert np.abs(want[k]).max() > 0
        assert rel_l2(got[k], want[k]) < TOL_FP32, k
    if extra:
        assert rel_l2(got["image5s"], want["image5s"]) < TOL_FP32
        assert rel_l2(got["image3s"], want["image3s"]) < TOL_DECOMP


@pytest.mark.gpu
def test_gpu_rtm_gpu_program_real_data(rtmlib, oracle, tmp_path):
    """The drop-in program with dataflag 1: parameter file, coarse velocity file, a recorded
    SU file; it regrids the model (dx0 20 m -> 10 m, dt0 2 ms -> 1.9 ms), scans the shots into
    shotprofileId.dat and migrates through rtm_real.  Against the oracle on the regridded
    model; a second run reuses the cached table."""
    import subprocess
    from conftest import ROOT
    from gubingluo_b200.synthetic import write_shot_file
    exe = os.path.join(ROOT, "gubingluo_b200", "rtm_gpu")
    if not os.path.exists(exe):
        pytest.skip("rtm_gpu not built")
    nx0, nz0, nt0, dx0, dt0 = 61, 21, 250, 20.0, float(np.float32(0.002))
    rng = np.random.default_rng(9)
    vp0 = np.full((nz0, nx0), 1800, np.float32)
    vp0[10:] = 2500
    vp0 += (100 * rng.random((nz0, nx0))).astype(np.float32)
    inp, sre, outd = tmp_path / "input", tmp_path / "seisReal", tmp_path / "output"
    for d in (inp, sre, outd):
        d.mkdir()
    with open(inp / "vel.su", "wb") as f:
        for ix in range(nx0):
            f.write(b"\0" * 240)
            f.write(np.ascontiguousarray(vp0[:, ix]).tobytes())
    t = np.arange(nt0) * dt0
    shots = []
    for sx, off, ntr in ((0, 40, 20), (200, 40, 25), (500, 20, 30)):
        h = off + dx0 * np.arange(ntr)
        a = (np.pi * 15.0 * (t[:, None] - np.sqrt(0.15 ** 2 + (h / 1800.0) ** 2)[None, :])) ** 2
        shots.append((sx, off, ((1 - 2 * a) * np.exp(-a)).astype(np.float32)))
    write_shot_file(str(sre / "shots.su"), shots, nt0, dt0, dx0)
    (inp / "cmd.in").write_text("parameter file name\nparam.txt\n")
    vals = [f"{dt0} {nt0} 1.0", f"{(nx0 - 1) * dx0} {(nz0 - 1) * dx0} {dx0} {dx0}", "15 1 0.1", "0 20 0", "0 0",
            "1 3 1 3", "20", "1 1", "1.2 0.02", "0", "3", "1", "1", "0", "0", "0", "vel.su", "shots.su"]
    (inp / "param.txt").write_text("".join(f"# comment {i}\n{v}\n" for i, v in enumerate(vals)))
    env = dict(os.environ, RTM_B200_EXTRA_IMAGES="0")
    for run in range(2):
        r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=300, env=env)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "The program calculate over" in r.stdout
    table = np.loadtxt(tmp_path / "shotprofileId.dat", dtype=np.int64).T
    assert table.tolist() == [[0, 200, 500], [20, 25, 30], [1, 21, 46], [40, 40, 20]]
    # the same regridding through the library, then the oracle
    L = rtmlib.lib()
    dx, dz, dt, vmin, vmax = (C.c_float() for _ in range(5))
    nx, nz, nt, lx, lz = (C.c_int() for _ in range(5))
    L.rtm_get_constant(np.ascontiguousarray(vp0).ctypes.data, C.c_float(15), C.c_float(dx0), C.c_float(dx0), nx0,
                       nz0, nt0, C.c_float(dt0), C.byref(dx), C.byref(dz), C.byref(nx), C.byref(nz), C.byref(nt),
                       C.byref(dt), C.byref(lx), C.byref(lz), C.byref(vmin), C.byref(vmax))
    assert (lx.value, nx.value) == (2, 121) and nt.value > nt0
    vp = np.zeros((nz.value, nx.value), np.float32)
    L.rtm_interp_model(np.ascontiguousarray(vp0).ctypes.data, vp.ctypes.data, nx0, nz0, nx.value, nz.value, lx.value,
                       lz.value)
    s = dict(nx=nx.value, nz=nz.value, nt=nt.value, dx=dx.value, dz=dz.value, dt=dt.value, npml=20, fdom=15.0, amp=1.0,
             alp=0.1, spz0=20.0, medium_flag=1, ismth=1, direct=1.2, direct0=0.02, mute=1, receiver_depth=0)
    want = oracle.rtm_real(s, str(sre / "shots.su"), table, [1, 2, 3], vp, np.full_like(vp, 2000.0), nt0, dt0, dx0)
    for name, k in (("Image1", "image1"), ("Image2s", "image2s"), ("Illum", "illum")):
        raw = np.fromfile(outd / f"0{name}.su", np.uint8).reshape(nx.value, 240 + 4 * nz.value)
        got = raw[:, 240:].copy().view(np.float32).reshape(nx.value, nz.value).T
        assert np.abs(want[k]).max() > 0
        assert rel_l2(got, want[k]) < TOL_FP32, name
