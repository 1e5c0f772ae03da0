"""CUDA path (librtm_b200.so, through its C-ABI) against the reference's own output (golden
fixtures) and against the CPU oracle.

Tolerances (FP32 stencil): gathers and images within 1e-4 rel-L2 of the
reference / oracle; the reduced-precision forms (fp16/bf16 strips and gathers, fp64
accumulation) within 1e-3 rel-L2 of the FP64 oracle (bf16 strips and gathers: 2e-2, below
the bar; their 8-bit mantissa alone rounds each stored value by up to 2^-9).  Checked bit for
bit against the reference's own output: the device PML profiles and the device mute mask of
the reference's unit run; the shot geometry (source cell) through rtm_shot_geometry.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_case, rel_l2, survey_from_case

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-4
TOL_MIXED = 1e-3
# The wavefield-decomposition image switches on the signs of products that are close to zero
# in many cells; rounding differences of order 1e-7 flip some of those decisions.
TOL_DECOMP = 3e-3
# The Poynting-angle images keep, step by step, the cells whose angle lies in (0, 60] degrees;
# a cell on either edge of that window moves in or out with the last bit of acosf, which
# differs between the device and the host library (measured: 2.4e-3 rel-L2 for the
# illumination-normalised image).  A wrong index or operand gives errors near 1.
TOL_ANGLE = 1e-2


def cfg_from(G, s):
    return G.SurveyConfig(**s)


def golden_run(G, name, options=None):
    z, prm = load_case(name)
    s = survey_from_case(prm)
    shots = list(range(1, prm["nshot"] + 1))
    gathers = None
    if prm["mode"] == 1:
        src, _ = load_case(prm["data_from"])
        gathers = [src[f"gather{i}"] for i in shots]
    out = G.migrate(cfg_from(G, s), options or G.RunOptions(), shots, z["vp0"], z["rho0"], gathers=gathers)
    return z, prm, out


@pytest.mark.parametrize("name", ["caseB", "caseC", "caseD"])
def test_images_match_reference(rtmlib, name):
    z, prm, out = golden_run(rtmlib, name)
    for k in ("image1", "image2s", "image2m", "illum"):
        assert rel_l2(out[k], z[k]) < TOL_FP32, (k, rel_l2(out[k], z[k]))
    if prm["mode"] == 0:
        for i in range(1, prm["nshot"] + 1):
            assert rel_l2(out["gathers"][i - 1], z[f"gather{i}"]) < TOL_FP32


def test_forward_matches_reference_steps(rtmlib):
    """300 forward steps against the reference's 9-launch step (golden units run)."""
    z = np.load(os.path.join(GOLDEN, "ref_units.npz"))
    nxl, nzl, npml, dx, dz, dt, fdom, nt, nsx, nsz, amp, alp = z["units_meta"]
    nxl, nzl, npml, nt, nsx, nsz = map(int, (nxl, nzl, npml, nt, nsx, nsz))
    nsteps = int(z["units_meta2"][2])
    sv = rtmlib.SurveyConfig(nx=nxl, nz=nzl, nt=nt, dx=float(dx), dz=float(dz), dt=float(dt), npml=npml,
                             fdom=float(fdom), amp=float(amp), alp=float(alp), layout=2,
                             spx0=(nsx - npml) * float(dx), spz0=(nsz - npml) * float(dz), mode=0)
    g = rtmlib.geometry(sv, 1)
    assert (g.nsx, g.nsz) == (nsx, nsz)
    v = z["model_v"].reshape(nzl, nxl)
    r = z["model_rho"].reshape(nzl, nxl)
    p, vx, vz, gat = rtmlib.forward(sv, rtmlib.RunOptions(), 1, v, r, nsteps)
    X, Z = nxl + 2 * npml, nzl + 2 * npml
    assert rel_l2(p, z["fwd_p"].reshape(Z, X)) < TOL_FP32
    assert rel_l2(vx, z["fwd_vx"].reshape(Z, X - 1)) < TOL_FP32
    assert rel_l2(vz, z["fwd_vz"].reshape(Z - 1, X)) < TOL_FP32
    assert rel_l2(gat, z["fwd_gather"].reshape(nsteps, nxl)) < TOL_FP32


def _units_survey(rtmlib, z, mode):
    """The survey of the reference's unit run (ref_units.npz): 96 x 64 interior, npml 32,
    source at (nsx, nsz), receivers on the first interior row, nw = 60 and tlength = 50 for
    the direct-wave mute (direct = 1.5, direct0 = 0.05 s)."""
    nxl, nzl, npml, dx, dz, dt, fdom, nt, nsx, nsz, amp, alp = z["units_meta"]
    nxl, nzl, npml, nt, nsx, nsz = map(int, (nxl, nzl, npml, nt, nsx, nsz))
    f = lambda v: float(np.float32(v))
    return rtmlib.SurveyConfig(nx=nxl, nz=nzl, nt=nt, dx=f(dx), dz=f(dz), dt=f(dt), npml=npml, fdom=f(fdom),
                               amp=f(amp), alp=f(alp), layout=2, spx0=(nsx - npml) * f(dx),
                               spz0=(nsz - npml) * f(dz), mode=mode, direct=1.5, direct0=f(0.05), mute=1)


def test_device_pml_profiles_bit_exact(rtmlib):
    """The session's device PML profiles (k_setup_pml, from the vpmax of the shot's model
    window) equal the reference's cuda_pmlCoeffpx/pz/vx/vz output bit for bit.  The
    reference's unit run used vpmax = 3000 m/s; the model is capped there so that the
    session's vpmax = sqrt(max v^2) is exactly 3000."""
    z = np.load(os.path.join(GOLDEN, "ref_units.npz"))
    assert float(z["units_meta2"][1]) == 3000.0
    s = _units_survey(rtmlib, z, 1)
    v = np.minimum(z["model_v"].reshape(s.nz, s.nx), np.float32(3000.0))
    assert v.max() == np.float32(3000.0)
    r = z["model_rho"].reshape(s.nz, s.nx)
    g = rtmlib.geometry(s, 1)
    with rtmlib.Session(s, rtmlib.RunOptions(), [1], v, r) as ss:
        got = ss.pml_profiles(0, g.nxpad, g.nzpad)
    for name, a in zip(("pml_ddx", "pml_ddz", "pml_ddxvx", "pml_ddzvz"), got):
        assert np.array_equal(a.view(np.int32), z[name].view(np.int32)), name


def test_device_mute_mask_bit_exact(rtmlib):
    """The device mute (k_mute on the session's gather) of an all-ones gather equals the
    reference's cuda_mute1 mask bit for bit (receivers on the first interior row, the unit
    run's model, nw = 60, tlength = 50)."""
    z = np.load(os.path.join(GOLDEN, "ref_units.npz"))
    s = _units_survey(rtmlib, z, 1)
    v = z["model_v"].reshape(s.nz, s.nx)
    r = z["model_rho"].reshape(s.nz, s.nx)
    assert list(z["mute_meta"]) == [int(np.float32(1.5) / (np.float32(s.fdom) * np.float32(s.dt))), 50]
    with rtmlib.Session(s, rtmlib.RunOptions(), [1], v, r) as ss:
        ss.set_gather(0, np.ones((s.nt, ss.nrec(0)), np.float32))
        got = ss.gather(0)
    want = z["mute_mask"].reshape(s.nt, s.nx)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    assert 0 < (got == 0).sum() < got.size   # the mask cuts part of every trace, not all


def _random_model(nz, nx, seed):
    rng = np.random.default_rng(seed)
    zz = np.arange(nz)[:, None] * 10.0
    v = 1800 + 0.9 * zz + 150 * rng.random((nz, nx))
    v[nz // 2:, :] += 500
    rho = 1900 + 200 * rng.random((nz, nx))
    return v.astype(np.float32), rho.astype(np.float32)


GENERAL = [
    # general npml, sizes that leave partial tiles, receivers below z = 0, constant density
    dict(nx=77, nz=45, nt=260, npml=40, layout=2, spx0=300.0, spz0=20.0, dspx=200.0, nshot=2, rdepth=0,
         rho="const", fdom=25.0, alp=0.1),
    dict(nx=101, nz=53, nt=240, npml=13, layout=2, spx0=150.0, spz0=35.0, dspx=330.0, nshot=2, rdepth=3,
         rho="var", fdom=25.0, alp=0.06),
    # bilateral apertures of different widths in one batch, PML smoothing, ismth reconstruction
    dict(nx=150, nz=41, nt=220, npml=24, layout=1, spx0=100.0, spz0=20.0, dspx=450.0, nshot=3, rdepth=0,
         rho="var", offsetmax=900.0, medium_flag=1, ismth=2, fdom=25.0, alp=0.1),
    # unilateral layouts with a minimum offset
    dict(nx=120, nz=40, nt=200, npml=20, layout=3, spx0=60.0, spz0=20.0, dspx=300.0, nshot=2, rdepth=0,
         rho="const", offset=50.0, offsetmax=600.0, fdom=25.0, alp=0.1),
    dict(nx=120, nz=40, nt=200, npml=20, layout=4, spx0=700.0, spz0=20.0, dspx=300.0, nshot=2, rdepth=0,
         rho="const", offset=50.0, offsetmax=600.0, fdom=25.0, alp=0.1),
]


def _survey(c, mode):
    return dict(nx=c["nx"], nz=c["nz"], nt=c["nt"], dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=c["npml"],
                fdom=c["fdom"], amp=1.0, alp=c["alp"], layout=c["layout"], spx0=c["spx0"], spz0=c["spz0"],
                dspx=c["dspx"], offset=c.get("offset", 0.0), offsetmax=c.get("offsetmax", 0.0), mode=mode,
                medium_flag=c.get("medium_flag", 0), ismth=c.get("ismth", 0), direct=1.5, direct0=0.0, mute=1,
                receiver_depth=c["rdepth"])


@pytest.mark.parametrize("ci", range(len(GENERAL)))
def test_rtm_matches_oracle_general(rtmlib, oracle, ci):
    c = GENERAL[ci]
    v, rho = _random_model(c["nz"], c["nx"], ci)
    if c["rho"] == "const":
        rho = np.full_like(rho, 2000.0)
    shots = list(range(1, c["nshot"] + 1))
    s = _survey(c, 0)
    ref = oracle.rtm_model(s, shots, v, rho)
    out = rtmlib.migrate(cfg_from(rtmlib, s), rtmlib.RunOptions(), shots, v, rho)
    for k in range(len(shots)):
        assert rel_l2(out["gathers"][k], ref["gathers"][k]) < TOL_FP32
    for k in ("image1", "image2s", "illum"):
        assert rel_l2(out[k], ref[k]) < TOL_FP32, (k, rel_l2(out[k], ref[k]))
    # mode 1 on the modelled data with a smoothed migration model
    vm = oracle.velsmooth(v, 3)
    s1 = _survey(c, 1)
    ref1 = oracle.rtm_model(s1, shots, vm, rho, gathers=ref["gathers"])
    out1 = rtmlib.migrate(cfg_from(rtmlib, s1), rtmlib.RunOptions(), shots, vm, rho, gathers=ref["gathers"])
    for k in ("image1", "image2s", "illum"):
        assert rel_l2(out1[k], ref1[k]) < TOL_FP32, (k, rel_l2(out1[k], ref1[k]))


def test_batching_is_bitwise_invariant(rtmlib):
    """A batch of uneven apertures in one launch gives exactly the per-shot results."""
    c = GENERAL[2]
    v, rho = _random_model(c["nz"], c["nx"], 7)
    s = cfg_from(rtmlib, _survey(c, 0))
    shots = [1, 2, 3]
    a = rtmlib.migrate(s, rtmlib.RunOptions(batch=1), shots, v, rho)
    b = rtmlib.migrate(s, rtmlib.RunOptions(batch=3), shots, v, rho)
    for k in ("image1", "image2s", "illum"):
        assert np.array_equal(a[k], b[k]), k
    for ga, gb in zip(a["gathers"], b["gathers"]):
        assert np.array_equal(ga, gb)
    assert a["stats"].batches == 3 and b["stats"].batches == 1


@pytest.mark.parametrize("strips,gathers,fp64", [("fp16", "fp16", True), ("bf16", "bf16", True),
                                                 ("fp16", "fp32", False), ("fp32", "fp32", True),
                                                 ("fp16", "fp16", 3)])
def test_precision_forms_against_fp64_oracle(rtmlib, oracle, strips, gathers, fp64):
    c = GENERAL[0]
    v, rho = _random_model(c["nz"], c["nx"], 11)
    shots = [1, 2]
    s0 = _survey(c, 0)
    data = oracle.rtm_model(s0, shots, v, rho)["gathers"]
    vm = oracle.velsmooth(v, 3)
    s1 = _survey(c, 1)
    ref64 = oracle.rtm_model(s1, shots, vm, rho, gathers=data, precision="f64")
    out = rtmlib.migrate(cfg_from(rtmlib, s1), rtmlib.RunOptions(strip_precision=strips, gather_precision=gathers,
                                                                 accum_fp64=fp64), shots, vm, rho, gathers=data)
    tol = TOL_MIXED if (strips != "fp32" or gathers != "fp32") else TOL_FP32
    if strips == "bf16":
        tol = 2e-2   # 8-bit mantissa storage; reported, not the north-star form
    for k in ("image1", "image2s", "illum"):
        err = rel_l2(out[k], ref64[k])
        assert err < tol, (k, err)
    if fp64:
        f = out["f64"]
        assert rel_l2(f["image2s"], ref64["image2s"]) < tol


def test_reconstructed_source_wavefield_drift(rtmlib, oracle):
    """The fp16 boundary strips perturb the reconstructed source wavefield only slightly."""
    c = GENERAL[0]
    v, rho = _random_model(c["nz"], c["nx"], 12)
    s = rtmlib.SurveyConfig(**_survey(c, 0))
    res = {}
    for prec in ("fp32", "fp16"):
        with rtmlib.Session(s, rtmlib.RunOptions(strip_precision=prec, batch=1), [1], v, rho) as ss:
            ss.run()
            g = rtmlib.geometry(s, 1)
            res[prec] = ss.wavefields(0, g.nxpad, g.nzpad)[0]
    npml = c["npml"]
    inner = (slice(npml, -npml), slice(npml, -npml))
    drift = rel_l2(res["fp16"][inner], res["fp32"][inner])
    assert drift < 1e-3, drift


def test_dropin_rtm_model_writes_reference_files(rtmlib, tmp_path, monkeypatch):
    """rtm_model() with the reference's argument list: mode 0 writes the gathers the
    reference wrote (byte for byte in the headers), mode 1 reads them back; the images match
    the reference's, image3/4/5 too with the reference's indexing selected."""
    monkeypatch.setenv("RTM_B200_EXTRA_IMAGES", "2")
    z, prm = load_case("caseB")
    zc, prmc = load_case("caseC")
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        os.makedirs("seisReal")
        os.makedirs("output")
        nx, nz = prm["nx"], prm["nz"]
        imgs = [np.zeros((nz, nx), np.float32) for _ in range(10)]
        coef = rtmlib.coef_table()
        wl = np.zeros(prm["nt"], np.float32)
        L = rtmlib.lib()
        f = lambda x: C.c_float(float(x))

        def call(p, vp, rho):
            L.rtm_model(0, p["nshot"], 1, 1, p["mode"], p["medium_flag"], p["layout"], 0, 0, p["ismth"], nx, nz,
                        p["nt"], f(p["dx"]), f(p["dx"]), f(p["dt"]), p["npml"], f(p["direct"]), f(p["direct0"]),
                        f(0.25), f(p["fdom"]), f(p["spx0"]), f(p["spz0"]), f(p["dspx"]), f(p["offset"]),
                        f(p["offsetmax"]), f(p["amp"]), f(p["alp"]), vp.ctypes.data_as(C.c_void_p),
                        rho.ctypes.data_as(C.c_void_p), coef.ctypes.data_as(C.c_void_p),
                        wl.ctypes.data_as(C.c_void_p), *[a.ctypes.data_as(C.c_void_p) for a in imgs])
            assert L.rtm_last_error() == b""

        call(prm, np.ascontiguousarray(z["vp0"]), np.ascontiguousarray(z["rho0"]))
        for i in (1, 2):
            raw = np.fromfile(f"seisReal/{i}seisreal.su", np.uint8).reshape(prm["nx"], 240 + 4 * prm["nt"])
            assert np.array_equal(raw[:, :240], z[f"gather{i}_headers"])
            data = raw[:, 240:].copy().view(np.float32).reshape(prm["nx"], prm["nt"]).T
            assert rel_l2(data, z[f"gather{i}"]) < TOL_FP32
        assert rel_l2(imgs[0], z["image1"]) < TOL_FP32
        assert rel_l2(imgs[1], z["image2s"]) < TOL_FP32
        assert rel_l2(imgs[9], z["illum"]) < TOL_FP32
        for k, i in (("image4s", 3), ("image5s", 4), ("image4m", 7), ("image5m", 8)):
            assert rel_l2(imgs[i], z[k]) < TOL_FP32, k
        for k, i in (("image3s", 2), ("image3m", 6)):
            assert rel_l2(imgs[i], z[k]) < TOL_DECOMP, k
        hdr = np.fromfile("output/Image1temp.su", np.uint8)
        assert np.array_equal(hdr[:240], z["image_su_header0"]) and hdr.size == z["image_su_bytes"][0]
        # mode 1 reads ./seisReal written above (the reference's own caseC run did the same)
        call(prmc, np.ascontiguousarray(zc["vp0"]), np.ascontiguousarray(zc["rho0"]))
        assert rel_l2(imgs[1], zc["image2s"]) < TOL_FP32
        assert rel_l2(imgs[0], zc["image1"]) < TOL_FP32
    finally:
        os.chdir(cwd)


def test_edge_cases(rtmlib, oracle):
    v, rho = _random_model(30, 40, 3)
    base = dict(nx=40, nz=30, nt=2, dx=10.0, dz=10.0, dt=float(np.float32(1e-3)), npml=10, fdom=25.0, amp=1.0,
                alp=0.1, layout=2, spx0=200.0, spz0=20.0, dspx=0.0, mode=0, direct=1.5, direct0=0.0)
    # minimum time axis and minimum PML width
    out = rtmlib.migrate(rtmlib.SurveyConfig(**base), rtmlib.RunOptions(), [1], v, rho)
    ref = oracle.rtm_model(dict(base, offset=0.0, offsetmax=0.0, medium_flag=0, ismth=0, mute=1, receiver_depth=0),
                           [1], v, rho)
    assert rel_l2(out["gathers"][0], ref["gathers"][0]) < TOL_FP32
    # zero amplitude: everything stays exactly zero
    out = rtmlib.migrate(rtmlib.SurveyConfig(**dict(base, nt=50, amp=0.0)), rtmlib.RunOptions(), [1], v, rho)
    assert not out["image1"].any() and not out["gathers"][0].any()
    # source Gaussian wide enough to cover the whole grid (alp = 0 -> flat source)
    s = dict(base, nt=40, alp=0.0)
    out = rtmlib.migrate(rtmlib.SurveyConfig(**s), rtmlib.RunOptions(), [1], v, rho)
    ref = oracle.rtm_model(dict(s, offset=0.0, offsetmax=0.0, medium_flag=0, ismth=0, mute=1, receiver_depth=0),
                           [1], v, rho)
    assert rel_l2(out["gathers"][0], ref["gathers"][0]) < TOL_FP32
    # mode 1 without data is an error, not a crash
    with pytest.raises(rtmlib.RtmError, match="gather"):
        with rtmlib.Session(rtmlib.SurveyConfig(**dict(base, mode=1)), rtmlib.RunOptions(), [1], v, rho) as ss:
            ss.run()
    # a survey larger than the device is refused up front (strips of 10^8 steps, ~1 TB)
    big = dict(base, nt=100_000_000)
    with pytest.raises(rtmlib.RtmError, match="device memory"):
        rtmlib.Session(rtmlib.SurveyConfig(**big), rtmlib.RunOptions(), [1], v, rho)


EXTRA = ("image3s", "image4s", "image5s", "image3m", "image4m", "image5m", "imagetrue")


@pytest.mark.parametrize("name", ["caseB", "caseC", "caseD"])
def test_extra_images_match_reference(rtmlib, name):
    """The reference's other imaging conditions, with its own indexing (extra_images=2),
    against the image3/4/5 its rtm_model() returned."""
    z, prm, out = golden_run(rtmlib, name, rtmlib.RunOptions(extra_images=2))
    for k in ("image4s", "image4m", "image5s", "image5m"):
        assert rel_l2(out[k], z[k]) < TOL_FP32, (k, rel_l2(out[k], z[k]))
    for k in ("image3s", "image3m"):
        assert rel_l2(out[k], z[k]) < TOL_DECOMP, (k, rel_l2(out[k], z[k]))


@pytest.mark.parametrize("extra", [1, 2])
def test_extra_images_match_oracle(rtmlib, oracle, extra):
    """Both indexing forms against the oracle at an amplitude where the Poynting angles are
    not degenerate (at amp = 1 the float product under its square root underflows, as in the
    reference, and every angle weight is 1/sqrt(2))."""
    c = dict(GENERAL[1], amp=1e4)
    v, rho = _random_model(c["nz"], c["nx"], 11)
    shots = list(range(1, c["nshot"] + 1))
    s = dict(_survey(c, 0), amp=1e4)
    ref = oracle.rtm_model(s, shots, v, rho, extra=extra)
    out = rtmlib.migrate(cfg_from(rtmlib, s), rtmlib.RunOptions(extra_images=extra), shots, v, rho)
    assert rel_l2(ref["image4m"], ref["image1"] / np.sqrt(2)) > 0.1   # the angles matter here
    for k in ("image1", "image5s", "image5m"):
        assert rel_l2(out[k], ref[k]) < TOL_FP32, (k, rel_l2(out[k], ref[k]))
    for k in ("image4s", "image4m"):
        assert rel_l2(out[k], ref[k]) < TOL_ANGLE, (k, rel_l2(out[k], ref[k]))
    # imagetrue weights each term by 1/sin(theta) with theta = pi/2 - acos(w)/2: where the
    # source and receiver Poynting vectors are nearly opposite (w -> -1, at reflectors) the
    # weight diverges and acos has an infinite slope, so the few time steps near that point
    # decide each cell's sum and last-bit rounding of the wavefields moves it.  The oracle's
    # own fp32 and fp64 forms differ by 0.57 rel-L2 on this case (and by 1.0 with the
    # reference's indexing); the device result lies 0.12-0.36 from the fp32 oracle.  Only a
    # loose bound is meaningful.
    assert rel_l2(out["imagetrue"], ref["imagetrue"]) < 0.5, rel_l2(out["imagetrue"], ref["imagetrue"])
    for k in ("image3s", "image3m"):
        assert rel_l2(out[k], ref[k]) < TOL_DECOMP, (k, rel_l2(out[k], ref[k]))


def test_extra_images_leave_the_main_images_unchanged(rtmlib):
    """Turning the other imaging conditions on changes nothing in image1/image2s/illum."""
    z, prm, a = golden_run(rtmlib, "caseB")
    _, _, b = golden_run(rtmlib, "caseB", rtmlib.RunOptions(extra_images=1))
    for k in ("image1", "image2s", "illum"):
        assert np.array_equal(a[k], b[k]), k


def test_rtm_batch_refuses_null_without_gpu(rtmlib):
    assert rtmlib.lib().rtm_batch(None, None) == rtmlib.RTM_ERR_ARG


@pytest.mark.gpu
def test_rtm_batch_descriptor_equals_session(rtmlib):
    """rtm_batch (one descriptor: survey, options, shots, models, gathers, images) gives the
    images and gathers of the session API, bit for bit."""
    G = rtmlib
    c = GENERAL[2]
    v, rho = _random_model(c["nz"], c["nx"], 2)
    shots = list(range(1, c["nshot"] + 1))
    s = cfg_from(G, _survey(c, 0))
    opts = G.RunOptions(batch=2)
    want = G.migrate(s, opts, shots, v, rho)
    d = G.BatchDesc()
    d.survey, d.options = s.c(), opts.c()
    ids = np.ascontiguousarray(shots, np.int32)
    d.shots, d.nshots = ids.ctypes.data_as(C.POINTER(C.c_int)), len(shots)
    v32, r32 = np.ascontiguousarray(v, np.float32), np.ascontiguousarray(rho, np.float32)
    d.vp, d.rho = v32.ctypes.data, r32.ctypes.data
    gouts = [np.zeros_like(g) for g in want["gathers"]]
    gp = (C.c_void_p * len(shots))(*[g.ctypes.data for g in gouts])
    d.gathers_out = C.cast(gp, C.POINTER(C.c_void_p))
    imgs = {k: np.zeros((c["nz"], c["nx"]), np.float32) for k in ("image1", "image2s", "image2m", "illum")}
    for k, a in imgs.items():
        setattr(d, k, a.ctypes.data)
    st = G.Stats()
    assert G.lib().rtm_batch(C.byref(d), C.byref(st)) == 0, G.lib().rtm_last_error()
    assert st.shots == len(shots) and st.batches == 2
    for k in ("image1", "image2s", "illum"):
        assert np.array_equal(imgs[k], want[k]), k
    for a, b in zip(gouts, want["gathers"]):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("fp64", [False, True])
def test_interior_tile_form_is_bitwise_identical(rtmlib, monkeypatch, fp64):
    """The pressure kernel's interior-tile form (tiles with no PML, source or receiver cell)
    gives the same bits as the general form on every tile (RTM_B200_FAST_TILES=0): gathers
    and images of the general cases, fp32 and fp64 accumulators, with the other imaging
    conditions."""
    G = rtmlib
    for ci, c in enumerate(GENERAL):
        v, rho = _random_model(c["nz"], c["nx"], ci)
        shots = list(range(1, c["nshot"] + 1))
        s = cfg_from(G, _survey(c, 0))
        opts = G.RunOptions(accum_fp64=fp64, extra_images=1)
        monkeypatch.setenv("RTM_B200_FAST_TILES", "0")
        want = G.migrate(s, opts, shots, v, rho)
        monkeypatch.delenv("RTM_B200_FAST_TILES")
        got = G.migrate(s, opts, shots, v, rho)
        for k in ("image1", "image2s", "illum", "image3s", "image4s", "image5s", "imagetrue"):
            assert np.array_equal(got[k], want[k]), (ci, k)
        for a, b in zip(got["gathers"], want["gathers"]):
            assert np.array_equal(a, b), ci


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_packed_strips_and_gathers_survive_subnormal_values(rtmlib, prec):
    """The source lies 150-200 cells from the strips and the receiver row, so the stencil's
    exponentially small forerunner arrives there long before the wave: the first non-zero
    values of the strips and of the gather are subnormal floats, whose power-of-two scale has
    no finite reciprocal.  The packed forms must stay finite and close to fp32."""
    G = rtmlib
    v, rho = _random_model(300, 400, 5)
    # dt = 0.5 ms keeps v dt / dx = 0.26 for the model's fastest cells (5140 m/s) inside the
    # stability limit (about 0.48 for this 20th-order scheme in 2-D)
    s = dict(nx=400, nz=300, nt=1600, dx=10.0, dz=10.0, dt=float(np.float32(5e-4)), npml=20, fdom=25.0, amp=1.0,
             alp=0.1, layout=2, spx0=2000.0, spz0=1500.0, dspx=0.0, offset=0.0, offsetmax=0.0, mode=0,
             medium_flag=0, ismth=0, direct=1.5, direct0=0.0, mute=1, receiver_depth=0)
    cfg = cfg_from(G, s)
    ref = G.migrate(cfg, G.RunOptions(accum_fp64=True), [1], v, rho)
    got = G.migrate(cfg, G.RunOptions(strip_precision=prec, gather_precision=prec, accum_fp64=True), [1], v, rho)
    tol = 1e-3 if prec == "fp16" else 2e-2
    for k in ("image1", "image2s", "illum"):
        assert np.isfinite(got[k]).all(), k
        assert np.abs(ref[k]).max() > 0
        assert rel_l2(got[k], ref[k]) < tol, (k, rel_l2(got[k], ref[k]))


@pytest.mark.gpu
def test_tile_heights_do_not_change_the_bits(rtmlib, monkeypatch):
    """Tile heights (and with them the row groups and the interior/general split of the tiles)
    only reorganise the work: gathers and images are bit-identical for every choice, the
    reconstruction pressure's height different from the other pressure kernels' too."""
    G = rtmlib
    c = GENERAL[2]
    v, rho = _random_model(c["nz"], c["nx"], 7)
    shots = list(range(1, c["nshot"] + 1))
    s = cfg_from(G, _survey(c, 0))
    runs = []
    for vel, recon, pres, pres_recon in ((None, None, None, None), ("16", "32", "32", "8"), ("8", "8", "8", "32"),
                                         ("64", "16", "64", "16")):
        for k, val in (("RTM_B200_BZ_VEL", vel), ("RTM_B200_BZ_VEL_RECON", recon), ("RTM_B200_BZ_PRES", pres),
                       ("RTM_B200_BZ_PRES_RECON", pres_recon)):
            if val is None:
                monkeypatch.delenv(k, raising=False)
            else:
                monkeypatch.setenv(k, val)
        runs.append(G.migrate(s, G.RunOptions(extra_images=1), shots, v, rho))
    for r in runs[1:]:
        for k in ("image1", "image2s", "illum", "image3s", "image5s"):
            assert np.array_equal(r[k], runs[0][k]), k
        for a, b in zip(r["gathers"], runs[0]["gathers"]):
            assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("strips,graph", [("fp32", 1), ("fp16", 1), ("fp32", 2), ("fp16", 2)])
def test_graph_replay_is_bitwise_identical(rtmlib, monkeypatch, strips, graph):
    """use_graph: each pass's time loop captured once per launch shape (1) or per rounded
    grid (2, blocks past the batch's tiles return) and replayed gives the gathers and images of
    direct launches bit for bit.  One shot per launch over shots of three window widths
    (layout 1, offsetmax cut at the model's edges), so that graphs are both captured and
    replayed, with packed strips too."""
    G = rtmlib
    monkeypatch.setenv("RTM_B200_TUNE", "0")   # tile-height trials would add launches to the first run only
    c = GENERAL[2]
    v, rho = _random_model(c["nz"], c["nx"], 9)
    s = cfg_from(G, _survey(c, 0))
    shots = [1, 2, 3, 1, 3]
    widths = {G.geometry(s, k).nxpad for k in shots}
    assert len(widths) > 1
    base = dict(batch=1, strip_precision=strips)
    want = G.migrate(s, G.RunOptions(**base), shots, v, rho)
    got = G.migrate(s, G.RunOptions(use_graph=graph, **base), shots, v, rho)
    for k in ("image1", "image2s", "illum"):
        assert np.array_equal(got[k], want[k]), k
    for a, b in zip(got["gathers"], want["gathers"]):
        assert np.array_equal(a, b)
    assert got["stats"].kernel_launches == want["stats"].kernel_launches


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp32", "fp64", "fp16"])
def test_vector_kernel_form_is_bitwise_identical(rtmlib, monkeypatch, form):
    """The four-columns-by-U-rows kernels (default) give the bits of the one-column kernels
    (RTM_B200_KERNELS=scalar): gathers and images of the general cases (partial tiles, npml
    13-40, layouts 1-4, receivers below z = 0), at every tile height, with fp64 accumulators
    and the other imaging conditions, and with packed strips and gathers."""
    G = rtmlib
    opts = dict(fp32=dict(), fp64=dict(accum_fp64=True, extra_images=1),
                fp16=dict(strip_precision="fp16", gather_precision="fp16"))[form]
    heights = [(None, None, None), ("16", "32", "32"), ("8", "8", "8")]
    for ci, c in enumerate(GENERAL):
        v, rho = _random_model(c["nz"], c["nx"], 20 + ci)
        shots = list(range(1, c["nshot"] + 1))
        s = cfg_from(G, _survey(c, 0))
        for vel, recon, pres in heights[:1] if ci else heights:
            for k, val in (("RTM_B200_BZ_VEL", vel), ("RTM_B200_BZ_VEL_RECON", recon), ("RTM_B200_BZ_PRES", pres)):
                if val is None:
                    monkeypatch.delenv(k, raising=False)
                else:
                    monkeypatch.setenv(k, val)
            monkeypatch.setenv("RTM_B200_KERNELS", "scalar")
            want = G.migrate(s, G.RunOptions(**opts), shots, v, rho)
            monkeypatch.setenv("RTM_B200_KERNELS", "vector")
            got = G.migrate(s, G.RunOptions(**opts), shots, v, rho)
            keys = ["image1", "image2s", "illum"] + (["image3s", "image4s", "image5s"] if form == "fp64" else [])
            for k in keys:
                assert np.array_equal(got[k], want[k]), (ci, vel, k)
            for a, b in zip(got["gathers"], want["gathers"]):
                assert np.array_equal(a, b), (ci, vel)


@pytest.mark.gpu
def test_tile_height_tuner(rtmlib, monkeypatch, tmp_path):
    """The tuner times 8-, 16- and 32-row tiles before the first batch of a launch shape,
    keeps a height per kernel family, records it in RTM_B200_TUNE_CACHE, and changes no bit
    of the results (RTM_B200_TUNE=0 runs the default heights)."""
    G = rtmlib
    c = dict(GENERAL[1], nx=97)   # a launch shape no other test uses
    v, rho = _random_model(c["nz"], c["nx"], 31)
    shots = list(range(1, c["nshot"] + 1))
    s = cfg_from(G, _survey(c, 0))
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("RTM_B200_TUNE_CACHE", str(cache))
    for k in ("RTM_B200_BZ_VEL", "RTM_B200_BZ_VEL_RECON", "RTM_B200_BZ_PRES", "RTM_B200_BZ_PRES_RECON", "RTM_B200_TUNE"):
        monkeypatch.delenv(k, raising=False)
    with G.Session(s, G.RunOptions(), shots, v, rho) as ss:
        ss.run()
        h = ss.tile_heights()
        tuned = ss.images()
        gathers = [ss.gather(k) for k in range(len(shots))]
    assert set(h.values()) <= {8, 16, 32}
    lines = cache.read_text().split("\n")
    want_line = [str(h[k]) for k in ("vel", "vel_recon", "pres", "pres_recon")]
    assert any(ln.split()[1:5] == want_line for ln in lines if ln), lines
    monkeypatch.setenv("RTM_B200_TUNE", "0")
    want = G.migrate(s, G.RunOptions(), shots, v, rho)
    for k in ("image1", "image2s", "illum"):
        assert np.array_equal(tuned[k], want[k]), k
    for a, b in zip(gathers, want["gathers"]):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_compensated_fp32_accumulation(rtmlib, monkeypatch):
    """accum_fp64 = 2: compensated fp32 pairs (Kahan) for the per-shot g1 and illumination,
    stacked in fp64: within 1e-6 rel-L2 of fp64 accumulation of the same FP32 wavefields, and
    the same bits from both kernel forms."""
    G = rtmlib
    c = GENERAL[0]
    v, rho = _random_model(c["nz"], c["nx"], 13)
    shots = [1, 2]
    s = cfg_from(G, _survey(c, 0))
    d64 = G.migrate(s, G.RunOptions(accum_fp64=1), shots, v, rho)
    dk = G.migrate(s, G.RunOptions(accum_fp64=2), shots, v, rho)
    for k in ("image1", "image2s", "illum"):
        assert np.abs(d64["f64"][k]).max() > 0
        assert rel_l2(dk["f64"][k], d64["f64"][k]) < 1e-6, (k, rel_l2(dk["f64"][k], d64["f64"][k]))
    monkeypatch.setenv("RTM_B200_KERNELS", "scalar")
    ds = G.migrate(s, G.RunOptions(accum_fp64=2), shots, v, rho)
    for k in ("image1", "image2s", "illum"):
        assert np.array_equal(ds["f64"][k], dk["f64"][k]), k


@pytest.mark.gpu
def test_blocked_fp64_accumulation(rtmlib, monkeypatch):
    """accum_fp64 = 3: the steps image into fp32 partial sums, which a flush adds into fp64
    totals every 32 steps and after the last (nt - 1 backward steps, not a multiple of 32
    here): within 1e-6 rel-L2 of fp64 accumulation every step; the same bits from both kernel
    forms, from graph replays, from one shot per launch, and from the whole-step kernel; the
    other imaging conditions (their accumulators fp64 as before) within 1e-6 too."""
    G = rtmlib
    c = GENERAL[0]
    assert (c["nt"] - 1) % 32
    v, rho = _random_model(c["nz"], c["nx"], 17)
    shots = [1, 2]
    s = cfg_from(G, _survey(c, 0))
    d64 = G.migrate(s, G.RunOptions(accum_fp64=1, extra_images=1), shots, v, rho)
    db = G.migrate(s, G.RunOptions(accum_fp64=3, extra_images=1), shots, v, rho)
    for k in ("image1", "image2s", "illum"):
        assert np.abs(d64["f64"][k]).max() > 0
        assert rel_l2(db["f64"][k], d64["f64"][k]) < 1e-6, (k, rel_l2(db["f64"][k], d64["f64"][k]))
    for k in ("image3s", "image4s", "image5s"):   # normalised by the (blocked) illumination
        assert rel_l2(db[k], d64[k]) < 1e-6, (k, rel_l2(db[k], d64[k]))
    variants = [("scalar", {}, {"RTM_B200_KERNELS": "scalar"}), ("vector", {}, {"RTM_B200_KERNELS": "vector"}),
                ("graph", {"use_graph": 1}, {}), ("rounded graph", {"use_graph": 2, "batch": 1}, {}),
                ("per shot", {"batch": 1}, {}),
                ("whole step", {}, {"RTM_B200_FUSED": "1", "RTM_B200_TZ_STEP": "16"})]
    for name, opts, env in variants:
        with monkeypatch.context() as m:
            for k, val in env.items():
                m.setenv(k, val)
            dv = G.migrate(s, G.RunOptions(accum_fp64=3, **opts), shots, v, rho)
        for k in ("image1", "image2s", "illum"):
            assert np.array_equal(dv["f64"][k], db["f64"][k]), (name, k)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp32", "fp64", "fp16", "kahan"])
def test_whole_step_kernel_is_bitwise_identical(rtmlib, monkeypatch, form):
    """The whole-step kernel (velocity and pressure of a step in one launch, two buffers per
    field; RTM_B200_FUSED=1) gives the bits of the split kernels: gathers, images (the other
    imaging conditions too) and the final wavefields of the general cases, at 16- and 32-row
    tiles, with packed strips and gathers, fp64 and compensated accumulators, and with the
    passes replayed as CUDA graphs."""
    G = rtmlib
    opts = dict(fp32=dict(), fp64=dict(accum_fp64=1, extra_images=1),
                fp16=dict(strip_precision="fp16", gather_precision="fp16", use_graph=2),
                kahan=dict(accum_fp64=2, batch=1))[form]
    for ci, c in enumerate(GENERAL):
        v, rho = _random_model(c["nz"], c["nx"], 40 + ci)
        shots = list(range(1, c["nshot"] + 1))
        s = cfg_from(G, _survey(c, 0))
        monkeypatch.setenv("RTM_B200_FUSED", "0")
        want = G.migrate(s, G.RunOptions(**opts), shots, v, rho)
        for tz in ("16", "32"):
            monkeypatch.setenv("RTM_B200_FUSED", "1")
            monkeypatch.setenv("RTM_B200_TZ_STEP", tz)
            got = G.migrate(s, G.RunOptions(**opts), shots, v, rho)
            keys = ["image1", "image2s", "illum"] + (["image3s", "image4s", "image5s", "imagetrue"] if form == "fp64" else [])
            for k in keys:
                assert np.array_equal(got[k], want[k]), (ci, tz, k)
            for a, b in zip(got["gathers"], want["gathers"]):
                assert np.array_equal(a, b), (ci, tz)
        monkeypatch.delenv("RTM_B200_TZ_STEP")


@pytest.mark.gpu
def test_whole_step_kernel_wavefields_and_forward(rtmlib, monkeypatch):
    """With the whole-step kernel, the final wavefields of a migration and the fields after a
    number of forward steps (odd and even, so either buffer ends current) are those of the
    split kernels, bit for bit."""
    G = rtmlib
    c = GENERAL[1]
    v, rho = _random_model(c["nz"], c["nx"], 50)
    s = cfg_from(G, _survey(c, 0))
    g = G.geometry(s, 1)
    res = {}
    for fused in ("0", "1"):
        monkeypatch.setenv("RTM_B200_FUSED", fused)
        with G.Session(s, G.RunOptions(batch=1), [1], v, rho) as ss:
            ss.run()
            res[fused] = ss.wavefields(0, g.nxpad, g.nzpad)
        for nsteps in (37, 60):
            res[(fused, nsteps)] = G.forward(s, G.RunOptions(), 1, v, rho, nsteps)
    # the reconstruction writes its region (interior and strips, [npml-10, npml+n+10)); outside
    # it the second buffer holds older forward values that nothing reads
    npml = c["npml"]
    reg = (slice(npml - 10, g.nzpad - npml + 10), slice(npml - 10, g.nxpad - npml + 10))
    assert np.array_equal(res["1"][0][reg], res["0"][0][reg])
    assert np.array_equal(res["1"][1], res["0"][1])
    for nsteps in (37, 60):
        for a, b in zip(res[("1", nsteps)], res[("0", nsteps)]):
            assert np.array_equal(a, b), nsteps


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp32", "fp64", "kahan"])
def test_persistent_passes_are_bitwise_identical(rtmlib, monkeypatch, form):
    """RTM_B200_PERSIST=1: each pass in one persistent launch (device work queue, per-shot
    completion counters) gives the bits of the per-step launches: gathers and images of the
    general cases, several shots of uneven windows in one batch."""
    G = rtmlib
    opts = dict(fp32=dict(), fp64=dict(accum_fp64=1), kahan=dict(accum_fp64=2))[form]
    for ci, c in enumerate(GENERAL):
        v, rho = _random_model(c["nz"], c["nx"], 60 + ci)
        shots = list(range(1, c["nshot"] + 1))
        s = cfg_from(G, _survey(c, 0))
        monkeypatch.setenv("RTM_B200_PERSIST", "0")
        monkeypatch.setenv("RTM_B200_KERNELS", "scalar")
        monkeypatch.setenv("RTM_B200_TUNE", "0")
        want = G.migrate(s, G.RunOptions(**opts), shots, v, rho)
        monkeypatch.setenv("RTM_B200_PERSIST", "1")
        got = G.migrate(s, G.RunOptions(**opts), shots, v, rho)
        for k in ("image1", "image2s", "illum"):
            assert np.array_equal(got[k], want[k]), (ci, k)
        for a, b in zip(got["gathers"], want["gathers"]):
            assert np.array_equal(a, b), ci


@pytest.mark.gpu
def test_persistent_pass_wait_runs_out_cleanly(rtmlib, monkeypatch):
    """A persistent pass whose waits for other blocks' work items are bounded by 0 us gives up
    at its first unmet dependency: the call returns an error naming it (no hang), and the next
    run on the same device succeeds."""
    G = rtmlib
    c = GENERAL[1]
    v, rho = _random_model(c["nz"], c["nx"], 70)
    s = cfg_from(G, _survey(c, 0))
    monkeypatch.setenv("RTM_B200_PERSIST", "1")
    monkeypatch.setenv("RTM_B200_PASS_WAIT_US", "0")
    with pytest.raises(G.RtmError, match="persistent pass gave up"):
        G.migrate(s, G.RunOptions(), [1, 2], v, rho)
    monkeypatch.delenv("RTM_B200_PASS_WAIT_US")
    out = G.migrate(s, G.RunOptions(), [1, 2], v, rho)
    assert np.isfinite(out["image1"]).all() and np.abs(out["image1"]).max() > 0
