"""Host-side pieces of the path, checked without a GPU: the product's C-ABI host functions
(librtm_b200.so) against the reference's own host C++ (oracle/_ref/libref_host.so, built from
its sources) and against the oracle; the exported C-ABI; files byte for byte."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_case

_p = lambda a: a.ctypes.data_as(C.c_void_p)


def _model(nz, nx, seed=0):
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None]
    v = 1500 + 4.0 * z + 200 * rng.random((nz, nx))
    return v.astype(np.float32)


def test_capi_exports_every_declared_symbol(rtmlib):
    hdr = open(os.path.join(ROOT, "include", "rtm_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"\b(rtm_[a-z0-9_]+)\s*\(", hdr))
    assert "rtm_model" in names and "rtm_session_run" in names
    L = rtmlib.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", rtmlib.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}$", out, re.M), n


def test_coef_table_matches_reference(rtmlib, reflib, oracle):
    c = rtmlib.coef_table().reshape(10, 10)
    for h in range(1, 11):
        ref = np.zeros(10, np.float32)
        reflib.ref_Diff_coeffVelStrLiuyang(_p(ref), 2 * h)
        assert np.array_equal(c[h - 1, :h], ref[:h])
        assert not c[h - 1, h:].any()
    assert np.array_equal(oracle.coef_table(), c.ravel())


@pytest.mark.parametrize("npml,medium", [(32, 0), (40, 1), (11, 1)])
def test_prepare_model_matches_reference(rtmlib, reflib, npml, medium):
    nz, nx, nx1, nx2 = 37, 53, 7, 41
    v = _model(nz, nx)
    rho = (2000 + 100 * np.random.default_rng(3).random((nz, nx))).astype(np.float32)
    nxl = nx2 - nx1 + 1
    X, Z = nxl + 2 * npml, nz + 2 * npml
    vp2 = np.zeros((Z, X), np.float32)
    rp = np.zeros((Z, X), np.float32)
    assert rtmlib.lib().rtm_prepare_model(_p(v), _p(rho), nx, nz, nx1, nx2, npml, medium, _p(vp2), _p(rp)) == 0
    for arr, src, extract in ((vp2, v, reflib.ref_extractvel1), (rp, rho, reflib.ref_extractrho1)):
        tmp = np.zeros((nz, nxl), np.float32)
        extract(_p(tmp), _p(src), nx, nz, nx1, nx2)
        ref = np.zeros((Z, X), np.float32)
        reflib.ref_extendvel1(_p(ref), _p(tmp), nxl, nz, npml)
        if medium:
            reflib.ref_pmlvelsmooth1d(_p(ref), X, Z, npml)
        assert np.array_equal(arr.view(np.int32), ref.view(np.int32))


@pytest.mark.parametrize("nsp", [1, 3, 6])
def test_velsmooth_matches_reference(rtmlib, reflib, oracle, nsp):
    a = _model(23, 31, seed=nsp) ** 2
    ref = a.copy()
    reflib.ref_velsmooth1d(_p(ref), 23, 31, nsp)
    got = a.copy()
    assert rtmlib.lib().rtm_velsmooth(_p(got), 23, 31, nsp) == 0
    assert np.array_equal(got.view(np.int32), ref.view(np.int32))
    assert np.array_equal(oracle.velsmooth(a, nsp).view(np.int32), ref.view(np.int32))


def test_interp_and_get_constant_match_reference(rtmlib, reflib, oracle):
    nx0, nz0 = 21, 13
    v = _model(nz0, nx0, 5)
    for lx, lz in ((1, 1), (2, 2), (4, 2)):
        nx, nz = (nx0 - 1) * lx + 1, (nz0 - 1) * lz + 1
        ref = np.zeros((nz, nx), np.float32)
        reflib.ref_interpvel1(_p(v), _p(ref), nx0, nz0, nx, nz, lx, lz)
        got = np.zeros((nz, nx), np.float32)
        assert rtmlib.lib().rtm_interp_model(_p(v), _p(got), nx0, nz0, nx, nz, lx, lz) == 0
        assert np.array_equal(got, ref)
    # get_constant: one case that passes unchanged, one that regrids and one that re-times
    for fdom, dx0, dt0 in ((20.0, 10.0, 1e-3), (60.0, 10.0, 1e-3), (20.0, 10.0, 3e-3)):
        outs_ref = [np.zeros(1, t) for t in (np.float32, np.float32, np.int32, np.int32, np.int32, np.float32,
                                             np.int32, np.int32, np.float32, np.float32)]
        outs_got = [np.zeros_like(o) for o in outs_ref]
        outs_orc = [np.zeros_like(o) for o in outs_ref]
        reflib.ref_get_constant(_p(v), fdom, dx0, dx0, nx0, nz0, 1000, dt0, *[_p(o) for o in outs_ref])
        rtmlib.lib().rtm_get_constant(_p(v), fdom, dx0, dx0, nx0, nz0, 1000, dt0, *[_p(o) for o in outs_got])
        oracle.lib().orc_get_constant(_p(v), fdom, dx0, dx0, nx0, nz0, 1000, dt0, *[_p(o) for o in outs_orc])
        for a, b, c in zip(outs_ref, outs_got, outs_orc):
            assert a.tobytes() == b.tobytes() == c.tobytes()


def test_laplace_and_scale_match_reference(rtmlib, reflib, oracle):
    img = np.random.default_rng(9).standard_normal((31, 47)).astype(np.float32)
    for dx, dz in ((10, 10), (12, 7)):
        ref = img.copy()
        reflib.ref_laplacefd1d(47, 31, dx, dz, _p(ref))
        got = img.copy()
        rtmlib.lib().rtm_laplace_image(_p(got), 47, 31, dx, dz)
        orc = img.copy()
        oracle.lib().orc_laplacefd1d(47, 31, dx, dz, _p(orc))
        assert np.array_equal(got, ref) and np.array_equal(orc, ref)
    illum = np.abs(img) + 0.1
    ref = img.copy()
    reflib.ref_scaleimage1d(_p(illum), _p(ref), img.size)
    got = img.copy()
    rtmlib.lib().rtm_scale_image(_p(illum), _p(got), img.size)
    assert np.array_equal(got, ref)


LAYOUT_CASES = [
    dict(layout=2, nx=401, spx0=2000.0, dspx=25.0, offset=0.0, offsetmax=0.0),
    dict(layout=1, nx=3201, spx0=100.0, dspx=125.0, offset=0.0, offsetmax=4000.0),
    dict(layout=3, nx=300, spx0=40.0, dspx=37.5, offset=55.0, offsetmax=900.0),
    dict(layout=4, nx=300, spx0=40.0, dspx=37.5, offset=55.0, offsetmax=900.0),
    dict(layout=1, nx=96, spx0=200.0, dspx=550.0, offset=0.0, offsetmax=860.0),
]


@pytest.mark.parametrize("case", LAYOUT_CASES)
def test_geometry_matches_oracle(rtmlib, oracle, case):
    for ishot in (1, 2, 5, 13):
        sv = rtmlib.SurveyConfig(nx=case["nx"], nz=50, nt=700, dx=10.0, dz=10.0, dt=1e-3, npml=40,
                                 layout=case["layout"], spx0=case["spx0"], spz0=20.0, dspx=case["dspx"],
                                 offset=case["offset"], offsetmax=case["offsetmax"])
        try:
            g = rtmlib.geometry(sv, ishot)
        except rtmlib.RtmError:
            continue
        o = oracle.geometry(case["layout"], ishot, case["nx"], 50, 700, 10.0, 10.0, 1e-3, 40, case["spx0"], 20.0,
                            case["dspx"], case["offset"], case["offsetmax"])
        for k in ("nx1", "nx2", "nxlength", "noffset", "nsx", "nsz", "nxpad", "nzpad", "rx0", "nrec",
                  "iTraceAll", "iTrace", "Offset", "sx", "gx", "Ntrace"):
            assert getattr(g, k) == getattr(o, k), (k, ishot)
        assert (g.Nt, g.Dt) == (o.Nt, o.Dt) and g.Dx == o.Dx


def test_gather_su_bytes_match_reference(rtmlib, reflib, tmp_path):
    nt, ntr = 37, 11
    g = np.random.default_rng(1).standard_normal((nt, ntr)).astype(np.float32)
    geo = rtmlib.Geometry()
    geo.iTraceAll, geo.iTrace, geo.Offset, geo.sx, geo.gx = 101, 1, -480, 480, 0
    geo.Nt, geo.Dt, geo.Dx, geo.Ntrace = nt, 1000, 12.5, ntr
    for sgy in (0, 1):
        for endian in (0, 1):
            ours = str(tmp_path / f"o{sgy}{endian}.su")
            refp = str(tmp_path / f"r{sgy}{endian}.su")
            assert rtmlib.lib().rtm_write_gather_su(ours.encode(), _p(g), C.byref(geo), nt, sgy, endian) == 0
            reflib.ref_Outseisfile1d(_p(g), 101, 1, -480, 480, 0, nt, 1000, 12.5, ntr, 0, sgy, endian, refp.encode())
            assert open(ours, "rb").read() == open(refp, "rb").read()
            back = np.zeros((nt, ntr), np.float32)
            n1, n2 = C.c_int(), C.c_int()
            keys = rtmlib.Geometry()
            assert rtmlib.lib().rtm_read_gather_su(ours.encode(), sgy, _p(back), C.byref(n1), C.byref(n2),
                                                   C.byref(keys)) == 0
            assert (n1.value, n2.value) == (nt, ntr) and np.array_equal(back, g)
            assert (keys.iTraceAll, keys.Offset, keys.sx, keys.Dt) == (101, -480, 480, 1000)
            refback = np.zeros((nt, ntr), np.float32)
            rk = np.zeros(8, np.int32)
            rdx = np.zeros(1, np.float32)
            reflib.ref_Inseisfile1d(_p(refback), 0, sgy, ours.encode(), _p(rk), _p(rdx))
            assert np.array_equal(refback, g) and rk[0] == 101 and rk[7] == ntr


def test_image_su_bytes_match_reference(rtmlib, reflib, tmp_path):
    img = np.random.default_rng(2).standard_normal((29, 17)).astype(np.float32)
    for d in (10.0, 12.5, 5.0, 0.004):
        ours, refp = str(tmp_path / "o.su"), str(tmp_path / "r.su")
        rtmlib.lib().rtm_write_image_su(ours.encode(), _p(img), 29, 17, d)
        reflib.ref_Output1d(_p(img), 29, 17, d, refp.encode(), 1)
        assert open(ours, "rb").read() == open(refp, "rb").read(), d


def test_golden_su_headers_reproduced(rtmlib):
    """The reference's own gather files (written on the B200 run) are reproduced byte for
    byte from the shot geometry: header keys of every trace."""
    z, prm = load_case("caseB")
    for ishot in (1, 2):
        sv = rtmlib.SurveyConfig(nx=prm["nx"], nz=prm["nz"], nt=prm["nt"], dx=prm["dx"], dz=prm["dx"], dt=prm["dt"],
                                 npml=prm["npml"], layout=prm["layout"], spx0=prm["spx0"], spz0=prm["spz0"],
                                 dspx=prm["dspx"])
        g = rtmlib.geometry(sv, ishot)
        hdr = z[f"gather{ishot}_headers"]
        data = z[f"gather{ishot}"]
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "g.su")
            rtmlib.lib().rtm_write_gather_su(p.encode(), _p(np.ascontiguousarray(data)), C.byref(g), prm["nt"], 0, 0)
            raw = np.fromfile(p, np.uint8).reshape(g.Ntrace, 240 + 4 * prm["nt"])
        assert np.array_equal(raw[:, :240], hdr)


def test_read_params_and_velocity(rtmlib, tmp_path):
    inp = tmp_path / "input"
    inp.mkdir()
    (inp / "cmd.in").write_text("parameter file name\nparam.txt\n")
    vals = ["0.001 2000 0.1", "4000 2000 10 10", "20 1 0.1", "2000 20 25", "0 0", "1 1 1 1", "40",
            "0 0", "1.5 0", "0", "2", "0", "0", "0", "0", "0", "vel.su"]
    text = "".join(f"# comment {i}\n{v}\n" for i, v in enumerate(vals))
    (inp / "param.txt").write_text(text)
    P = rtmlib.Params()
    assert rtmlib.lib().rtm_read_params(str(inp).encode(), C.byref(P)) == 0
    assert (P.nt0, P.npml, P.flag_layout, P.nshot) == (2000, 40, 2, 1)
    assert abs(P.dt0 - 0.001) < 1e-9 and P.vp_file == b"vel.su" and abs(P.spz0 - 20) < 1e-6
    # velocity: nx traces of (240-byte header + nz floats)
    nx, nz = 5, 4
    v = np.arange(nx * nz, dtype=np.float32).reshape(nz, nx)
    with open(inp / "vel.su", "wb") as f:
        for ix in range(nx):
            f.write(b"\0" * 240)
            f.write(v[:, ix].tobytes())
    out = np.zeros((nz, nx), np.float32)
    assert rtmlib.lib().rtm_read_velocity(str(inp / "vel.su").encode(), nx, nz, _p(out)) == 0
    assert np.array_equal(out, v)
    assert rtmlib.lib().rtm_read_velocity(b"/nonexistent/v.su", nx, nz, _p(out)) == rtmlib.RTM_ERR_IO
    assert rtmlib.lib().rtm_read_params(str(tmp_path / "nowhere").encode(), C.byref(P)) == rtmlib.RTM_ERR_IO
    assert b"cmd.in" in rtmlib.lib().rtm_last_error()


def test_truncated_gather_is_rejected(rtmlib, tmp_path):
    p = tmp_path / "bad.su"
    p.write_bytes(b"\0" * 100)
    n1, n2 = C.c_int(), C.c_int()
    assert rtmlib.lib().rtm_read_gather_su(str(p).encode(), 0, None, C.byref(n1), C.byref(n2), None) == rtmlib.RTM_ERR_IO


def test_rtm_gpu_selfdoc():
    exe = os.path.join(ROOT, "gubingluo_b200", "rtm_gpu")
    if not os.path.exists(exe):
        pytest.skip("rtm_gpu not built")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=30)
    assert r.returncode == 0 and "parameter file" in r.stdout


def test_session_rejects_bad_surveys_without_gpu(rtmlib):
    """Argument errors are reported before any device work."""
    sv = rtmlib.SurveyConfig(nx=50, nz=40, nt=100, dx=10.0, dz=10.0, dt=1e-3, npml=5)
    v = np.full((40, 50), 2000, np.float32)
    with pytest.raises(rtmlib.RtmError, match="npml"):
        rtmlib.Session(sv, rtmlib.RunOptions(), [1], v, v)
    sv = rtmlib.SurveyConfig(nx=50, nz=40, nt=100, dx=10.0, dz=10.0, dt=1e-3, npml=20, layout=7)
    with pytest.raises(rtmlib.RtmError):
        rtmlib.geometry(sv, 1)


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++17")])
def test_header_compiles_and_links_from_c_and_cpp(rtmlib, tmp_path, lang, std):
    """The C-ABI header compiles warning-free as C99 and as C++17 (-pedantic -Werror), and a
    caller built from it links against librtm_b200.so and calls entries that need no GPU:
    the coefficient table (the reference's Liu-Yang table, FD_function.cpp:73-165) and a
    refused session (status code and message, no device touched)."""
    src = tmp_path / ("caller.c" if lang == "c" else "caller.cpp")
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "rtm_b200.h"
int main(void) {
    float c[100];
    rtm_coef_table(c);
    rtm_session *ss = 0;
    int rc = rtm_session_open(&ss, 0, 0, 0, 0, 0, 0, 0, 0, 0);
    printf("%s|%.9g|%.9g|%d|%s\n", rtm_version(), (double)c[0], (double)c[99], rc != 0 && ss == 0,
           rtm_last_error());
    return 0;
}
''')
    exe = tmp_path / "caller"
    libdir = os.path.dirname(rtmlib.LIB_PATH)
    cmd = ["gcc" if lang == "c" else "g++", "-x", lang, f"-std={std}", "-Wall", "-Wextra", "-Werror", "-pedantic",
           f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe), f"-L{libdir}", "-lrtm_b200",
           f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.strip().split("|")
    coef = rtmlib.coef_table()
    assert out[0] and np.float32(out[1]) == coef[0] and np.float32(out[2]) == coef[99]   # %.9g round-trips a float
    assert out[3] == "1" and "null" in out[4]
