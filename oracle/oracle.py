"""Python driver of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/liboracle.so`` (the C restatement in rtm_oracle.c) and restates the
reference's shot loop (gubingluo rtm_model.cu:117-488) on top of it: per-shot geometry,
model window + square + padding (+ optional PML smoothing), one ``orc_shot`` per shot and
the per-shot stacking.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline use this module; the product never imports it.

``load_reference_host()`` loads ``oracle/_ref/libref_host.so``: the reference's own host
C++ compiled from its sources (oracle/ref/Makefile), used to pin the restatement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_HOST = os.path.join(HERE, "_ref", "libref_host.so")
# The reference checkout: $RTM_REFERENCE_DIR, else a directory named "reference" beside this
# repository's root.
REFERENCE_DIR = os.environ.get("RTM_REFERENCE_DIR") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))

_vp = C.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class OrcShot(C.Structure):
    _fields_ = [("X", C.c_int), ("Z", C.c_int), ("npml", C.c_int), ("nt", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
                ("nsx", C.c_int), ("nsz", C.c_int), ("amp", C.c_float), ("alp", C.c_float),
                ("fdom", C.c_float), ("rz", C.c_int), ("rx0", C.c_int), ("nrec", C.c_int),
                ("vpmax", C.c_float)]


class OrcGeom(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("nx1", "nx2", "nxlength", "noffset", "nsx", "nsz", "nxpad",
                                        "nzpad", "rx0", "nrec", "iTraceAll", "iTrace", "Offset", "sx",
                                        "gx")]
                + [("Nt", C.c_ushort), ("Dt", C.c_ushort), ("Dx", C.c_float), ("Ntrace", C.c_int)])


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        for name in ("orc_shot_f32", "orc_shot_f64"):
            getattr(L, name).argtypes = [C.POINTER(OrcShot)] + [_vp] * 6 + [C.c_int, _vp, C.c_int, C.c_int,
                                                                             C.c_int] + [_vp] * 4
        for name in ("orc_shot_ex_f32", "orc_shot_ex_f64"):
            getattr(L, name).argtypes = [C.POINTER(OrcShot)] + [_vp] * 6 + [C.c_int, _vp, C.c_int, C.c_int,
                                                                             C.c_int] + [_vp] * 4 + [C.c_int] + [_vp] * 4
        for name in ("orc_finalize_extra_f32", "orc_finalize_extra_f64"):
            getattr(L, name).argtypes = [_vp] * 5 + [C.c_int] * 4 + [_vp] * 7
        for name in ("orc_forward_f32", "orc_forward_f64"):
            getattr(L, name).argtypes = [C.POINTER(OrcShot), _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp]
        L.orc_finalize_f32.argtypes = [_vp, _vp] + [C.c_int] * 4 + [_vp] * 3
        L.orc_finalize_f64.argtypes = [_vp, _vp] + [C.c_int] * 4 + [_vp] * 3
        L.orc_geometry.argtypes = [C.POINTER(OrcGeom)] + [C.c_int] * 5 + [C.c_float] * 3 + [C.c_int] + [C.c_float] * 5
        L.orc_coef_table.argtypes = [_vp]
        L.orc_ricker_device.argtypes = [_vp, C.c_float, C.c_float, C.c_int]
        L.orc_ricker_host.argtypes = [_vp, C.c_float, C.c_int, C.c_float]
        L.orc_pml_profiles.argtypes = [_vp] * 4 + [C.c_float] * 3 + [C.c_int] * 3
        L.orc_norder.argtypes = [_vp] * 3 + [C.c_int] * 2
        L.orc_source.argtypes = [_vp] + [C.c_int] * 4 + [C.c_float] * 4
        L.orc_interp_gather.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_int]
        L.orc_fk_interp.argtypes = [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_mute.argtypes = [_vp, _vp] + [C.c_int] * 9 + [C.c_float] * 3
        L.orc_taper.argtypes = [_vp, C.c_int, C.c_int, C.c_float]
        L.orc_taper_nwin.argtypes = [C.c_int]
        L.orc_extractvel1.argtypes = [_vp, _vp] + [C.c_int] * 5
        L.orc_extendvel1.argtypes = [_vp, _vp] + [C.c_int] * 3
        L.orc_pmlvelsmooth1d.argtypes = [_vp] + [C.c_int] * 3
        L.orc_velsmooth1d.argtypes = [_vp] + [C.c_int] * 3
        L.orc_interpvel1.argtypes = [_vp, _vp] + [C.c_int] * 6
        L.orc_laplacefd1d.argtypes = [C.c_int] * 4 + [_vp]
        L.orc_scaleimage1d.argtypes = [_vp, _vp, C.c_int]
        L.orc_get_constant.argtypes = [_vp, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                       C.c_float] + [_vp] * 10
        _lib = L
    return _lib


def num_threads():
    return lib().orc_num_threads()


def coef_table():
    c = np.zeros(100, np.float32)
    lib().orc_coef_table(_p(c))
    return c


def geometry(layout, ishot, nx, nz, nt, dx, dz, dt, npml, spx0, spz0, dspx, offset=0.0, offsetmax=0.0):
    g = OrcGeom()
    rc = lib().orc_geometry(C.byref(g), layout, ishot, nx, nz, nt, dx, dz, dt, npml, spx0, spz0, dspx,
                            offset, offsetmax)
    if rc:
        raise ValueError("bad layout")
    return g


def pad_model(v, nx1, nx2, npml, square, medium_flag=0):
    """extractvel1/extractrho1 + extendvel1 (+ pmlvelsmooth1d)."""
    v = f32(v)
    nz, nx = v.shape
    nxl = nx2 - nx1 + 1
    tmp = np.zeros((nz, nxl), np.float32)
    lib().orc_extractvel1(_p(tmp), _p(v), nx, nz, nx1, nx2, int(square))
    pad = np.zeros((nz + 2 * npml, nxl + 2 * npml), np.float32)
    lib().orc_extendvel1(_p(pad), _p(tmp), nxl, nz, npml)
    if medium_flag:
        lib().orc_pmlvelsmooth1d(_p(pad), pad.shape[1], pad.shape[0], npml)
    return pad


def velsmooth(a, nsp):
    a = f32(a).copy()
    lib().orc_velsmooth1d(_p(a), a.shape[0], a.shape[1], nsp)
    return a


def pml_profiles(vpmax, dx, dz, npml, X, Z):
    out = [np.zeros(n, np.float32) for n in (X, Z, X - 1, Z - 1)]
    lib().orc_pml_profiles(*[_p(a) for a in out], vpmax, dx, dz, npml, X, Z)
    return out


def norder(X, Z):
    n = np.zeros((Z, X), np.int32)
    nx_ = np.zeros(X - 1, np.int32)
    nz_ = np.zeros(Z - 1, np.int32)
    lib().orc_norder(_p(n), _p(nx_), _p(nz_), X, Z)
    return n, nx_, nz_


def shot_struct(X, Z, npml, nt, dx, dz, dt, nsx, nsz, amp, alp, fdom, rz, rx0, nrec, vpmax):
    s = OrcShot()
    for k, v in dict(X=X, Z=Z, npml=npml, nt=nt, dx=dx, dz=dz, dt=dt, nsx=nsx, nsz=nsz, amp=amp,
                     alp=alp, fdom=fdom, rz=rz, rx0=rx0, nrec=nrec, vpmax=vpmax).items():
        setattr(s, k, v)
    return s


def forward(shot: OrcShot, vp2, rho, nsteps, precision="f32", coef=None, wavelet=None):
    """nsteps forward steps from rest -> (p, vx, vz, gather)."""
    dt = np.float32 if precision == "f32" else np.float64
    X, Z = shot.X, shot.Z
    p = np.zeros((Z, X), dt)
    vx = np.zeros((Z, X - 1), dt)
    vz = np.zeros((Z - 1, X), dt)
    g = np.zeros((nsteps, shot.nrec), dt)
    coef = coef_table() if coef is None else f32(coef)
    fn = lib().orc_forward_f32 if precision == "f32" else lib().orc_forward_f64
    fn(C.byref(shot), _p(f32(vp2)), _p(f32(rho)), _p(coef), _p(None if wavelet is None else f32(wavelet)),
       nsteps, _p(p), _p(vx), _p(vz), _p(g))
    return p, vx, vz, g


def shot(shot: OrcShot, vp2f, rhof, vp2b=None, rhob=None, mode=1, gather=None, mute=1, nw=0,
         tlength=0, precision="f32", coef=None, wavelet=None, want_fields=False, extra=0):
    """One shot of RTM (source pass, backward loop, imaging); returns dict with g1, illum,
    gather (modelled in mode 0) and optionally the final ps/p wavefields.  extra = 1 or 2
    adds the decomposition, Poynting and energy-norm images g2, g3, g3t, g4 (2: with the
    reference's indexing of vx and vz)."""
    dt = np.float32 if precision == "f32" else np.float64
    nzi, nxi = shot.Z - 2 * shot.npml, shot.X - 2 * shot.npml
    g1 = np.zeros((nzi, nxi), dt)
    il = np.zeros((nzi, nxi), dt)
    ps = np.zeros((shot.Z, shot.X), dt) if want_fields else None
    pr = np.zeros((shot.Z, shot.X), dt) if want_fields else None
    if gather is None:
        gather = np.zeros((shot.nt, shot.nrec), np.float32)
    else:
        gather = f32(gather).copy()
    coef = coef_table() if coef is None else f32(coef)
    vp2f, rhof = f32(vp2f), f32(rhof)
    vp2b = vp2f if vp2b is None else f32(vp2b)
    rhob = rhof if rhob is None else f32(rhob)
    ex = [np.zeros((nzi, nxi), dt) for _ in range(4)] if extra else [None] * 4
    fn = lib().orc_shot_ex_f32 if precision == "f32" else lib().orc_shot_ex_f64
    rc = fn(C.byref(shot), _p(vp2f), _p(rhof), _p(vp2b), _p(rhob), _p(coef),
            _p(None if wavelet is None else f32(wavelet)), mode, _p(gather), mute, nw, tlength,
            _p(g1), _p(il), _p(ps), _p(pr), extra, *[_p(a) for a in ex])
    if rc:
        raise MemoryError("oracle allocation failed")
    return dict(g1=g1, illum=il, gather=gather, ps=ps, p=pr, g2=ex[0], g3=ex[1], g3t=ex[2], g4=ex[3])


def _migrate_shot(s, g, vp, rho, vp_mig, rho_mig, mode, gather, mute, nw, tlength, precision, keep_fields,
                  extra, images, fields, out_gathers):
    """One shot of the reference's shot loop for geometry ``g``: model window + padding
    (+ PML smoothing), migration model (+ smoothing), the shot, then the per-shot stacking
    into ``images`` (rtm_model.cu:150-488, rtm_real.cu:196-468)."""
    nx, nz = s["nx"], s["nz"]
    vp2f = pad_model(vp, g.nx1, g.nx2, s["npml"], True, s.get("medium_flag", 0))
    rhof = pad_model(rho, g.nx1, g.nx2, s["npml"], False, s.get("medium_flag", 0))
    if vp_mig is not None or s.get("ismth", 0) > 0:
        vb = vp_mig if vp_mig is not None else vp
        rb = rho_mig if rho_mig is not None else rho
        vp2b = pad_model(vb, g.nx1, g.nx2, s["npml"], True, s.get("medium_flag", 0))
        rhob = pad_model(rb, g.nx1, g.nx2, s["npml"], False, s.get("medium_flag", 0))
        if s.get("ismth", 0) > 0:
            vp2b = velsmooth(vp2b, s["ismth"])
            rhob = velsmooth(rhob, s["ismth"])
    else:
        vp2b, rhob = vp2f, rhof
    vpmax = float(np.sqrt(np.float32(vp2f.max()), dtype=np.float32))
    rz = s["npml"] + s.get("receiver_depth", 0)
    sh = shot_struct(g.nxpad, g.nzpad, s["npml"], s["nt"], s["dx"], s["dz"], s["dt"], g.nsx, g.nsz,
                     s["amp"], s["alp"], s["fdom"], rz, g.rx0, g.nrec, vpmax)
    r = shot(sh, vp2f, rhof, vp2b, rhob, mode=mode, gather=gather, mute=mute, nw=nw, tlength=tlength,
             precision=precision, want_fields=keep_fields, extra=extra)
    out_gathers.append(r["gather"])
    if keep_fields:
        fields.append((r["ps"], r["p"]))
    fin = lib().orc_finalize_f32 if precision == "f32" else lib().orc_finalize_f64
    fin(_p(r["g1"]), _p(r["illum"]), g.nxlength, nz, nx, g.nx1, _p(images["image1"]), _p(images["image2s"]),
        _p(images["illum"]))
    if extra:   # after fin, which tapered r["illum"] in place
        fx = lib().orc_finalize_extra_f32 if precision == "f32" else lib().orc_finalize_extra_f64
        fx(_p(r["g2"]), _p(r["g3"]), _p(r["g4"]), _p(r["g3t"]), _p(r["illum"]), g.nxlength, nz, nx, g.nx1,
           *[_p(images[k]) for k in XNAMES])


XNAMES = ("image3s", "image4s", "image5s", "image3m", "image4m", "image5m", "imagetrue")


def _new_images(nz, nx, precision, extra):
    acc = np.float32 if precision == "f32" else np.float64
    names = ("image1", "image2s", "illum") + (XNAMES if extra else ())
    return {k: np.zeros((nz, nx), acc) for k in names}


def _mute_lengths(s):
    nw = int(np.float32(s["direct"]) / (np.float32(s["fdom"]) * np.float32(s["dt"])))
    tlength = int(np.float32(s["direct0"]) / np.float32(s["dt"]))
    return nw, tlength


def rtm_model(survey: dict, shots, vp, rho, vp_mig=None, rho_mig=None, gathers=None,
              precision="f32", keep_fields=False, extra=0):
    """Restatement of the reference's rtm_model shot loop for one layout (mode 0 models each
    gather in (vp, rho) first; mode 1 migrates ``gathers``).  ``survey`` keys: nx nz nt dx dz
    dt npml fdom amp alp layout spx0 spz0 dspx offset offsetmax mode medium_flag ismth direct
    direct0 mute receiver_depth.  Returns stacked images (+ gathers); with extra = 1 or 2
    also image3s, image4s, image5s, image3m, image4m, image5m and imagetrue."""
    s = survey
    nx, nz = s["nx"], s["nz"]
    images = _new_images(nz, nx, precision, extra)
    out_gathers, fields = [], []
    nw, tlength = _mute_lengths(s)
    for k, ishot in enumerate(shots):
        g = geometry(s["layout"], ishot, nx, nz, s["nt"], s["dx"], s["dz"], s["dt"], s["npml"],
                     s["spx0"], s["spz0"], s["dspx"], s.get("offset", 0.0), s.get("offsetmax", 0.0))
        _migrate_shot(s, g, vp, rho, vp_mig, rho_mig, s["mode"], None if s["mode"] == 0 else gathers[k],
                      s.get("mute", 1), nw, tlength, precision, keep_fields, extra, images, fields, out_gathers)
    return dict(image2m=images["image1"].copy(), gathers=out_gathers, fields=fields, **images)


# ---- the real-data path (rtm_real.cu) ----
class RealGeom:
    """Shot window of one recorded shot; the attributes of OrcGeom that the shot loop uses."""


def real_geometry(s: dict, sx: int, offset: int, ntrace: int, dx0: float):
    """rtm_real.cu:134-157 in the reference's float arithmetic: the spread runs from the
    source to offsetmax = offset + (ntrace-1)*dx0 on its right.  Returns (geometry, ncols0),
    ncols0 = the spread's width on the data grid."""
    f = np.float32
    dx, dz, npml = f(s["dx"]), f(s["dz"]), s["npml"]
    dx0 = f(dx0)
    offsetmax = f(f(offset) + f(ntrace - 1) * dx0)
    off, spx = f(offset), f(sx)
    noffset0 = int(off / dx0)
    nx10 = int(spx / dx0)
    nx20 = int(f(spx + offsetmax) / dx0)
    g = RealGeom()
    g.noffset = int(off / dx)
    g.nx1 = int(spx / dx)
    g.nx2 = int(f(spx + offsetmax) / dx)
    g.nxlength = g.nx2 - g.nx1 + 1
    spx = f(spx - f(g.nx1) * dx)
    spx = f(spx + f(npml) * dx)
    spz = f(f(s["spz0"]) + f(npml) * dz)
    g.nxpad = g.nxlength + 2 * npml
    g.nzpad = s["nz"] + 2 * npml
    g.nsx = int(spx / dx)
    g.nsz = int(spz / dz)
    g.rx0 = npml + g.noffset
    g.nrec = g.nxlength - g.noffset
    return g, nx20 - nx10 + 1 - noffset0


def read_traces(path, sgyflag, endianflag, nt0, itrace_all, ntrace, ncols):
    """The trace loop of rtm_real.cu:379-394 with numpy: [nt0][ncols], unread columns zero."""
    dt = np.dtype(">f4" if endianflag else "<f4")
    tb = 240 + 4 * nt0
    raw = np.fromfile(path, dtype=np.uint8)
    out = np.zeros((nt0, ncols), np.float32)
    first = (itrace_all - 1) * tb + 3600 * (1 if sgyflag else 0)
    for ix in range(min(ntrace, ncols)):
        o = first + ix * tb + 240
        out[:, ix] = np.frombuffer(raw[o:o + 4 * nt0].tobytes(), dt)
    return out


def interp_gather(seisobs, nx, nt, dt, dt0, mirror=0):
    """Interpseis2d (orc_interp.c): seisobs [nt0][nx0] -> [nt][nx]."""
    obs = f32(seisobs)
    nt0, nx0 = obs.shape
    out = np.zeros((nt, nx), np.float32)
    rc = lib().orc_interp_gather(_p(obs), nx0, nt0, _p(out), nx, nt, dt, dt0, mirror)
    if rc:
        raise ValueError(f"orc_interp_gather failed ({rc})")
    return out


def fk_interp(seisin, nx, lx, mirror=0):
    """GeneralFKinterp (orc_interp.c): seisin [nt0][nx0] -> [nt0][nx]."""
    a = f32(seisin)
    nt0, nx0 = a.shape
    out = np.zeros((nt0, nx), np.float32)
    rc = lib().orc_fk_interp(_p(a), _p(out), nx, nx0, nt0, lx, mirror)
    if rc:
        raise ValueError(f"orc_fk_interp failed ({rc})")
    return out


def rtm_real(survey: dict, path: str, profile, shots, vp, rho, nt0, dt0, dx0, sgyflag=0, endianflag=0,
             precision="f32", extra=0, mirror=0):
    """Restatement of the reference's rtm_real shot loop (rtm_real.cu:130-468): per shot
    (1-based numbers into ``profile`` = [sx, ntrace, first trace, offset] rows) the geometry,
    the recorded traces, Interpseis2d onto the model grid, the direct-wave mute in the
    migration model (the reference mutes after smoothing) and the migration.  ``survey``
    keys as for rtm_model (layout, spx0, dspx, offset, offsetmax unused)."""
    s = dict(survey)
    nx, nz = s["nx"], s["nz"]
    images = _new_images(nz, nx, precision, extra)
    out_gathers, fields = [], []
    nw, tlength = _mute_lengths(s)
    prof = np.asarray(profile)
    for ishot in shots:
        sx, ntrace, itr, off = (int(prof[r][ishot - 1]) for r in range(4))
        g, ncols0 = real_geometry(s, sx, off, ntrace, dx0)
        obs = read_traces(path, sgyflag, endianflag, nt0, itr, ntrace, ncols0)
        gather = interp_gather(obs, g.nrec, s["nt"], s["dt"], dt0, mirror)
        _migrate_shot(s, g, vp, rho, None, None, 1, gather, 2 if s.get("mute", 1) else 0, nw, tlength, precision,
                      False, extra, images, fields, out_gathers)
    return dict(image2m=images["image1"].copy(), gathers=out_gathers, **images)


# ---- the reference's own host code (compiled from its sources) ----
_ref = None


def build_reference_host():
    if not os.path.isdir(REFERENCE_DIR):
        return False
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), "host", f"REF={REFERENCE_DIR}"], check=True)
    return os.path.exists(REF_HOST)


def load_reference_host():
    """The reference's host C++ (libref_host.so) or None when it cannot be built here."""
    global _ref
    if _ref is not None:
        return _ref
    if not os.path.exists(REF_HOST) and not build_reference_host():
        return None
    L = C.CDLL(REF_HOST)
    L.ref_Diff_coeffVelStrLiuyang.argtypes = [_vp, C.c_int]
    L.ref_Ricker.argtypes = [_vp, C.c_float, C.c_int, C.c_float, C.c_int]
    L.ref_pmlvelsmooth1d.argtypes = [_vp] + [C.c_int] * 3
    L.ref_velsmooth1d.argtypes = [_vp] + [C.c_int] * 3
    L.ref_interpvel1.argtypes = [_vp, _vp] + [C.c_int] * 6
    L.ref_extendvel1.argtypes = [_vp, _vp] + [C.c_int] * 3
    L.ref_extractvel1.argtypes = [_vp, _vp] + [C.c_int] * 4
    L.ref_extractrho1.argtypes = [_vp, _vp] + [C.c_int] * 4
    L.ref_laplacefd1d.argtypes = [C.c_int] * 4 + [_vp]
    L.ref_scaleimage1d.argtypes = [_vp, _vp, C.c_int]
    L.ref_Maxval1.argtypes = [_vp, C.c_int]
    L.ref_Maxval1.restype = C.c_float
    L.ref_get_constant.argtypes = [_vp, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                   C.c_float] + [_vp] * 10
    L.ref_Output1d.argtypes = [_vp, C.c_int, C.c_int, C.c_float, C.c_char_p, C.c_int]
    L.ref_ReadVelMod.argtypes = [C.c_char_p, C.c_int, C.c_int, _vp]
    L.ref_Outseisfile1d.argtypes = ([_vp] + [C.c_int] * 7 + [C.c_float] + [C.c_int] * 4 + [C.c_char_p])
    L.ref_Inseisfile1d.argtypes = [_vp, C.c_int, C.c_int, C.c_char_p, _vp, _vp]
    L.ref_get_parameter.argtypes = [C.c_char_p, C.c_int, _vp, _vp, _vp, _vp]
    _ref = L
    return L
