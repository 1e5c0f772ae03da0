"""Seeded synthetic surveys for the benchmark configurations.

The reference ships no data; its benchmark configurations describe velocity models by recipe.
Each builder returns the true velocity, the migration velocity (the true model smoothed in
velocity), a constant density of 2000 kg/m^3 (the reference's default without a density file,
RTM_GPU_velstr.cpp:148) and the survey parameters.  Random fields use numpy PCG64 with seed
20260000 + config number (faults / salt: 20260100 + config number; per-shot apertures:
20260200 + config number).
"""
from __future__ import annotations

import math

import numpy as np

from . import SurveyConfig, geometry


def _gaussian_smooth(a: np.ndarray, sigma_z: float, sigma_x: float) -> np.ndarray:
    """Separable Gaussian smoothing (sigma in cells) with edge replication."""
    out = a.astype(np.float64)
    for axis, sig in ((0, sigma_z), (1, sigma_x)):
        if sig <= 0:
            continue
        r = int(math.ceil(3 * sig))
        k = np.exp(-0.5 * (np.arange(-r, r + 1) / sig) ** 2)
        k /= k.sum()
        pad = [(0, 0), (0, 0)]
        pad[axis] = (r, r)
        e = np.pad(out, pad, mode="edge")
        acc = np.zeros_like(out)
        for i, w in enumerate(k):
            sl = [slice(None), slice(None)]
            sl[axis] = slice(i, i + out.shape[axis])
            acc += w * e[tuple(sl)]
        out = acc
    return out


def gaussian_random_field(nz, nx, dz, dx, sigma, corr_z, corr_x, rng) -> np.ndarray:
    """FFT-filtered white noise with an anisotropic Gaussian spectrum, rescaled to std sigma."""
    w = rng.standard_normal((nz, nx))
    kz = np.fft.fftfreq(nz, d=dz)[:, None]
    kx = np.fft.fftfreq(nx, d=dx)[None, :]
    spec = np.exp(-((math.pi * kz * corr_z) ** 2 + (math.pi * kx * corr_x) ** 2))
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * spec))
    f -= f.mean()
    s = f.std()
    return f * (sigma / s) if s > 0 else f


def _thrust_faults(v: np.ndarray, dz: float, dx: float, throw_m: float, nfaults: int, rng) -> np.ndarray:
    """Planar dipping thrust faults: the hanging wall (above each fault plane) is lifted by
    throw_m, i.e. it takes the layering from throw_m deeper."""
    nz, nx = v.shape
    shift = int(round(throw_m / dz))
    out = v.copy()
    for _ in range(nfaults):
        x0 = rng.uniform(0.15, 0.85) * nx * dx
        dip = math.radians(rng.uniform(25.0, 40.0))
        sgn = rng.choice([-1.0, 1.0])
        zz = np.arange(nz)[:, None] * dz
        xx = np.arange(nx)[None, :] * dx
        hanging = zz < sgn * (xx - x0) * math.tan(dip)
        src = np.vstack([out[shift:], np.repeat(out[-1:], shift, axis=0)])
        out = np.where(hanging, src, out)
    return out


def config(n: int, nshots: int | None = None, nt: int | None = None):
    """Survey n (1..5) of the benchmark configurations.  Returns
    (SurveyConfig, shots, vp_true, vp_mig, rho, meta)."""
    rng = np.random.default_rng(20260000 + n)
    frng = np.random.default_rng(20260100 + n)
    if n == 1:
        nx, nz, d, npml, fdom, dt, NT = 401, 201, 10.0, 40, 20.0, 1e-3, 2000
        zz = np.arange(nz)[:, None] * d
        xx = np.arange(nx)[None, :] * d
        v = np.where(zz < 500, 1500.0, np.where(zz < 1000, 2000.0, np.where(zz < 1500, 2500.0, 3000.0)))
        v = np.where(zz >= 1700 + xx * math.tan(math.radians(10.0)), 3500.0, v) + 0 * xx
        smooth_m = 150.0
        shots = [1]
        s = SurveyConfig(nx=nx, nz=nz, nt=NT, dx=d, dz=d, dt=dt, npml=npml, fdom=fdom, layout=2,
                         spx0=2000.0, spz0=20.0, dspx=0.0, receiver_depth=2)
    elif n in (2, 3):
        if n == 2:
            nx, nz, d, npml, fdom, dt, NT, ns = 1701, 351, 12.5, 50, 15.0, 1e-3, 4000, 64
        else:
            nx, nz, d, npml, fdom, dt, NT, ns = 4001, 1201, 5.0, 60, 25.0, 4e-4, 10000, 16
        zz = np.arange(nz)[:, None] * d
        v = 1500.0 + 0.6 * zz + gaussian_random_field(nz, nx, d, d, 150.0, 60.0, 200.0, rng)
        v = _thrust_faults(v, d, d, 150.0, 3, frng)
        smooth_m = 250.0
        if n == 2:   # sources every 25 grid points from column 50, at z = 12.5 m
            s = SurveyConfig(nx=nx, nz=nz, nt=NT, dx=d, dz=d, dt=dt, npml=npml, fdom=fdom, layout=2,
                             spx0=50 * d, spz0=d, dspx=25 * d, receiver_depth=1)
        else:        # 16 shots evenly spaced across the model
            step = (nx - 1) * d / ns
            s = SurveyConfig(nx=nx, nz=nz, nt=NT, dx=d, dz=d, dt=dt, npml=npml, fdom=fdom, layout=2,
                             spx0=step / 2, spz0=4 * d, dspx=step, receiver_depth=4)
        shots = list(range(1, ns + 1))
    elif n == 4:
        nx, nz, d, npml, fdom, dt, NT, ns = 3201, 801, 10.0, 40, 20.0, 8e-4, 5000, 256
        zz = np.arange(nz)[:, None] * d
        v = 1500.0 + 0.6 * zz + gaussian_random_field(nz, nx, d, d, 150.0, 60.0, 200.0, rng)
        smooth_m = 250.0
        # each shot's aperture drawn uniformly from 2-8 km (201-801 columns, centred on its
        # source; cut at the model's edges): meta["apertures"] maps shot number -> columns,
        # for shot_geometries.  The survey's offsetmax is the widest.
        step = (nx - 1) * d / ns
        s = SurveyConfig(nx=nx, nz=nz, nt=NT, dx=d, dz=d, dt=dt, npml=npml, fdom=fdom, layout=1,
                         spx0=step / 2, spz0=2 * d, dspx=step, offsetmax=8000.0, receiver_depth=2)
        shots = list(range(1, ns + 1))
        half = np.random.default_rng(20260200 + n).integers(100, 401, size=ns)
        apertures = {ishot: int(2 * h + 1) for ishot, h in zip(shots, half)}
    elif n == 5:
        nx, nz, d, npml, fdom, dt, NT, ns = 2401, 1001, 7.5, 80, 18.0, 5e-4, 8000, 128
        zz = np.arange(nz)[:, None] * d
        v = 1500.0 + 0.5 * zz + 0.0 * np.arange(nx)[None, :]
        g = gaussian_random_field(nz, nx, d, d, 1.0, 400.0, 800.0, frng)
        salt = (g > 1.0) & (zz >= 1200.0) & (zz <= 3500.0)
        v = np.where(salt, 4500.0, v)
        v = np.where(zz < 300.0, 1500.0, v)
        smooth_m = 150.0
        step = (nx - 1) * d / ns
        s = SurveyConfig(nx=nx, nz=nz, nt=NT, dx=d, dz=d, dt=dt, npml=npml, fdom=fdom, layout=2,
                         spx0=step / 2, spz0=2 * d, dspx=step, receiver_depth=2)
        shots = list(range(1, ns + 1))
    else:
        raise ValueError("configs are 1..5")
    v = np.clip(v, 1500.0, 5000.0).astype(np.float32)
    sig = smooth_m / d
    vm = _gaussian_smooth(v, sig, sig).astype(np.float32)
    rho = np.full_like(v, 2000.0)
    s.alp = float(np.float32(1.0 / d))   # Gaussian source of about one cell
    s.direct, s.direct0 = 1.5, 0.0
    if nt is not None:
        s.nt = nt
    meta = dict(config=n, smooth_m=smooth_m)
    if n == 4:
        meta["apertures"] = apertures
    if nshots is not None:
        shots = shots[:nshots]
    s.dt = float(np.float32(s.dt))
    return s, shots, v, vm, rho, meta


def shot_geometries(survey: SurveyConfig, shots, meta):
    """Per-shot geometry of a survey whose apertures differ shot by shot (meta["apertures"]:
    shot number -> columns, layout 1): the reference's layout-1 window of each shot
    (rtm_model.cu:122-154) with offsetmax set to its own aperture.  None when every shot
    follows the survey's own layout."""
    if "apertures" not in meta:
        return None
    if survey.layout != 1:
        raise ValueError("per-shot apertures need layout 1")
    out = []
    for ishot in shots:
        w = meta["apertures"][int(ishot)]
        sk = SurveyConfig(**{**survey.__dict__, "offsetmax": (w - 1) * survey.dx})
        out.append(geometry(sk, int(ishot)))
    return out


def write_shot_file(path: str, shots, nt0: int, dt0: float, dx0: float, sgyflag: int = 0,
                    big_endian: bool = False, first_trace: int = 1) -> None:
    """Writes a multi-shot SU (sgyflag 0) or SEG-Y (sgyflag 1: a zeroed 3600-byte volume
    header first) file of the layout the real-data driver reads (rtm_real.cu:379-394,
    sgyhead.h:92-103): per trace a 240-byte header, then nt0 IEEE floats.  Header keys
    written (byte offset): tracl 0, tracf 12, offset 36, sx 72, gx 80 (int32), ns 114, dt 116
    (int16, microseconds), d2 188 (float), ntr 208 (int32); the rest zero.  ``shots`` is a list
    of (sx, offset, gather[nt0][ntrace]) with receivers offset, offset+dx0, ... to the right
    of the source, as that driver assumes."""
    e = ">" if big_endian else "<"
    hdr = np.dtype([("tracl", e + "i4"), ("p0", "V8"), ("tracf", e + "i4"), ("p1", "V20"), ("offset", e + "i4"),
                    ("p2", "V32"), ("sx", e + "i4"), ("p3", "V4"), ("gx", e + "i4"), ("p4", "V30"),
                    ("ns", e + "i2"), ("dt", e + "i2"), ("p5", "V70"), ("d2", e + "f4"), ("p6", "V16"),
                    ("ntr", e + "i4"), ("p7", "V28")])
    assert hdr.itemsize == 240
    with open(path, "wb") as f:
        if sgyflag:
            f.write(bytes(3600))
        itr = first_trace
        for sx, offset, g in shots:
            g = np.asarray(g, np.float32)
            assert g.shape[0] == nt0
            for ix in range(g.shape[1]):
                h = np.zeros(1, hdr)
                h["tracl"] = itr
                h["tracf"] = ix + 1
                h["offset"] = int(offset + ix * dx0)
                h["sx"] = int(sx)
                h["gx"] = int(sx + offset + ix * dx0)
                h["ns"] = nt0
                h["dt"] = int(round(dt0 * 1e6))
                h["d2"] = dx0
                h["ntr"] = g.shape[1]
                f.write(h.tobytes())
                f.write(np.ascontiguousarray(g[:, ix]).astype(e + "f4").tobytes())
                itr += 1
