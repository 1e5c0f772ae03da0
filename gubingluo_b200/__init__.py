"""gubingluo_b200 — B200 (sm_100a) implementation of the gubingluo 2D acoustic prestack RTM
hot path, driven through the C-ABI of ``librtm_b200.so`` (declared in ``include/rtm_b200.h``).

This module is a thin ctypes binding: every computation runs in the CUDA library.  If the
library has not been built, importing the binding raises ``RuntimeError``; there is no CPU
fallback.

Reference interfaces mirrored (gubingluo/gubingluo): ``rtm_model`` (RTM_GPU_velstr.cpp:23-28,
rtm_model.cu:12-17), the parameter file (RTM_GPU_velstr.cpp:60-120) and the SU/SEG-Y files
(IO_function.cpp, sgyhead_function.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librtm_b200.so")

RTM_OK, RTM_ERR_ARG, RTM_ERR_CUDA, RTM_ERR_IO, RTM_ERR_NOMEM, RTM_ERR_NUMERIC = 0, -1, -2, -3, -4, -5
PREC = {"fp32": 0, "fp16": 1, "bf16": 2}

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class Survey(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("nt", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
                ("npml", C.c_int), ("fdom", C.c_float), ("amp", C.c_float), ("alp", C.c_float),
                ("layout", C.c_int), ("spx0", C.c_float), ("spz0", C.c_float), ("dspx", C.c_float),
                ("offset", C.c_float), ("offsetmax", C.c_float), ("mode", C.c_int),
                ("medium_flag", C.c_int), ("ismth", C.c_int), ("direct", C.c_float),
                ("direct0", C.c_float), ("mute", C.c_int), ("receiver_depth", C.c_int)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("strip_precision", C.c_int), ("gather_precision", C.c_int),
                ("accum_fp64", C.c_int), ("batch", C.c_int), ("use_graph", C.c_int),
                ("verbose", C.c_int), ("extra_images", C.c_int), ("tsnap", C.c_float)]


class Geometry(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nx1", "nx2", "nxlength", "noffset", "nsx", "nsz", "nxpad",
                                       "nzpad", "rz", "rx0", "nrec", "iTraceAll", "iTrace",
                                       "Offset", "sx", "gx", "Nt", "Dt", "Ntrace")] + [("Dx", C.c_float)]


class BatchDesc(C.Structure):
    _fields_ = [("survey", Survey), ("options", Options), ("shots", C.POINTER(C.c_int)), ("nshots", C.c_int),
                ("vp", C.c_void_p), ("rho", C.c_void_p), ("vp_mig", C.c_void_p), ("rho_mig", C.c_void_p),
                ("gathers_in", C.POINTER(C.c_void_p)), ("gathers_out", C.POINTER(C.c_void_p)),
                ("image1", C.c_void_p), ("image2s", C.c_void_p), ("image2m", C.c_void_p), ("illum", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("seconds_total", C.c_double), ("gcell_updates", C.c_double), ("shots", C.c_int),
                ("batches", C.c_int), ("kernel_launches", C.c_int)]


class Params(C.Structure):
    _fields_ = ([("dt0", C.c_float), ("nt0", C.c_int), ("tsnap", C.c_float), ("xmax", C.c_float),
                 ("zmax", C.c_float), ("dx0", C.c_float), ("dz0", C.c_float), ("fdom", C.c_float),
                 ("amp", C.c_float), ("alp", C.c_float), ("spx0", C.c_float), ("spz0", C.c_float),
                 ("dspx", C.c_float), ("offset", C.c_float), ("offsetmax", C.c_float)]
                + [(n, C.c_int) for n in ("startshot", "nshot", "dshot", "nshotall", "npml",
                                          "medium_flag", "ismth")]
                + [("direct", C.c_float), ("direct0", C.c_float)]
                + [(n, C.c_int) for n in ("idevice", "flag_layout", "mode", "dataflag", "sgyflag",
                                          "endianflag", "rhoflag")]
                + [("vp_file", C.c_char * 256), ("shotgather_file", C.c_char * 256),
                   ("rho_file", C.c_char * 256)])


_lib = None


def lib() -> C.CDLL:
    """Load librtm_b200.so (built in-tree by ``__graft_entry__.build()`` / ``make``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run `make -C gubingluo_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    S, O, G = C.POINTER(Survey), C.POINTER(Options), C.POINTER(Geometry)
    vp = C.c_void_p
    L.rtm_last_error.restype = C.c_char_p
    L.rtm_version.restype = C.c_char_p
    L.rtm_session_open.argtypes = [C.POINTER(vp), S, O, C.POINTER(C.c_int), C.c_int, vp, vp, vp, vp, vp]
    L.rtm_session_set_gather.argtypes = [vp, C.c_int, vp]
    L.rtm_session_run.argtypes = [vp, C.POINTER(Stats)]
    L.rtm_session_get_gather.argtypes = [vp, C.c_int, vp]
    L.rtm_session_run_range.argtypes = [vp, C.c_int, C.c_int, C.POINTER(Stats)]
    L.rtm_session_model.argtypes = [vp]
    L.rtm_session_image_ptrs.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    L.rtm_session_get_images.argtypes = [vp, vp, vp, vp, vp]
    L.rtm_session_get_images_f64.argtypes = [vp, vp, vp, vp]
    L.rtm_session_get_images_extra.argtypes = [vp] * 8
    L.rtm_session_reset_images.argtypes = [vp]
    L.rtm_session_nrec.argtypes = [vp, C.c_int]
    L.rtm_session_get_pml.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.rtm_session_tile_heights.argtypes = [vp] + [C.POINTER(C.c_int)] * 4
    L.rtm_session_prepare.argtypes = [vp, C.c_int, C.c_int]
    L.rtm_session_batch_size.argtypes = [vp]
    L.rtm_session_stream.argtypes = [vp]
    L.rtm_session_stream.restype = vp
    L.rtm_session_kernel_ms.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int)]
    L.rtm_session_kernel_ms.restype = C.c_double
    L.rtm_session_get_wavefields.argtypes = [vp, C.c_int, vp, vp]
    L.rtm_session_close.argtypes = [vp]
    L.rtm_session_close.restype = None
    L.rtm_forward.argtypes = [S, O, C.c_int, vp, vp, C.c_int, vp, vp, vp, vp]
    L.rtm_shot_geometry.argtypes = [S, C.c_int, G]
    L.rtm_coef_table.argtypes = [vp]
    L.rtm_coef_table.restype = None
    L.rtm_prepare_model.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]
    L.rtm_velsmooth.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.rtm_pmlsmooth.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.rtm_interp_model.argtypes = [vp, vp] + [C.c_int] * 6
    L.rtm_get_constant.argtypes = ([vp, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                    C.c_float] + [vp] * 10)
    L.rtm_get_constant.restype = None
    L.rtm_laplace_image.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.rtm_laplace_image.restype = None
    L.rtm_scale_image.argtypes = [vp, vp, C.c_int]
    L.rtm_scale_image.restype = None
    L.rtm_read_params.argtypes = [C.c_char_p, C.POINTER(Params)]
    L.rtm_read_velocity.argtypes = [C.c_char_p, C.c_int, C.c_int, vp]
    L.rtm_write_image_su.argtypes = [C.c_char_p, vp, C.c_int, C.c_int, C.c_float]
    L.rtm_write_gather_su.argtypes = [C.c_char_p, vp, G, C.c_int, C.c_int, C.c_int]
    L.rtm_read_gather_su.argtypes = [C.c_char_p, C.c_int, vp, C.POINTER(C.c_int), C.POINTER(C.c_int), G]
    L.rtm_migrate.argtypes = [S, O, C.POINTER(C.c_int), C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                              C.POINTER(Stats)]
    L.rtm_model.restype = None
    L.rtm_real.restype = None
    L.rtm_batch.argtypes = [C.POINTER(BatchDesc), C.POINTER(Stats)]
    L.rtm_session_save_checkpoint.argtypes = [vp, C.c_char_p, C.c_int]
    L.rtm_session_load_checkpoint.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int)]
    L.rtm_checkpoint_info.argtypes = [C.c_char_p] + [C.POINTER(C.c_int)] * 5 + [C.POINTER(C.c_ulonglong)]
    L.rtm_session_config_hash.argtypes = [vp]
    L.rtm_session_config_hash.restype = C.c_ulonglong
    L.rtm_session_guard_count.argtypes = [vp]
    L.rtm_session_open_geometry.argtypes = [C.POINTER(vp), S, O, C.POINTER(C.c_int), G, C.c_int, vp, vp, vp,
                                            vp, vp]
    L.rtm_session_set_gather_raw.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, C.c_float, C.c_int]
    L.rtm_scan_shotgather.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int), vp, C.c_int]
    L.rtm_real_geometry.argtypes = [S, C.c_int, C.c_int, C.c_int, C.c_float, G, C.POINTER(C.c_int)]
    L.rtm_read_shot_traces.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_int, C.c_int,
                                       vp]
    L.rtm_interp_gather.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                    C.c_int]
    _lib = L
    return L


class RtmError(RuntimeError):
    pass


def _check(rc: int):
    if rc != RTM_OK:
        raise RtmError(f"rtm_b200 error {rc}: {lib().rtm_last_error().decode()}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


@dataclass
class SurveyConfig:
    """Python mirror of ``rtm_survey`` (reference parameter-file fields)."""
    nx: int
    nz: int
    nt: int
    dx: float
    dz: float
    dt: float
    npml: int = 32
    fdom: float = 20.0
    amp: float = 1.0
    alp: float = 0.1
    layout: int = 2
    spx0: float = 0.0
    spz0: float = 0.0
    dspx: float = 0.0
    offset: float = 0.0
    offsetmax: float = 0.0
    mode: int = 1
    medium_flag: int = 0
    ismth: int = 0
    direct: float = 1.5
    direct0: float = 0.0
    mute: int = 1
    receiver_depth: int = 0

    def c(self) -> Survey:
        s = Survey()
        for k in self.__dataclass_fields__:
            setattr(s, k, getattr(self, k))
        return s


@dataclass
class RunOptions:
    device: int = 0
    strip_precision: str = "fp32"
    gather_precision: str = "fp32"
    accum_fp64: int = 0     # 0 fp32, 1 (or True) fp64, 2 compensated fp32 pairs, 3 fp64 totals of
                            # 32-step fp32 partial sums; 1-3 stack in fp64
    batch: int = 0
    use_graph: int = 0      # 1: each pass as a CUDA graph per launch shape; 2: with rounded fixed grids
    verbose: bool = False
    extra_images: int = 0   # 1: image3/4/5 and imagetrue, indexing corrected; 2: the reference's
    tsnap: float = 0.0      # with verbose: print max |p| per shot every tsnap seconds

    def c(self) -> Options:
        o = Options()
        o.device = self.device
        o.strip_precision = PREC[self.strip_precision]
        o.gather_precision = PREC[self.gather_precision]
        o.accum_fp64 = int(self.accum_fp64)
        o.batch = self.batch
        o.use_graph = int(self.use_graph)
        o.verbose = int(self.verbose)
        o.extra_images = int(self.extra_images)
        o.tsnap = float(self.tsnap)
        return o


def geometry(survey: SurveyConfig, ishot: int) -> Geometry:
    g = Geometry()
    _check(lib().rtm_shot_geometry(C.byref(survey.c()), ishot, C.byref(g)))
    return g


def coef_table() -> np.ndarray:
    c = np.zeros(100, np.float32)
    lib().rtm_coef_table(_ptr(c))
    return c


class Session:
    """Device-resident migration of a list of shots (``rtm_session_*``).  ``geometries``
    (one ``Geometry`` per shot, e.g. from ``real_geometry``) replaces the survey's layout."""

    def __init__(self, survey: SurveyConfig, options: RunOptions, shots, vp, rho, vp_mig=None,
                 rho_mig=None, diffcoef=None, geometries=None):
        self.survey, self.options = survey, options
        self.shots = np.ascontiguousarray(shots, dtype=np.int32)
        self._keep = [f32(vp), f32(rho)] + [None if a is None else f32(a) for a in (vp_mig, rho_mig, diffcoef)]
        h = C.c_void_p()
        ids = self.shots.ctypes.data_as(C.POINTER(C.c_int))
        if geometries is None:
            _check(lib().rtm_session_open(C.byref(h), C.byref(survey.c()), C.byref(options.c()), ids,
                                          len(self.shots), *[_ptr(a) for a in self._keep]))
        else:
            if len(geometries) != len(self.shots):
                raise ValueError("one geometry per shot")
            self._geoms = (Geometry * len(geometries))(*geometries)
            _check(lib().rtm_session_open_geometry(C.byref(h), C.byref(survey.c()), C.byref(options.c()), ids,
                                                   self._geoms, len(self.shots), *[_ptr(a) for a in self._keep]))
        self.h = h

    def save_checkpoint(self, path: str, shots_done: int):
        """Stacked images after ``shots_done`` shots, for ``load_checkpoint``."""
        _check(lib().rtm_session_save_checkpoint(self.h, path.encode(), shots_done))

    def load_checkpoint(self, path: str) -> int:
        """Restores the images of a checkpoint of the same configuration; returns the number of
        shots it had stacked (continue with ``run_range`` from there)."""
        done = C.c_int(0)
        _check(lib().rtm_session_load_checkpoint(self.h, path.encode(), C.byref(done)))
        return done.value

    def config_hash(self) -> int:
        return lib().rtm_session_config_hash(self.h)

    def guard_count(self) -> int:
        """Guard bands of the checking mode (RTM_B200_GUARDS=1 when the session opened)."""
        return lib().rtm_session_guard_count(self.h)

    def set_gather_raw(self, k: int, seisobs, dt0: float, mirror: int = 0):
        """Recorded traces [nt0][nx0] of shot k, resampled on the device to [nt][nrec_k]."""
        g = f32(seisobs)
        _check(lib().rtm_session_set_gather_raw(self.h, k, _ptr(g), g.shape[1], g.shape[0], dt0, mirror))

    def nrec(self, k: int) -> int:
        return lib().rtm_session_nrec(self.h, k)

    def set_gather(self, k: int, gather):
        g = f32(gather)
        _check(lib().rtm_session_set_gather(self.h, k, _ptr(g)))

    def run(self) -> Stats:
        st = Stats()
        _check(lib().rtm_session_run(self.h, C.byref(st)))
        return st

    def run_range(self, k0: int, n: int) -> Stats:
        st = Stats()
        _check(lib().rtm_session_run_range(self.h, k0, n, C.byref(st)))
        return st

    def model(self):
        """Mode-0 sessions: model every shot's gather (no migration)."""
        _check(lib().rtm_session_model(self.h))

    def image_ptrs(self):
        ptrs = [C.c_void_p() for _ in range(4)]
        _check(lib().rtm_session_image_ptrs(self.h, *[C.byref(p) for p in ptrs]))
        return dict(zip(("image1", "image2s", "image2m", "illum"), [p.value for p in ptrs]))

    def gather(self, k: int) -> np.ndarray:
        g = np.zeros((self.survey.nt, self.nrec(k)), np.float32)
        _check(lib().rtm_session_get_gather(self.h, k, _ptr(g)))
        return g

    def images(self):
        n = (self.survey.nz, self.survey.nx)
        out = [np.zeros(n, np.float32) for _ in range(4)]
        _check(lib().rtm_session_get_images(self.h, *[_ptr(a) for a in out]))
        return dict(zip(("image1", "image2s", "image2m", "illum"), out))

    def images_f64(self):
        n = (self.survey.nz, self.survey.nx)
        out = [np.zeros(n, np.float64) for _ in range(3)]
        _check(lib().rtm_session_get_images_f64(self.h, *[_ptr(a) for a in out]))
        return dict(zip(("image1", "image2s", "illum"), out))

    EXTRA_IMAGES = ("image3s", "image4s", "image5s", "image3m", "image4m", "image5m", "imagetrue")

    def images_extra(self):
        """The other imaging conditions' stacked images (options.extra_images != 0)."""
        n = (self.survey.nz, self.survey.nx)
        out = [np.zeros(n, np.float32) for _ in self.EXTRA_IMAGES]
        _check(lib().rtm_session_get_images_extra(self.h, *[_ptr(a) for a in out]))
        return dict(zip(self.EXTRA_IMAGES, out))

    def reset_images(self):
        _check(lib().rtm_session_reset_images(self.h))

    def stream(self) -> int:
        return lib().rtm_session_stream(self.h)

    def kernel_ms(self, name: str):
        n = C.c_int(0)
        ms = lib().rtm_session_kernel_ms(self.h, name.encode(), C.byref(n))
        return ms, n.value

    def prepare(self, k0: int, n: int):
        """Choose the kernel configuration of every launch shape of run_range(k0, n) now."""
        _check(lib().rtm_session_prepare(self.h, k0, n))

    def batch_size(self) -> int:
        """Shots per launch (batch slots) of the session."""
        return lib().rtm_session_batch_size(self.h)

    def tile_heights(self):
        """Rows per tile in use: {"vel", "vel_recon", "pres", "pres_recon"} (tuned per launch
        shape)."""
        v = [C.c_int(0) for _ in range(4)]
        _check(lib().rtm_session_tile_heights(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("vel", "vel_recon", "pres", "pres_recon"), [x.value for x in v]))

    def pml_profiles(self, k: int, X: int, Z: int):
        """Shot k's device PML damping profiles (ddx [X], ddz [Z], ddxvx [X-1], ddzvz [Z-1])."""
        out = [np.zeros(n, np.float32) for n in (X, Z, X - 1, Z - 1)]
        _check(lib().rtm_session_get_pml(self.h, k, *[_ptr(a) for a in out]))
        return out

    def wavefields(self, slot: int, X: int, Z: int):
        ps = np.zeros((Z, X), np.float32)
        pr = np.zeros((Z, X), np.float32)
        _check(lib().rtm_session_get_wavefields(self.h, slot, _ptr(ps), _ptr(pr)))
        return ps, pr

    def close(self):
        if getattr(self, "h", None):
            lib().rtm_session_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def forward(survey: SurveyConfig, options: RunOptions, ishot: int, vp, rho, nsteps: int):
    """Forward modelling of one shot for ``nsteps`` steps (``rtm_forward``)."""
    g = geometry(survey, ishot)
    X, Z = g.nxpad, g.nzpad
    p = np.zeros((Z, X), np.float32)
    vx = np.zeros((Z, X - 1), np.float32)
    vz = np.zeros((Z - 1, X), np.float32)
    gat = np.zeros((nsteps, g.nrec), np.float32)
    vp, rho = f32(vp), f32(rho)
    _check(lib().rtm_forward(C.byref(survey.c()), C.byref(options.c()), ishot, _ptr(vp), _ptr(rho),
                             nsteps, _ptr(p), _ptr(vx), _ptr(vz), _ptr(gat)))
    return p, vx, vz, gat


def migrate(survey: SurveyConfig, options: RunOptions, shots, vp, rho, gathers=None, vp_mig=None,
            rho_mig=None):
    """Migrate ``shots``; mode 1 needs ``gathers`` (list of [nt][nrec] arrays).  Returns the
    stacked images and, in mode 0, the modelled gathers."""
    with Session(survey, options, shots, vp, rho, vp_mig, rho_mig) as ss:
        if survey.mode == 1:
            for k, g in enumerate(gathers):
                ss.set_gather(k, g)
        stats = ss.run()
        out = ss.images()
        if options.accum_fp64:
            out["f64"] = ss.images_f64()
        if options.extra_images:
            out.update(ss.images_extra())
        if survey.mode == 0:
            out["gathers"] = [ss.gather(k) for k in range(len(ss.shots))]
        out["stats"] = stats
    return out


def checkpoint_info(path: str) -> dict:
    """Header of a checkpoint file (no device work)."""
    v = [C.c_int(0) for _ in range(5)]
    h = C.c_ulonglong(0)
    _check(lib().rtm_checkpoint_info(path.encode(), *[C.byref(x) for x in v], C.byref(h)))
    return dict(zip(("nx", "nz", "nshots", "shots_done", "elem_bytes"), [x.value for x in v]), config_hash=h.value)


# ---- real-data path ----
def scan_shotgather(path: str, sgyflag: int = 0, max_shots: int = 100000):
    """scanshotgather: (profile [4][nshots] with rows sx, traces, first trace, offset;
    endianflag)."""
    prof = np.zeros((4, max_shots), np.int32)
    endian = C.c_int(0)
    n = lib().rtm_scan_shotgather(path.encode(), sgyflag, C.byref(endian), _ptr(prof), max_shots)
    _check(min(n, 0))
    return np.ascontiguousarray(prof[:, :n]), endian.value


def real_geometry(survey: SurveyConfig, sx: int, offset: int, ntrace: int, dx0: float):
    """Geometry of one recorded shot and the number of data-grid columns (ncols0)."""
    g = Geometry()
    nc = C.c_int(0)
    _check(lib().rtm_real_geometry(C.byref(survey.c()), sx, offset, ntrace, dx0, C.byref(g), C.byref(nc)))
    return g, nc.value


def read_shot_traces(path: str, sgyflag: int, endianflag: int, nt0: int, itrace_all: int, ntrace: int,
                     ncols: int) -> np.ndarray:
    out = np.zeros((nt0, ncols), np.float32)
    _check(lib().rtm_read_shot_traces(path.encode(), sgyflag, endianflag, nt0, itrace_all, ntrace, ncols,
                                      _ptr(out)))
    return out


def interp_gather(seisobs, nx: int, nt: int, dt: float, dt0: float, mirror: int = 0, device: int = 0):
    """Interpseis2d on the GPU: [nt0][nx0] -> [nt][nx]."""
    obs = f32(seisobs)
    out = np.zeros((nt, nx), np.float32)
    _check(lib().rtm_interp_gather(_ptr(obs), obs.shape[1], obs.shape[0], _ptr(out), nx, nt, dt, dt0, mirror,
                                   device))
    return out


def migrate_real(survey: SurveyConfig, options: RunOptions, path: str, profile, shots, vp, rho, nt0: int,
                 dt0: float, dx0: float, sgyflag: int = 0, endianflag: int = 0, mirror: int = 0):
    """The real-data driver through a session: recorded shots ``shots`` (1-based numbers into
    ``profile``) of the file at ``path``, resampled, muted in the migration model and
    migrated.  ``survey.mode`` must be 1; ``survey.mute`` 2 mutes as the reference does."""
    prof = np.asarray(profile)
    geoms, cols = [], []
    for ishot in shots:
        sx, ntrace, _, off = (int(prof[r][ishot - 1]) for r in range(4))
        g, nc = real_geometry(survey, sx, off, ntrace, dx0)
        geoms.append(g)
        cols.append(nc)
    with Session(survey, options, shots, vp, rho, geometries=geoms) as ss:
        for k, ishot in enumerate(shots):
            obs = read_shot_traces(path, sgyflag, endianflag, nt0, int(prof[2][ishot - 1]),
                                   int(prof[1][ishot - 1]), cols[k])
            ss.set_gather_raw(k, obs, dt0, mirror)
        stats = ss.run()
        out = ss.images()
        if options.extra_images:
            out.update(ss.images_extra())
        out["stats"] = stats
    return out
