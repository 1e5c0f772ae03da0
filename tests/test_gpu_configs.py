"""The CUDA path at the benchmark configurations' own sizes and lengths, through the C-ABI,
against the CPU oracle (FP32 restatement and FP64 build of the same scheme).

* Configuration 1 in full (401 x 201, 40-cell PML, nt = 2000, 20 Hz, receivers 20 m deep,
  layered model with a dipping wedge, one shot): the gather modelled in the true model and
  the images of the migration in the 150 m-smoothed model within 1e-4 rel-L2 of the FP32
  oracle, and within 1e-4 of the FP64 oracle.
* Configuration 4 at full length (nt = 5000, 0.8 ms) on its narrowest and widest drawn
  apertures (201 and 801 columns; 281 x 881 and 881 x 881 padded): fp16 boundary strips and
  gathers with fp64 image accumulation (every step, and fp64 totals of 32-step fp32 partial
  sums) within 1e-3 rel-L2 of the FP64 oracle, bf16 strips and gathers too, plain FP32 within
  1e-4.  The drift of the source wavefield reconstructed
  from fp16 strips against the one reconstructed from fp32 strips, taken at the end of the
  backward pass (t = 0, where the field is the young source wavelet and smallest), is
  reported and held to 1e-2.

The measured errors are printed (pytest -s shows them).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-4
TOL_MIXED = 1e-3
TOL_DRIFT = 1e-2


def _report(name, errs):
    print(f"\n{name}: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))


def test_config1_full_size_against_oracle(rtmlib, oracle):
    from gubingluo_b200 import synthetic

    G = rtmlib
    s, shots, v, vm, rho, meta = synthetic.config(1)
    sd = dict(s.__dict__)
    assert (s.nx, s.nz, s.npml, s.nt) == (401, 201, 40, 2000)
    # modelling in the true model (mode 0 records the gather in the source pass)
    ref0 = oracle.rtm_model(dict(sd, mode=0), shots, v, rho)
    out0 = G.migrate(G.SurveyConfig(**dict(sd, mode=0)), G.RunOptions(), shots, v, rho)
    errs = {"gather": rel_l2(out0["gathers"][0], ref0["gathers"][0])}
    # migration of the oracle's gather in the smoothed model
    data = ref0["gathers"]
    s1 = dict(sd, mode=1)
    ref1 = oracle.rtm_model(s1, shots, vm, rho, gathers=data)
    ref64 = oracle.rtm_model(s1, shots, vm, rho, gathers=data, precision="f64")
    out1 = G.migrate(G.SurveyConfig(**s1), G.RunOptions(), shots, vm, rho, gathers=data)
    for k in ("image1", "image2s", "illum"):
        errs[k] = rel_l2(out1[k], ref1[k])
        errs[k + " vs f64"] = rel_l2(out1[k], ref64[k])
    _report("config 1 (GPU against the FP32 oracle / the FP64 oracle)", errs)
    assert np.abs(out1["image1"]).max() > 0
    for k, e in errs.items():
        assert e < TOL_FP32, (k, e)


def _config4_shot(which):
    from gubingluo_b200 import synthetic

    s, shots, v, vm, rho, meta = synthetic.config(4)
    ap = meta["apertures"]
    ish = (min if which == "narrowest" else max)(shots, key=lambda k: (ap[k], -k if which == "widest" else k))
    sd = dict(s.__dict__, offsetmax=(ap[ish] - 1) * s.dx)
    return sd, ish, ap[ish], v, vm, rho


@pytest.mark.parametrize("which", ["narrowest", "widest"])
def test_config4_precision_form_full_length(rtmlib, oracle, which):
    G = rtmlib
    sd, ish, width, v, vm, rho = _config4_shot(which)
    assert sd["nt"] == 5000 and width in (201, 801)
    # the shot's data: modelled by this library in the true model (the input of both arms)
    out0 = G.migrate(G.SurveyConfig(**dict(sd, mode=0)), G.RunOptions(), [ish], v, rho)
    data = out0["gathers"]
    s1 = dict(sd, mode=1)
    ref64 = oracle.rtm_model(s1, [ish], vm, rho, gathers=data, precision="f64")
    cfg = G.SurveyConfig(**s1)
    forms = {"fp32": G.RunOptions(),
             "fp16": G.RunOptions(strip_precision="fp16", gather_precision="fp16", accum_fp64=True),
             "fp16 blocked": G.RunOptions(strip_precision="fp16", gather_precision="fp16", accum_fp64=3),
             "bf16": G.RunOptions(strip_precision="bf16", gather_precision="bf16", accum_fp64=True)}
    errs = {}
    for name, opts in forms.items():
        out = G.migrate(cfg, opts, [ish], vm, rho, gathers=data)
        for k in ("image1", "image2s", "illum"):
            errs[f"{name} {k}"] = rel_l2(out[k], ref64[k])
    # drift of the reconstructed source wavefield (end of the backward pass) from fp16 strips
    g = G.geometry(cfg, ish)
    fields = {}
    for prec in ("fp32", "fp16"):
        with G.Session(cfg, G.RunOptions(strip_precision=prec, batch=1), [ish], vm, rho) as ss:
            ss.set_gather(0, data[0])
            ss.run()
            fields[prec] = ss.wavefields(0, g.nxpad, g.nzpad)[0]
    npml = sd["npml"]
    inner = (slice(npml, -npml), slice(npml, -npml))
    assert np.abs(fields["fp32"][inner]).max() > 0
    errs["fp16 strip drift"] = rel_l2(fields["fp16"][inner], fields["fp32"][inner])
    _report(f"config 4, shot {ish} ({width} columns, {g.nxpad} x {g.nzpad} padded), against the FP64 oracle", errs)
    for k, e in errs.items():
        tol = TOL_FP32 if k.startswith("fp32") else TOL_DRIFT if k.endswith("drift") else TOL_MIXED
        assert e < tol, (k, e)
