import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def reflib():
    from oracle import oracle as O
    L = O.load_reference_host()
    if L is None:
        pytest.skip("reference sources not available to build oracle/_ref")
    return L


@pytest.fixture(scope="session")
def rtmlib():
    """The product library (built in-tree; never a fallback)."""
    so = os.path.join(ROOT, "gubingluo_b200", "librtm_b200.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "gubingluo_b200", "csrc")], check=True)
    import gubingluo_b200 as G
    G.lib()
    return G


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def load_case(name):
    import json
    path = os.path.join(GOLDEN, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} not present")
    z = np.load(path)
    prm = json.loads(bytes(z["params"]).decode())
    return z, prm


def survey_from_case(prm):
    """Survey dict (float fields rounded to float32 as the reference's parameters are)."""
    f = lambda v: float(np.float32(v))
    return dict(nx=prm["nx"], nz=prm["nz"], nt=prm["nt"], dx=f(prm["dx"]), dz=f(prm["dx"]),
                dt=f(prm["dt"]), npml=prm["npml"], fdom=f(prm["fdom"]), amp=f(prm["amp"]),
                alp=f(prm["alp"]), layout=prm["layout"], spx0=f(prm["spx0"]), spz0=f(prm["spz0"]),
                dspx=f(prm["dspx"]), offset=f(prm["offset"]), offsetmax=f(prm["offsetmax"]),
                mode=prm["mode"], medium_flag=prm["medium_flag"], ismth=prm["ismth"],
                direct=f(prm["direct"]), direct0=f(prm["direct0"]), mute=1, receiver_depth=0)
