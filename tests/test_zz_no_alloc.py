"""rtm_laplace_image_noalloc (GPU Laplacian through a fixed device scratch, no allocation)
against the host filter rtm_laplace_image, through the C-ABI.

The file name sorts last, so in a full run these tests follow every other test of the
session; each test also passes on its own."""
import ctypes as C

import numpy as np
import pytest

SCRATCH_CELLS = 6 * 1024 * 1024   # the entry's stated limit on nx * nz


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _noalloc(rtmlib):
    f = rtmlib.lib().rtm_laplace_image_noalloc
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    f.restype = C.c_int
    return f


def test_noalloc_refuses_bad_arguments_before_touching_the_device(rtmlib):
    f = _noalloc(rtmlib)
    img = np.zeros(16, np.float32)
    assert f(_p(img), 4096, 2049, 10, 10) == -1            # 8,392,704 cells > scratch
    assert b"scratch" in rtmlib.lib().rtm_last_error()
    assert f(_p(img), SCRATCH_CELLS // 1024 + 1, 1024, 10, 10) == -1
    assert f(None, 4, 4, 10, 10) == -1
    assert f(_p(img), 0, 4, 10, 10) == -1


@pytest.mark.gpu
def test_noalloc_laplace_matches_host_filter_on_consecutive_calls(rtmlib):
    f = _noalloc(rtmlib)
    L = rtmlib.lib()
    rng = np.random.default_rng(2026)
    # two consecutive calls (the second smaller, so stale scratch cells lie beyond it), then
    # the largest image the scratch takes
    for (nz, nx), dx, dz in (((351, 1701), 12, 12), ((173, 301), 10, 7), ((2048, 3072), 5, 5)):
        img = rng.standard_normal((nz, nx)).astype(np.float32)
        want = img.copy()
        L.rtm_laplace_image(_p(want), nx, nz, dx, dz)
        got = img.copy()
        rc = f(_p(got), nx, nz, dx, dz)
        assert rc == 0, L.rtm_last_error()
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_noalloc_laplace_degenerate_shapes(rtmlib):
    """Images one cell wide or tall, and 2 x 2, are all border: every cell must come back
    exactly as the host filter gives it (zero), whatever the scratch held before."""
    f = _noalloc(rtmlib)
    L = rtmlib.lib()
    rng = np.random.default_rng(7)
    # a full call first leaves non-zero values in the scratch
    big = rng.standard_normal((64, 96)).astype(np.float32)
    assert f(_p(big), 96, 64, 10, 10) == 0, L.rtm_last_error()
    for nz, nx in ((1, 257), (311, 1), (2, 2), (1, 1), (3, 2)):
        img = rng.standard_normal((nz, nx)).astype(np.float32)
        want = img.copy()
        L.rtm_laplace_image(_p(want), nx, nz, 10, 10)
        got = img.copy()
        rc = f(_p(got), nx, nz, 10, 10)
        assert rc == 0, L.rtm_last_error()
        assert np.array_equal(got, want), (nz, nx)
