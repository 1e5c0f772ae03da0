"""Scheme tests of the oracle on small grids: how much the split-field PML echoes back.

The echo of a PML is measured against a run whose grid is large enough that no boundary
echo reaches the receivers within the record: the model of the small run, edge-replicated by
E cells on every side (the medium the small run's PML absorbs), with the source and the
receiver line at the same physical cells.  The difference between the two gathers is the
echo of the small run's PML (the PML formula is the reference's, kernel.cu:174-269, with
its Crank-Nicolson update kernel.cu:542-1185).

E is chosen so that the shortest path source -> outer boundary -> receiver of the large
run, 2 (rz + E) - nxi/2 cells, is longer than the distance v nt dt travelled in the record.
"""
import numpy as np
import pytest


def _gather(oracle, nxi, nzi, E, npml, v, dx, dt, fdom, nt, sx, sz, rz, precision):
    X, Z = nxi + 2 * (E + npml), nzi + 2 * (E + npml)
    vp2 = np.full((Z, X), np.float32(v) ** 2, np.float32)
    rho = np.full((Z, X), 2000.0, np.float32)
    off = npml + E
    shot = oracle.shot_struct(X, Z, npml, nt, dx, dx, dt, off + sx, off + sz, 1.0, 1.0 / dx, fdom,
                              off + rz, off, nxi, np.float32(v))
    return oracle.forward(shot, vp2, rho, nt, precision=precision)[3].astype(np.float64)


# (dx, dt, fdom, npml, E, bound on the echo's peak / the gather's peak); measured peaks:
# 1.5e-7 with the 80-cell PML at 7.5 m, 18 Hz, 0.5 ms (the high-contrast configuration's
# settings), 3.0e-6 with the reference's 32-cell PML at 12.5 m, 15 Hz, 1 ms.
CASES = {
    "npml80_dx7.5": (7.5, 5e-4, 18.0, 80, 160, 1e-6),
    "npml32_dx12.5": (12.5, 1e-3, 15.0, 32, 180, 2e-5),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_pml_echo_is_small(oracle, name):
    dx, dt, fdom, npml, E, bound = CASES[name]
    v, nxi, nzi, sx, sz, rz, nt = 2000.0, 201, 101, 100, 10, 10, 1600
    assert 2 * (rz + E) - nxi // 2 > v * nt * dt / dx, "the large run's own echo would reach the receivers"
    small = _gather(oracle, nxi, nzi, 0, npml, v, dx, dt, fdom, nt, sx, sz, rz, "f64")
    large = _gather(oracle, nxi, nzi, E, npml, v, dx, dt, fdom, nt, sx, sz, rz, "f64")
    echo = small - large
    peak = np.abs(echo).max() / np.abs(large).max()
    assert peak < bound, f"PML echo peak {peak:.2e} of the gather's peak"
    assert np.sum(echo ** 2) < bound ** 2 * np.sum(large ** 2)


def test_pml_echo_detects_a_missing_pml(oracle):
    """The same measurement on a run whose PML has no damping (vpmax ~ 0 gives d0 ~ 0): the
    outer boundary then reflects, and the echo is of the order of the direct wave."""
    dx, dt, fdom, npml, E = 12.5, 1e-3, 15.0, 32, 180
    v, nxi, nzi, sx, sz, rz, nt = 2000.0, 201, 101, 100, 10, 10, 1600
    X, Z = nxi + 2 * npml, nzi + 2 * npml
    vp2 = np.full((Z, X), np.float32(v) ** 2, np.float32)
    rho = np.full((Z, X), 2000.0, np.float32)
    shot = oracle.shot_struct(X, Z, npml, nt, dx, dx, dt, npml + sx, npml + sz, 1.0, 1.0 / dx, fdom,
                              npml + rz, npml, nxi, np.float32(1e-6))
    undamped = oracle.forward(shot, vp2, rho, nt, precision="f64")[3].astype(np.float64)
    large = _gather(oracle, nxi, nzi, E, npml, v, dx, dt, fdom, nt, sx, sz, rz, "f64")
    assert np.abs(undamped - large).max() / np.abs(large).max() > 1e-2
