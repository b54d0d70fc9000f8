"""2D solver on the GPU (FP64) against the CPU oracle and analytic times."""
import numpy as np
import pytest

import oracle_lib as O
from models import linear_vz_cells

pytestmark = pytest.mark.gpu


def _setup(fk, nz, nx, h, vel, src, nsweep=2, eps=5.0):
    s = fk.fteik2d()
    s.initialize(nx, nz, h, h, nsweep=nsweep, eps=eps)
    s.setCellVelocityNatural(vel)
    s.setSources(src[1], src[0])
    return s


@pytest.mark.parametrize("shape,src", [((41, 37), (203.3, 148.1)), ((30, 75), (0.0, 401.0)),
                                       ((25, 26), (239.99, 249.99)), ((33, 33), (160.0, 160.0))])
def test_2d_matches_oracle(fk, shape, src):
    nz, nx = shape
    h = 10.0
    vel = linear_vz_cells(nz, nx, 2, h)[0]
    s = _setup(fk, nz, nx, h, vel, src)
    s.solveSourceLSM(1)
    tt = s.getTravelTimeField()
    si, sa = O.source_snap(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), (src[0], src[1], 0.0))
    ref, _ = O.solve2d((nz, nx), (h, h), 1.0 / vel.ravel(), si[:2], sa[:2], 5.0, 2)
    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    s.solveSourceFSM(1)
    assert np.array_equal(s.getTravelTimeField(), tt)
    xz = s.getTravelTimeField(order=fk.FTEIK_XZ_ORDERING)
    assert np.array_equal(xz, tt.reshape(nx, nz).T.ravel())
    s.free()


def test_2d_receivers_and_solveLSM(fk):
    nz, nx, h = 51, 61, 20.0
    vel = linear_vz_cells(nz, nx, 2, h)[0]
    s = fk.fteik2d()
    s.initialize(nx, nz, h, h, nsweep=2, eps=5.0)
    s.setCellVelocityNatural(vel)
    zs, xs = [100.0, 700.0, 0.0], [300.0, 950.0, 1111.0]
    s.setSources(xs, zs)
    zr, xr = np.linspace(0, 1000, 7), np.linspace(0, 1200, 7)
    s.setReceivers(xr, zr)
    s.solveLSM()
    ttr = s.getTravelTimes()
    for k in range(3):
        si, sa = O.source_snap(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), (zs[k], xs[k], 0.0))
        ref, _ = O.solve2d((nz, nx), (h, h), 1.0 / vel.ravel(), si[:2], sa[:2], 5.0, 2)
        want, _ = O.receivers(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), zr, xr, None, ref)
        assert np.max(np.abs(ttr[k] - want)) <= 1e-12 * np.max(want)
    s.free()


def test_2d_linear_gradient_vs_analytic(fk):
    """configuration 1 shape: 201 x 201, h = 10 m, v(z) = 3000 + 0.5 z."""
    nz = nx = 201
    h = 10.0
    vel = linear_vz_cells(nz, nx, 2, h)[0]
    src = (1234.5, 876.5)
    s = _setup(fk, nz, nx, h, vel, src, nsweep=3)
    s.solveSourceLSM(1)
    tt = s.getTravelTimeField()
    ta = O.analytic_linear((nz, nx, 1), (0, 0, 0), (h, h, 1.0), 3000.0, 3000.0 + 0.5 * (nz - 1) * h,
                           (src[0], src[1], 0.0))
    rel = np.abs(tt - ta) / np.maximum(ta, 1e-9)
    far = ta > 10 * h / 3000.0
    assert np.median(rel[far]) < 0.01
    s.free()
