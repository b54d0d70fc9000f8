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


def test_2d_solveLSM_batch_equals_source_loop(fk):
    """solveLSM runs all sources in one launch; each source's receiver times
    and the field left behind (the last source's) equal solveSourceLSM's."""
    nz, nx, h = 41, 53, 15.0
    rng = np.random.default_rng(8)
    zc = (np.arange(nz - 1) + 0.5) * h
    vel = (3000.0 + 1.5 * zc)[None, :] * (1.0 + 0.05 * rng.standard_normal((nx - 1, nz - 1)))
    nsrc = 37
    zs = rng.uniform(0, (nz - 1) * h, nsrc)
    xs = rng.uniform(0, (nx - 1) * h, nsrc)
    zs[0], xs[1] = 0.0, (nx - 1) * h            # surface source, source on the last node
    zr, xr = rng.uniform(0, (nz - 1) * h, 11), rng.uniform(0, (nx - 1) * h, 11)
    s = fk.fteik2d()
    s.initialize(nx, nz, h, h, nsweep=2, eps=5.0)
    s.setCellVelocityNatural(vel.ravel())
    s.setSources(xs, zs)
    s.setReceivers(xr, zr)
    s.solveLSM()
    batch = s.getTravelTimes().copy()
    last = s.getTravelTimeField().copy()
    for k in range(nsrc):
        s.solveSourceLSM(k + 1)
    loop = s.getTravelTimes()
    assert np.array_equal(batch, loop)
    assert np.array_equal(last, s.getTravelTimeField())
    for k in (0, 1, nsrc - 1):
        si, sa = O.source_snap(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), (zs[k], xs[k], 0.0))
        ref, _ = O.solve2d((nz, nx), (h, h), 1.0 / vel.ravel(), si[:2], sa[:2], 5.0, 2)
        want, _ = O.receivers(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), zr, xr, None, ref)
        assert np.max(np.abs(batch[k] - want)) <= 1e-12 * np.max(want)
    s.free()


def test_2d_gradient_and_trace_entry_points(fk):
    """solver2D.F90:984-1032 on the device equals the oracle's restatement
    applied to the same field, bit for bit; traceRaysToPoints returns what
    the reference's does (solver2D.F90:310-350)."""
    nz, nx, h = 31, 29, 10.0
    vel = linear_vz_cells(nz, nx, 2, h)[0]
    s = _setup(fk, nz, nx, h, vel, (101.0, 77.0))
    assert s.traceRaysToPoints([10.0], [10.0]) == 1                   # no field yet
    s.solveSourceLSM(1)
    gx, gz = s.getTravelTimeGradient()
    wx, wz = O.gradient2d((nz, nx), (h, h), s.getTravelTimeField())
    assert np.array_equal(gx, wx) and np.array_equal(gz, wz)
    assert s.traceRaysToPoints([0.0, 0.0], [0.0, 100.0]) == 0                # on the boundary
    assert s.traceRaysToPoints([1.0], [(nz - 1) * h + 0.5]) == 1       # below the model
    s.free()


@pytest.mark.parametrize("shape", [(30, 1300), (1100, 1050), (12, 2100)])
def test_2d_more_than_1024_columns(fk, shape):
    """Columns beyond one CTA's 1024 threads are walked block after block
    (thread 0 of a block takes its x-upwind value from the previous block's
    last thread through a ring): FP64 parity with the oracle."""
    nz, nx = shape
    h = 10.0
    rng = np.random.default_rng(nx)
    zc = (np.arange(nz - 1) + 0.5) * h
    vel = ((3000.0 + 0.5 * zc)[None, :] * (1.0 + 0.03 * rng.standard_normal((nx - 1, nz - 1)))).ravel()
    src = (0.37 * (nz - 1) * h, 0.61 * (nx - 1) * h)
    s = _setup(fk, nz, nx, h, vel, src, eps=3.0)
    s.solveSourceLSM(1)
    tt = s.getTravelTimeField()
    si, sa = O.source_snap(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), (src[0], src[1], 0.0))
    ref, _ = O.solve2d((nz, nx), (h, h), 1.0 / vel, si[:2], sa[:2], 3.0, 2)
    # one-ulp differences of hypot (device vs libm) in the near-source
    # analytic times propagate over a million nodes: 1e-11 of the largest time
    assert np.max(np.abs(tt - ref)) <= 1e-11 * np.max(ref)
    s.free()


@pytest.mark.parametrize("kind,order", [("nodal", 0), ("nodal", 1), ("cell", 0), ("cell", 1)])
def test_2d_velocity_setters_solve_like_oracle(fk, kind, order):
    """2D nodal and cell velocities in the ZX (0) and XZ (1) orderings
    (model.F90:311-607) set through the C ABI and solved on the GPU, against
    the oracle solving the slowness its restatement of the setter builds."""
    import ctypes
    from ctypes import byref, c_int
    nz, nx, h = 27, 31, 10.0
    src = (113.3, 171.9)
    rng = np.random.default_rng(12 + order)
    s = fk.fteik2d()
    s.initialize(nx, nz, h, h, nsweep=2, eps=5.0)
    n = nz * nx if kind == "nodal" else (nz - 1) * (nx - 1)
    vel = rng.uniform(2000.0, 5000.0, n)
    p = vel.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ierr = c_int(1)
    if kind == "nodal":
        s.lib.fteik_solver2d_setNodalVelocityModel64f(n, order, p, byref(ierr))
        slow = O.nodal_to_slowness((nz, nx, 1), order, vel)
    else:
        s.lib.fteik_solver2d_setCellVelocityModel64f(n, order, p, byref(ierr))
        slow = O.cell_to_slowness((nz, nx, 1), order, vel)
    assert ierr.value == 0
    s.setSources(src[1], src[0])
    s.solveSourceLSM(1)
    tt = s.getTravelTimeField()
    si, sa = O.source_snap(False, (nz, nx, 1), (0, 0, 0), (h, h, 1.0), (src[0], src[1], 0.0))
    ref, _ = O.solve2d((nz, nx), (h, h), slow, si[:2], sa[:2], 5.0, 2)
    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    s.free()
