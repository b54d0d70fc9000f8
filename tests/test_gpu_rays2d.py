"""2D ray paths (rays.F90:449-825) on the GPU against the oracle's
restatement, bit for bit: the integration points, the (cell, length) pieces
and the times, for the Euler, midpoint and RK4 integrators, traced in the
field and gradient the library itself computed (downloaded through the C
ABI and handed to the oracle)."""
import ctypes

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

NZ, NX, H = 41, 53, 10.0


def _solver(fk, vel, src):
    s = fk.fteik2d()
    s.initialize(NX, NZ, H, H, nsweep=2, eps=3.0)
    s.setCellVelocityNatural(vel)
    s.setSources(src[1], src[0])
    s.solveSourceLSM(1)
    return s


def _model(seed=4):
    rng = np.random.default_rng(seed)
    zc = (np.arange(NZ - 1) + 0.5) * H
    v = (2500.0 + 3.0 * zc)[None, :] * (1.0 + 0.03 * rng.standard_normal((NX - 1, NZ - 1)))
    return np.ascontiguousarray(v).ravel()          # [nx-1][nz-1], z fastest


# (x, z) end points whose rays reach the source grid point; rays from below or
# right of the source stall just outside the stopping radius (the backward
# differences of solver2D.F90:984-1032 put the gradient's zero half a cell
# off the source), in the oracle as here: see test_stalled_ray_fails_as_in_the_oracle
ENDS = [(0.0, 0.0), (37.3, 211.9), (455.5, 3.3), (100.0, 0.0), (10.0, 50.0), (300.0, 10.0)]


@pytest.mark.parametrize("integrator", [1, 2, 3])
def test_rays_match_oracle_bitwise(fk, integrator):
    vel = _model()
    src = (133.7, 241.2)                            # (z, x)
    s = _solver(fk, vel, src)
    assert s.setODEIntegrator(integrator) == 0
    xe = np.array([e[0] for e in ENDS])
    ze = np.array([e[1] for e in ENDS])
    assert s.traceRaysToPoints(xe, ze) == 0
    rays = s.getRays()
    tt = s.getTravelTimeField()
    gx, gz = s.getTravelTimeGradient()
    si, _ = O.source_snap(False, (NZ, NX, 1), (0, 0, 0), (H, H, 1.0), (src[0], src[1], 0.0))
    src_grid = ((si[1] - 1) * H, (si[0] - 1) * H)   # source.F90:180-181, relative to the origin
    for r, (xr, zr) in enumerate(ENDS):
        st, px, pz, cells, lens, tn, tne = O.ray2d((NZ, NX), (H, H), 1.0 / vel, tt, gx, gz, src_grid,
                                                   integrator, (xr, zr))
        got = rays[r]
        assert st == 0 and got["status"] == 0
        assert np.array_equal(got["x"], px) and np.array_equal(got["z"], pz), r
        assert (got["x"][-1], got["z"][-1]) == src_grid
        assert np.array_equal(got["cells"], cells) and np.array_equal(got["lengths"], lens), r
        assert got["t_step"] == tn and got["t_field"] == tne
        assert got["t_cell"] == pytest.approx(float(np.sum(lens * (1.0 / vel)[cells - 1])), rel=1e-14)
    s.free()


def test_ray_times_in_a_constant_medium(fk):
    """Straight rays: the path length is the distance to the source grid
    point to within the steps' discretisation, and the cell time is that
    length over the velocity."""
    v = 3000.0
    vel = np.full((NX - 1) * (NZ - 1), v)
    src = (200.0, 260.0)                             # on a node: the grid point is the source
    s = _solver(fk, vel, src)
    xe = np.array([10.0, 500.0, 250.0, 30.0])
    ze = np.array([390.0, 20.0, 5.0, 35.0])
    assert s.traceRaysToPoints(xe, ze) == 0
    for r, ray in enumerate(s.getRays()):
        d = np.hypot(xe[r] - src[1], ze[r] - src[0])
        L = float(np.sum(ray["lengths"]))
        assert L == pytest.approx(d, rel=1e-2)          # the Euler steps wiggle about the line
        assert ray["t_cell"] == pytest.approx(L / v, rel=1e-12)
        assert ray["t_field"] == pytest.approx(d / v, rel=2e-2)
    s.free()


def test_stalled_ray_fails_as_in_the_oracle(fk):
    """A ray from below the source ends where the interpolated
    finite-difference gradient vanishes, half a cell from the source and just
    outside the stopping radius (rays.F90:522), and does not reach the source
    within nx nz steps, in the oracle as on the GPU: the call then returns
    ierr = 1 and the other rays are still traced."""
    vel = _model()
    src = (133.7, 241.2)
    s = _solver(fk, vel, src)
    xe, ze = np.array([37.3, 200.0]), np.array([211.9, 399.99])
    assert s.traceRaysToPoints(xe, ze) == 1
    rays = s.getRays()
    tt = s.getTravelTimeField()
    gx, gz = s.getTravelTimeGradient()
    si, _ = O.source_snap(False, (NZ, NX, 1), (0, 0, 0), (H, H, 1.0), (src[0], src[1], 0.0))
    src_grid = ((si[1] - 1) * H, (si[0] - 1) * H)
    for r in range(2):
        st, px, pz, cells, lens, tn, tne = O.ray2d((NZ, NX), (H, H), 1.0 / vel, tt, gx, gz, src_grid, 1,
                                                   (xe[r], ze[r]))
        assert rays[r]["status"] == st == r
        assert np.array_equal(rays[r]["x"], px) and np.array_equal(rays[r]["z"], pz)
    s.free()


def test_integrator_reset_and_refusal(fk):
    """An invalid integrator is refused and leaves Euler; initialising the
    solver resets the integrator to Euler (rays.F90:143,176-229)."""
    vel = _model(7)
    s = _solver(fk, vel, (150.0, 200.0))
    s.traceRaysToPoints([450.0], [350.0])
    euler = s.getRays()[0]
    assert s.setODEIntegrator(7) == 1
    s.traceRaysToPoints([450.0], [350.0])
    assert np.array_equal(s.getRays()[0]["x"], euler["x"])
    assert s.setODEIntegrator(3) == 0
    s.traceRaysToPoints([450.0], [350.0])
    assert not np.array_equal(s.getRays()[0]["x"], euler["x"])
    s.free()
    s = _solver(fk, vel, (150.0, 200.0))             # initialise again: Euler
    s.traceRaysToPoints([450.0], [350.0])
    assert np.array_equal(s.getRays()[0]["x"], euler["x"])
    L = fk.lib()
    n, ierr = ctypes.c_int(), ctypes.c_int(0)
    L.fteik_b200_solver2d_getRayPath(2, 0, None, None, ctypes.byref(n), ctypes.byref(ierr))
    assert ierr.value == 1                            # only one ray traced
    s.free()
