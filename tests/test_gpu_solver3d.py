"""3D solver on the GPU (through the C ABI) against the FP64 CPU oracle.

* precision 8 (FP64 fields): same schedule-independent arithmetic as the
  oracle, so the fields agree to a few ulp;
* precision 4 (FP32 fields, FP64 near-source stencil): the product path,
  relative error <= 1e-4 against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle_lib as O
from models import interior_source, layered_grf_cells, linear_vz_cells

pytestmark = pytest.mark.gpu

TOL32 = 1e-4  # relative travel-time error of the FP32 path vs the FP64 oracle


def _case(name):
    if name == "grf":
        n, h = (23, 19, 17), (25.0, 20.0, 30.0)
        vel = layered_grf_cells(*n, seed=5, min_cells=3)
        src = interior_source(n, h, 7)
    elif name == "linear":
        n, h = (30, 21, 18), (50.0, 50.0, 50.0)
        vel = linear_vz_cells(*n, h[0])
        src = (0.0, 523.0, 411.0)           # surface source: z = 0 nudge
    elif name == "lastcell":
        n, h = (12, 14, 13), (10.0, 10.0, 10.0)
        vel = layered_grf_cells(*n, seed=9, min_cells=2)
        src = (109.99, 129.5, 119.2)        # source cell at nz-1, nx-1, ny-1
    elif name == "node":
        n, h = (15, 16, 17), (10.0, 10.0, 10.0)
        vel = np.full((16, 15, 14), 4000.0)
        src = (70.0, 80.0, 90.0)            # exactly on a node
    elif name == "wide":
        n, h = (9, 70, 11), (10.0, 10.0, 10.0)  # several warps across x
        vel = layered_grf_cells(*n, seed=3, min_cells=2)
        src = (41.0, 333.0, 52.0)
    return n, h, vel, src


def _gpu(fk, n, h, vel, src, precision, nsweep=2, eps=5.0, rec=None):
    s = fk.fteik3d()
    s.initialize(n[1], n[2], n[0], h[1], h[2], h[0], nsweep=nsweep, eps=eps, precision=precision)
    s.setCellSlownessNatural(vel)
    s.setSources(src[1], src[2], src[0])
    if rec is not None:
        s.setReceivers(rec[1], rec[2], rec[0])
    s.solveSourceLSM(1)
    return s


def _oracle(n, h, vel, src, nsweep=2, eps=5.0, **kw):
    si, sa = O.source_snap(True, n, (0, 0, 0), h, src)
    tt, npass = O.solve3d(n, h, 1.0 / np.ravel(vel), si, sa, eps, nsweep, **kw)
    return tt


@pytest.mark.parametrize("name", ["grf", "linear", "lastcell", "node", "wide"])
def test_fp64_matches_oracle(fk, name):
    n, h, vel, src = _case(name)
    s = _gpu(fk, n, h, vel, src, precision=8)
    tt = s.getTravelTimeField()
    ref = _oracle(n, h, vel, src)
    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    s.free()


@pytest.mark.parametrize("name", ["grf", "linear", "lastcell", "node", "wide"])
def test_fp32_within_tolerance(fk, name):
    n, h, vel, src = _case(name)
    s = _gpu(fk, n, h, vel, src, precision=4)
    tt = s.getTravelTimeField()
    ref = _oracle(n, h, vel, src)
    rel = np.abs(tt - ref) / np.maximum(ref, 1e-6)
    k = int(np.argmax(rel))
    where = (k % n[0], (k // n[0]) % n[1], k // (n[0] * n[1]))
    assert np.max(rel) <= TOL32, (np.max(rel), np.sqrt(np.mean(rel ** 2)), where, ref[k], tt[k])
    s.free()


@pytest.mark.parametrize("nsweep", [0, 1, 3])
def test_nsweep_passes(fk, nsweep):
    n, h, vel, src = _case("grf")
    s = _gpu(fk, n, h, vel, src, precision=8, nsweep=nsweep)
    tt = s.getTravelTimeField()
    ref = _oracle(n, h, vel, src, nsweep=nsweep)
    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    assert s.getSolveInfo()[1] == nsweep
    s.free()


def test_orderings_and_cells(fk):
    n, h, vel, src = _case("grf")
    nz, nx, ny = n
    s = _gpu(fk, n, h, vel, src, precision=8)
    nat = s.getTravelTimeField().reshape(ny, nx, nz)
    xyz = s.getTravelTimeField(order=fk.FTEIK_XYZ_ORDERING)
    zyx = s.getTravelTimeField(order=fk.FTEIK_ZYX_ORDERING)
    assert np.array_equal(xyz, nat.transpose(2, 0, 1).ravel())   # x fastest, z slowest
    assert np.array_equal(zyx, nat.transpose(1, 0, 2).ravel())   # z fastest, then y, x
    cell = s.getTravelTimeField(wantCell=True).reshape(ny - 1, nx - 1, nz - 1)
    avg = np.zeros_like(cell)
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                avg += nat[a:ny - 1 + a, b:nx - 1 + b, c:nz - 1 + c]
    assert np.allclose(cell, 0.125 * avg, rtol=1e-14, atol=0)
    s.free()


@pytest.mark.parametrize("precision", [8, 4])
@pytest.mark.parametrize("setter", ["nodal0", "nodal1", "nodal2", "cell32f"])
def test_velocity_setters_solve_like_oracle(fk, setter, precision):
    """Nodal velocities in each ordering (model.F90:311-449) and FP32 cell
    velocities (model.F90:719-754) set through the C ABI and solved on the
    GPU, against the oracle solving the slowness its own restatement of the
    setter builds."""
    import ctypes
    from ctypes import byref, c_int
    n, h = (14, 12, 11), (20.0, 25.0, 30.0)
    nz, nx, ny = n
    rng = np.random.default_rng(21)
    src = interior_source(n, h, 3)
    s = fk.fteik3d()
    s.initialize(nx, ny, nz, h[1], h[2], h[0], precision=precision)
    ierr = c_int(1)
    if setter.startswith("nodal"):
        order = int(setter[-1])
        vel = rng.uniform(2000.0, 5000.0, nz * nx * ny)
        s.lib.fteik_solver3d_setNodalVelocityModel64f(vel.size, order,
                                                      vel.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                      byref(ierr))
        slow = O.nodal_to_slowness(n, order, vel)
    else:
        v32 = rng.uniform(2000.0, 5000.0, (nz - 1) * (nx - 1) * (ny - 1)).astype(np.float32)
        s.lib.fteik_model_setVelocityModel32f(v32.size, v32.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              byref(ierr))
        slow = 1.0 / v32.astype(np.float64)
    assert ierr.value == 0
    s.setSources(src[1], src[2], src[0])
    s.solveSourceLSM(1)
    got = s.getTravelTimeField()
    si, sa = O.source_snap(True, n, (0, 0, 0), h, src)
    want, _ = O.solve3d(n, h, slow, si, sa, 5.0, 2)
    err = np.max(np.abs(got - want)) / np.max(want)
    assert err <= (1e-12 if precision == 8 else TOL32), err
    s.free()


def test_receivers_match_oracle(fk):
    n, h, vel, src = _case("grf")
    rng = np.random.default_rng(4)
    ext = [(n[i] - 1) * h[i] for i in range(3)]
    rec = [rng.uniform(0, ext[i], 25) for i in range(3)]
    rec[0][0], rec[1][1], rec[2][2] = ext[0], 0.0, ext[2]   # on the faces
    s = _gpu(fk, n, h, vel, src, precision=8, rec=rec)
    ttr = s.getTravelTimes()
    ref = _oracle(n, h, vel, src)
    want, ierr = O.receivers(True, n, (0, 0, 0), h, rec[0], rec[1], rec[2], ref)
    assert ierr == 0
    assert np.max(np.abs(ttr - want)) <= 1e-12 * np.max(want)
    s.free()


def test_errors_are_reported(fk):
    import ctypes
    L = fk.lib()
    ierr = ctypes.c_int(0)
    L.fteik_solver3d_free()
    L.fteik_solver3d_initialize(10, 10, 10, 0, 0, 0, 10, 10, 10, 2, 5.0, 0.0, 0, ctypes.byref(ierr))
    assert ierr.value == 0
    L.fteik_solver3d_solveSourceLSM(1, ctypes.byref(ierr))       # no model yet
    assert ierr.value == 1
    vel = np.full(9 ** 3, 3000.0)
    L.fteik_solver3d_setVelocityModel64f(vel.size, vel.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         ctypes.byref(ierr))
    assert ierr.value == 0
    L.fteik_solver3d_solveSourceLSM(1, ctypes.byref(ierr))       # no sources
    assert ierr.value == 1
    z = np.array([200.0])                                        # outside the model
    p = z.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    L.fteik_solver3d_setSources64f(1, p, p, p, ctypes.byref(ierr))
    assert ierr.value == 1
    L.fteik_solver3d_free()


def test_batched_multi_grid(fk):
    grids = [(14, 40, 12, 25.0, 25.0, 25.0), (20, 17, 15, 30.0, 20.0, 25.0)]
    for prec in (8, 4):
        b = fk.Batch3D(grids, nsweep=2, eps=5.0, precision=prec)
        cases = []
        for ig, (nz, nx, ny, dz, dx, dy) in enumerate(grids, start=1):
            vel = layered_grf_cells(nz, nx, ny, seed=20 + ig, min_cells=2)
            b.setVelocityModel(ig, vel)
            rng = np.random.default_rng(ig)
            srcs = [(rng.uniform(0, (nz - 1) * dz), rng.uniform(0, (nx - 1) * dx),
                     rng.uniform(0, (ny - 1) * dy)) for _ in range(3)]
            srcs[0] = (0.0, srcs[0][1], srcs[0][2])
            b.setSources(ig, [s[0] for s in srcs], [s[1] for s in srcs], [s[2] for s in srcs])
            cases.append((ig, (nz, nx, ny), (dz, dx, dy), vel, srcs))
        b.solve()
        for ig, n, h, vel, srcs in cases:
            for k, src in enumerate(srcs, start=1):
                tt = b.field(ig, k)
                ref = _oracle(n, h, vel, src)
                if prec == 8:
                    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
                else:
                    assert np.max(np.abs(tt - ref) / np.maximum(ref, 1e-6)) <= TOL32
            f32 = b.fields32(ig) if prec == 4 else None
            if f32 is not None:
                assert np.array_equal(f32.reshape(len(srcs), -1)[1], b.field(ig, 2).astype(np.float32))
        b.finalize()


def test_batch_rejects_nonpositive_velocity(fk):
    """The batch checks velocities on the device (flag in mapped host
    memory): a zero cell is refused, and the next valid model is accepted."""
    n, h = (10, 12, 11), (20.0, 20.0, 20.0)
    b = fk.Batch3D([(n[0], n[1], n[2], *h)], nsweep=1, eps=3.0, precision=4)
    vel = np.full((n[0] - 1) * (n[1] - 1) * (n[2] - 1), 3000.0)
    bad = vel.copy()
    bad[123] = 0.0
    with pytest.raises(fk.FteikError):
        b.setVelocityModel(1, bad)
    b.setVelocityModel(1, vel)
    b.setSources(1, [0.0], [100.0], [100.0])
    b.solve()
    tt = b.field(1, 1)
    ref = _oracle(n, h, vel, (0.0, 100.0, 100.0), nsweep=1, eps=3.0)
    assert np.max(np.abs(tt - ref) / np.maximum(ref, 1e-6)) <= TOL32
    b.finalize()


def test_source_pairs_match_single_source_bitwise(fk):
    """The batch's Gauss-Seidel passes walk two sources of a grid in the
    same threads (sharing indices, slowness and barriers, not arithmetic),
    and an odd last source walks alone: every source's FP32 field equals the
    one-source solve of that source bit for bit."""
    n, h = (21, 45, 19), (25.0, 25.0, 25.0)
    vel = layered_grf_cells(*n, seed=31, min_cells=2)
    rng = np.random.default_rng(12)
    srcs = [(rng.uniform(0, (n[0] - 1) * h[0]), rng.uniform(0, (n[1] - 1) * h[1]),
             rng.uniform(0, (n[2] - 1) * h[2])) for _ in range(3)]
    b = fk.Batch3D([(n[0], n[1], n[2], *h)], nsweep=2, eps=5.0, precision=4)
    b.setVelocityModel(1, vel)
    b.setSources(1, [s[0] for s in srcs], [s[1] for s in srcs], [s[2] for s in srcs])
    b.solve()
    f32 = b.fields32(1).reshape(len(srcs), -1)
    b.finalize()
    for k, src in enumerate(srcs):
        s = _gpu(fk, n, h, vel, src, 4)
        one = s.getTravelTimeField()
        s.free()
        assert np.array_equal(one.astype(np.float32), f32[k]), k


def test_batched_converged(fk):
    grids = [(16, 18, 14, 25.0, 25.0, 25.0)]
    nz, nx, ny, dz, dx, dy = grids[0]
    vel = layered_grf_cells(nz, nx, ny, seed=31, min_cells=2)
    src = (173.0, 211.0, 96.0)
    b = fk.Batch3D(grids, eps=5.0, convTol=0.0, maxPass=20, precision=8)
    b.setVelocityModel(1, vel)
    b.setSources(1, [src[0]], [src[1]], [src[2]])
    b.solve()
    tt = b.field(1, 1)
    res, npass = b.solveInfo(1, 1)
    ref = _oracle((nz, nx, ny), (dz, dx, dy), vel, src, conv_tol=0.0, max_pass=20)
    assert res == 0.0 and npass < 20
    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    b.finalize()


def test_layered_128cubed_converged_accuracy(fk):
    """128^3, h = 25 m, 4 layers x (1 + 0.05 GRF), interior off-grid source,
    solved to convergence: FP32 GPU vs the FP64 oracle, relative error
    <= 1e-4 at every node."""
    n, h = (128, 128, 128), (25.0, 25.0, 25.0)
    vel = layered_grf_cells(*n, seed=2)
    src = interior_source(n, h, 3)
    b = fk.Batch3D([(n[0], n[1], n[2], *h)], eps=5.0, convTol=0.0, maxPass=30, precision=4)
    b.setVelocityModel(1, vel)
    b.setSources(1, [src[0]], [src[1]], [src[2]])
    b.solve()
    tt = b.field(1, 1)
    res, npass = b.solveInfo(1, 1)
    b.finalize()
    ref = _oracle(n, h, vel, src, conv_tol=0.0, max_pass=30, level_set=True)
    rel = np.abs(tt - ref) / ref.clip(1e-6)
    assert npass < 30 and res == 0.0
    assert np.max(rel) <= TOL32, (np.max(rel), np.sqrt(np.mean(rel ** 2)), npass)


@pytest.mark.parametrize("precision", [8, 4])
def test_gradient_and_trace_entry_points(fk, precision):
    """solver3D.F90:1249-1321 on the device equals the oracle's restatement
    applied to the same field, bit for bit; traceRaysTo* return what the
    reference's do (solver3D.F90:756-823, rays.F90:271-347)."""
    n, h, vel, src = _case("grf")
    s = fk.fteik3d()
    s.initialize(n[1], n[2], n[0], h[1], h[2], h[0], nsweep=2, eps=5.0, precision=precision)
    s.setCellSlownessNatural(vel)
    s.setSources(src[1], src[2], src[0])
    assert s.traceRaysToPoints([10.0], [10.0], [10.0]) == 1          # no field yet
    s.solveSourceLSM(1)
    g = s.getTravelTimeGradient()
    want = O.gradient3d(n, h, s.getTravelTimeField())
    assert np.array_equal(g, want)
    ext = [(n[i] - 1) * h[i] for i in range(3)]                       # z, x, y extents
    assert s.traceRaysToPoints([0.0, ext[1]], [ext[2], 1.0], [ext[0], 0.0]) == 0
    assert s.traceRaysToPoints([ext[1] + 1.0], [1.0], [1.0]) == 1     # outside in x
    assert s.traceRaysToPoints([], [], []) == 1                       # no points
    import ctypes
    ierr = ctypes.c_int(0)
    fk.lib().fteik_solver3d_traceRaysToReceivers(ctypes.byref(ierr))
    assert ierr.value == 1                                            # no receivers
    s.setReceivers([1.0, 2.0], [3.0, 4.0], [5.0, 6.0])
    fk.lib().fteik_solver3d_traceRaysToReceivers(ctypes.byref(ierr))
    assert ierr.value == 0
    s.free()


def test_batched_async_downloads(fk):
    """getTravelTimeFields32fAsync: a download queued after one solve still
    delivers that solve's tables when the next solve runs before it is
    waited for, and equals the synchronous download."""
    grids = [(14, 40, 12, 25.0, 25.0, 25.0), (20, 17, 15, 30.0, 20.0, 25.0)]
    b = fk.Batch3D(grids, nsweep=2, eps=5.0, precision=4)
    rng = np.random.default_rng(6)
    srcs = []
    for ig, (nz, nx, ny, dz, dx, dy) in enumerate(grids, start=1):
        b.setVelocityModel(ig, layered_grf_cells(nz, nx, ny, seed=40 + ig, min_cells=2))
        srcs.append([(rng.uniform(0, (nz - 1) * dz, 3), rng.uniform(0, (nx - 1) * dx, 3),
                      rng.uniform(0, (ny - 1) * dy, 3)) for _ in range(2)])
    outs, refs = [], []
    for step in range(2):
        for ig in (1, 2):
            z, x, y = srcs[ig - 1][step]
            b.setSources(ig, z, x, y)
        b.solve()
        refs.append([b.fields32(ig).copy() for ig in (1, 2)])
        o = [np.full_like(r, -1.0) for r in refs[-1]]
        for ig in (1, 2):
            b.fields32Async(ig, o[ig - 1])
        outs.append(o)
    b.waitDownloads()
    for step in range(2):
        for ig in (0, 1):
            assert np.array_equal(outs[step][ig], refs[step][ig])
    assert not np.array_equal(refs[0][0], refs[1][0])
    b.finalize()


@pytest.mark.parametrize("precision", [8, 4])
@pytest.mark.parametrize("shape", ["deep", "wide"])
def test_deep_and_wide_grids(fk, shape, precision):
    """Grids beyond the slab kernel's default shared memory (nz = 520: the
    per-warp rings of the FP64 passes take 67 KB) and wider than 1024
    columns, against the oracle."""
    if shape == "deep":
        n, h, eps = (520, 5, 6), (10.0, 12.0, 12.0), 5.0
        src = (2511.3, 21.0, 33.0)
        vel = layered_grf_cells(*n, seed=13, min_cells=1)
    else:
        n, h, eps = (4, 1500, 5), (10.0, 10.0, 10.0), 3.0
        src = (11.0, 7403.7, 22.0)
        rng = np.random.default_rng(13)
        vel = linear_vz_cells(*n, h[0]) * (1.0 + 0.05 * rng.standard_normal((n[2] - 1, n[1] - 1, n[0] - 1)))
    s = _gpu(fk, n, h, vel, src, precision=precision, eps=eps)
    tt = s.getTravelTimeField()
    ref = _oracle(n, h, vel, src, eps=eps)
    if precision == 8:
        assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    else:
        assert np.max(np.abs(tt - ref) / np.maximum(ref, 1e-6)) <= TOL32
    s.free()
