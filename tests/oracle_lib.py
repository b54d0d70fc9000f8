"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: imported by tests/, the smoke check and the CPU
legs of bench.py, never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_HERE)
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_lib = None

c_int, c_double, c_float = ctypes.c_int, ctypes.c_double, ctypes.c_float
P = ctypes.POINTER


def _ptr(a, ct):
    return a.ctypes.data_as(P(ct))


def load():
    """Load (building first if needed) the oracle shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-C", ORACLE_DIR], stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(ORACLE_SO)
    lib.orc_source_snap.restype = c_int
    lib.orc_source_snap.argtypes = [c_int, c_int, c_int, c_int, c_double, c_double, c_double,
                                    c_double, c_double, c_double, c_double, c_double, c_double,
                                    P(c_int), P(c_int), P(c_int),
                                    P(c_double), P(c_double), P(c_double)]
    lib.orc_cell_velocity_to_slowness.restype = c_int
    lib.orc_cell_velocity_to_slowness.argtypes = [c_int, c_int, c_int, c_int, c_int,
                                                  P(c_double), P(c_double)]
    lib.orc_nodal_velocity_to_slowness.restype = c_int
    lib.orc_nodal_velocity_to_slowness.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int,
                                                   P(c_double), P(c_double)]
    lib.orc_solve3d.restype = c_int
    lib.orc_solve3d.argtypes = [c_int, c_int, c_int, c_double, c_double, c_double, P(c_double),
                                c_int, c_int, c_int, c_double, c_double, c_double,
                                c_double, c_int, c_double, c_int, c_int, c_int,
                                P(c_double), P(c_int)]
    lib.orc_sweep3d.restype = c_int
    lib.orc_sweep3d.argtypes = [c_int, c_int, c_int, c_int, c_int, c_double, c_double, c_double,
                                P(c_double), c_int, c_int, c_int, c_double, c_double, c_double,
                                c_double, P(c_double)]
    lib.orc_ray2d.restype = c_int
    lib.orc_ray2d.argtypes = [c_int, c_int, c_double, c_double] + [P(c_double)] * 4 + \
        [c_double, c_double, c_int, c_double, c_double, c_int, P(c_double), P(c_double), P(c_int), c_int,
         P(c_int), P(c_double), P(c_int), P(c_double), P(c_double)]
    lib.orc_count_updates3d.restype = None
    lib.orc_count_updates3d.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int,
                                        P(ctypes.c_int64), P(ctypes.c_int64)]
    lib.orc_solve2d.restype = c_int
    lib.orc_solve2d.argtypes = [c_int, c_int, c_int, c_double, c_double, P(c_double),
                                c_int, c_int, c_double, c_double, c_double, c_int,
                                c_double, c_int, P(c_double), P(c_int)]
    lib.orc_receiver_setup.restype = None
    lib.orc_receiver_setup.argtypes = [c_int, c_int, c_int, c_int, c_double, c_double, c_double,
                                       c_double, c_double, c_double, c_int,
                                       P(c_double), P(c_double), P(c_double),
                                       P(c_int), P(c_int), P(c_int),
                                       P(c_double), P(c_double), P(c_double), P(c_int)]
    lib.orc_receiver_interp.restype = None
    lib.orc_receiver_interp.argtypes = [c_int, c_int, c_int, c_int, c_double, c_double, c_double,
                                        P(c_double), c_int, P(c_int), P(c_int), P(c_int),
                                        P(c_double), P(c_double), P(c_double), P(c_double)]
    lib.orc_analytic_constant.restype = None
    lib.orc_analytic_constant.argtypes = [c_int, c_int, c_int] + [c_double] * 10 + [P(c_double)]
    lib.orc_analytic_linear.restype = None
    lib.orc_analytic_linear.argtypes = [c_int, c_int, c_int] + [c_double] * 11 + [P(c_double)]
    lib.orc_locate_l2.restype = None
    lib.orc_locate_l2.argtypes = [c_int, c_int, c_int, P(c_float), P(c_float), P(c_float),
                                  P(ctypes.c_ubyte), c_int, P(c_int), P(c_float), P(c_float)]
    lib.orc_locate_l2_field.restype = None
    lib.orc_locate_l2_field.argtypes = [c_int, c_int, c_int, P(c_float), P(c_float), P(c_float),
                                        P(ctypes.c_ubyte), c_int, P(c_float), P(c_float)]
    lib.orc_locate_l2_points64.restype = None
    lib.orc_locate_l2_points64.argtypes = [c_int, c_int, c_int, P(c_float), P(c_float),
                                           P(c_float), P(ctypes.c_ubyte), c_int, P(c_int),
                                           P(c_double), P(c_double)]
    lib.orc_gradient3d.restype = None
    lib.orc_gradient3d.argtypes = [c_int, c_int, c_int, c_double, c_double, c_double, P(c_double),
                                   P(c_double)]
    lib.orc_gradient2d.restype = None
    lib.orc_gradient2d.argtypes = [c_int, c_int, c_double, c_double, P(c_double), P(c_double),
                                   P(c_double)]
    _lib = lib
    return lib


def source_snap(is3d, n, origin, h, src):
    """source.F90:82-236 for one source -> ((zsi,xsi,ysi), (zsa,xsa,ysa)) 1-based."""
    lib = load()
    zi, xi, yi = c_int(), c_int(), c_int()
    za, xa, ya = c_double(), c_double(), c_double()
    nz, nx, ny = n
    rc = lib.orc_source_snap(int(is3d), nz, nx, ny, *origin, *h, *src,
                             ctypes.byref(zi), ctypes.byref(xi), ctypes.byref(yi),
                             ctypes.byref(za), ctypes.byref(xa), ctypes.byref(ya))
    if rc != 0:
        raise ValueError("source outside the model")
    return (zi.value, xi.value, yi.value), (za.value, xa.value, ya.value)


def solve3d(n, h, slow, si, sa, eps, nsweep, conv_tol=-1.0, max_pass=0,
            level_set=False, nthreads=0):
    """Full 3D solveSourceLSM; slow is the FP64 cell slowness (z fastest)."""
    lib = load()
    nz, nx, ny = n
    slow = np.ascontiguousarray(slow, dtype=np.float64).ravel()
    tt = np.empty(nz * nx * ny, dtype=np.float64)
    npass = c_int()
    rc = lib.orc_solve3d(nz, nx, ny, *h, _ptr(slow, c_double), *si, *sa, float(eps),
                         int(nsweep), float(conv_tol), int(max_pass), int(level_set),
                         int(nthreads), _ptr(tt, c_double), ctypes.byref(npass))
    if rc != 0:
        raise ValueError("oracle solve3d failed")
    return tt, npass.value


def solve2d(n, h, slow, si, sa, eps, nsweep, fsm=False, conv_tol=-1.0, max_pass=0):
    lib = load()
    nz, nx = n
    slow = np.ascontiguousarray(slow, dtype=np.float64).ravel()
    tt = np.empty(nz * nx, dtype=np.float64)
    npass = c_int()
    rc = lib.orc_solve2d(int(fsm), nz, nx, *h, _ptr(slow, c_double), si[0], si[1],
                         sa[0], sa[1], float(eps), int(nsweep), float(conv_tol),
                         int(max_pass), _ptr(tt, c_double), ctypes.byref(npass))
    if rc != 0:
        raise ValueError("oracle solve2d failed")
    return tt, npass.value


def cell_to_slowness(n, order, vel):
    """model.F90:505-607: cell velocities in ordering `order` -> FP64 cell
    slowness in natural order.  n = (nz, nx, ny); ny = 1 for 2D."""
    lib = load()
    nz, nx, ny = n
    is3d = ny > 1
    ncell = (nz - 1) * (nx - 1) * (ny - 1 if is3d else 1)
    vel = np.ascontiguousarray(vel, np.float64).ravel()
    slow = np.empty(ncell, np.float64)
    if lib.orc_cell_velocity_to_slowness(int(is3d), nz, nx, ny, int(order), _ptr(vel, c_double),
                                         _ptr(slow, c_double)) != 0:
        raise ValueError("non-positive velocity")
    return slow


def nodal_to_slowness(n, order, vel, keep_defects=False):
    """model.F90:311-449: nodal velocities in ordering `order` -> FP64 cell
    slowness in natural order; keep_defects reproduces the reference's
    XYZ-ordering scale (model.F90:353) and natural-ordering y-plane
    (model.F90:386-389) defects."""
    lib = load()
    nz, nx, ny = n
    is3d = ny > 1
    ncell = (nz - 1) * (nx - 1) * (ny - 1 if is3d else 1)
    vel = np.ascontiguousarray(vel, np.float64).ravel()
    slow = np.empty(ncell, np.float64)
    if lib.orc_nodal_velocity_to_slowness(int(is3d), nz, nx, ny, int(order), int(keep_defects),
                                          _ptr(vel, c_double), _ptr(slow, c_double)) != 0:
        raise ValueError("non-positive velocity")
    return slow


def ray2d(n, h, slow, tt, gx, gz, src_grid, integrator, end):
    """rays.F90:449-825 for one ray: n = (nz, nx), h = (dz, dx), FP64 arrays
    z fastest, src_grid and end = (x, z) relative to the model origin.
    Returns (status, x, z, cells, lengths, t_step, t_field)."""
    lib = load()
    nz, nx = n
    cap = nz * nx + 2
    px, pz = np.zeros(cap), np.zeros(cap)
    cells, lens = np.zeros(4 * cap, np.int32), np.zeros(4 * cap)
    npts, nseg, tn, tne = c_int(), c_int(), c_double(), c_double()
    a = [np.ascontiguousarray(v, np.float64) for v in (slow, tt, gx, gz)]
    st = lib.orc_ray2d(nz, nx, h[0], h[1], *[_ptr(v, c_double) for v in a], float(src_grid[0]),
                       float(src_grid[1]), int(integrator), float(end[0]), float(end[1]), cap,
                       _ptr(px, c_double), _ptr(pz, c_double), ctypes.byref(npts), 4 * cap,
                       _ptr(cells, c_int), _ptr(lens, c_double), ctypes.byref(nseg), ctypes.byref(tn),
                       ctypes.byref(tne))
    k, m = npts.value, nseg.value
    return st, px[:k], pz[:k], cells[:m], lens[:m], tn.value, tne.value


def count_updates3d(n, si):
    lib = load()
    a, b = ctypes.c_int64(), ctypes.c_int64()
    lib.orc_count_updates3d(n[0], n[1], n[2], si[0], si[1], si[2], ctypes.byref(a),
                            ctypes.byref(b))
    return a.value, b.value


def analytic_constant(n, origin, h, v, src):
    lib = load()
    nz, nx, ny = n
    tt = np.empty(nz * nx * ny, dtype=np.float64)
    lib.orc_analytic_constant(nz, nx, ny, *origin, *h, float(v), *src, _ptr(tt, c_double))
    return tt


def analytic_linear(n, origin, h, vtop, vbottom, src):
    lib = load()
    nz, nx, ny = n
    tt = np.empty(nz * nx * ny, dtype=np.float64)
    lib.orc_analytic_linear(nz, nx, ny, *origin, *h, float(vtop), float(vbottom), *src,
                            _ptr(tt, c_double))
    return tt


def receivers(is3d, n, origin, h, z, x, y, tt):
    lib = load()
    nz, nx, ny = n
    nrec = len(z)
    z = np.ascontiguousarray(z, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y if y is not None else np.zeros(nrec), np.float64)
    zri, xri, yri = (np.zeros(nrec, np.int32) for _ in range(3))
    zdr, xdr, ydr = (np.zeros(nrec, np.float64) for _ in range(3))
    ierr = c_int()
    lib.orc_receiver_setup(int(is3d), nz, nx, ny, *origin, *h, nrec, _ptr(z, c_double),
                           _ptr(x, c_double), _ptr(y, c_double), _ptr(zri, c_int),
                           _ptr(xri, c_int), _ptr(yri, c_int), _ptr(zdr, c_double),
                           _ptr(xdr, c_double), _ptr(ydr, c_double), ctypes.byref(ierr))
    tt = np.ascontiguousarray(tt, np.float64)
    out = np.zeros(nrec, np.float64)
    lib.orc_receiver_interp(int(is3d), nz, nx, ny, *h, _ptr(tt, c_double), nrec,
                            _ptr(zri, c_int), _ptr(xri, c_int), _ptr(yri, c_int),
                            _ptr(zdr, c_double), _ptr(xdr, c_double), _ptr(ydr, c_double),
                            _ptr(out, c_double))
    return out, ierr.value


def locate_l2(tables, obs, wts, skip, nthreads=0):
    """FP32 L2 locate for one event. tables: (ntf, ngrd) float32."""
    lib = load()
    tables = np.ascontiguousarray(tables, np.float32)
    ntf, ngrd = tables.shape
    obs = np.ascontiguousarray(obs, np.float32)
    wts = np.ascontiguousarray(wts, np.float32)
    skip = np.ascontiguousarray(skip, np.uint8)
    oi, t0, ob = c_int(), c_float(), c_float()
    lib.orc_locate_l2(ngrd, ngrd, ntf, _ptr(tables, c_float), _ptr(obs, c_float),
                      _ptr(wts, c_float), _ptr(skip, ctypes.c_ubyte), int(nthreads),
                      ctypes.byref(oi), ctypes.byref(t0), ctypes.byref(ob))
    return oi.value, t0.value, ob.value


def locate_l2_field(tables, obs, wts, skip, nthreads=0):
    lib = load()
    tables = np.ascontiguousarray(tables, np.float32)
    ntf, ngrd = tables.shape
    obs = np.ascontiguousarray(obs, np.float32)
    wts = np.ascontiguousarray(wts, np.float32)
    skip = np.ascontiguousarray(skip, np.uint8)
    obj = np.empty(ngrd, np.float32)
    t0 = np.empty(ngrd, np.float32)
    lib.orc_locate_l2_field(ngrd, ngrd, ntf, _ptr(tables, c_float), _ptr(obs, c_float),
                            _ptr(wts, c_float), _ptr(skip, ctypes.c_ubyte), int(nthreads),
                            _ptr(obj, c_float), _ptr(t0, c_float))
    return obj, t0


def locate_l2_best64(tables, obs, wts, nthreads=0):
    """Exhaustive FP64 L2 search for one event: 0-based index of the first
    minimum, FP64 t0 and misfit.  obs/wts: FP64 per table (weight 0 =
    skipped), picks already reduced."""
    lib = load()
    tables = np.ascontiguousarray(tables, np.float32)
    ntf, ngrd = tables.shape
    obs = np.ascontiguousarray(obs, np.float64)
    wts = np.ascontiguousarray(wts, np.float64)
    oi, t0, ob = c_int(), c_double(), c_double()
    nth = int(nthreads) if nthreads else (os.cpu_count() or 1)
    lib.orc_locate_l2_best64(ngrd, ngrd, ntf, _ptr(tables, c_float), _ptr(obs, c_double),
                             _ptr(wts, c_double), nth, ctypes.byref(oi), ctypes.byref(t0),
                             ctypes.byref(ob))
    return oi.value, t0.value, ob.value


def locate_l1_best64(tables, obs, wts, nthreads=0):
    """Exhaustive FP64 L1 search for one event (median origin time)."""
    lib = load()
    tables = np.ascontiguousarray(tables, np.float32)
    ntf, ngrd = tables.shape
    obs = np.ascontiguousarray(obs, np.float64)
    wts = np.ascontiguousarray(wts, np.float64)
    oi, t0, ob = c_int(), c_double(), c_double()
    nth = int(nthreads) if nthreads else (os.cpu_count() or 1)
    lib.orc_locate_l1_best64(ngrd, ngrd, ntf, _ptr(tables, c_float), _ptr(obs, c_double),
                             _ptr(wts, c_double), nth, ctypes.byref(oi), ctypes.byref(t0),
                             ctypes.byref(ob))
    return oi.value, t0.value, ob.value


def gradient3d(n, h, tt):
    """solver3D.F90:1249-1321 -> (ngrd, 3) array of dT/dx, dT/dy, dT/dz."""
    lib = load()
    nz, nx, ny = n
    tt = np.ascontiguousarray(tt, np.float64).ravel()
    g = np.empty(3 * tt.size, np.float64)
    lib.orc_gradient3d(nz, nx, ny, *h, _ptr(tt, c_double), _ptr(g, c_double))
    return g.reshape(-1, 3)


def gradient2d(n, h, tt):
    """solver2D.F90:984-1032 -> (gx, gz)."""
    lib = load()
    nz, nx = n
    tt = np.ascontiguousarray(tt, np.float64).ravel()
    gx, gz = np.empty(tt.size), np.empty(tt.size)
    lib.orc_gradient2d(nz, nx, *h, _ptr(tt, c_double), _ptr(gx, c_double), _ptr(gz, c_double))
    return gx, gz
