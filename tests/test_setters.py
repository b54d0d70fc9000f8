"""Velocity setters of model.F90 on the host (no GPU needed: the slowness is
built on the host and uploaded at the next solve), against the oracle's
restatement of model.F90:311-754, bit for bit; and the reference's own
Python wrappers binding every symbol they use against this library.

The reference averages nodal velocities with two defects (model.F90:353:
the XYZ ordering omits the 1/8 factor; model.F90:386-389: the natural
ordering uses one y-plane twice).  This library takes the true 8-corner mean;
the oracle reproduces the defects behind keep_defects, so both readings are
checked here: equal to the corrected mean, different from the defective one
where the reference has a defect.
"""
import ctypes
import importlib.util
import os
from ctypes import byref, c_bool, c_int
from importlib.machinery import SourcelessFileLoader

import numpy as np
import pytest

import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _geometry(L, n, h=(10.0, 12.0, 15.0)):
    nz, nx, ny = n
    ierr = c_int(1)
    L.fteik_model_initializeGeometry(ny > 1, nz, nx, ny, 0.0, 0.0, 0.0, *h, byref(ierr))
    assert ierr.value == 0


def _velocity(L, n):
    nz, nx, ny = n
    nv, ierr = c_int(), c_int(1)
    L.fteik_model_getVelocityModel64f(-1, byref(nv), None, byref(ierr))
    ncell = (nz - 1) * (nx - 1) * (ny - 1 if ny > 1 else 1)
    assert ierr.value == 0 and nv.value == ncell
    out = np.zeros(ncell + 3)
    L.fteik_model_getVelocityModel64f(out.size, byref(nv), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      byref(ierr))
    assert ierr.value == 0 and nv.value == ncell and np.all(out[ncell:] == 0.0)
    return out[:ncell]


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


N3, N2 = (7, 6, 5), (9, 8, 1)


@pytest.mark.parametrize("n", [N3, N2])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_cell_setter_orderings(fk, n, order):
    L = fk.lib()
    _geometry(L, n)
    nz, nx, ny = n
    ncell = (nz - 1) * (nx - 1) * (ny - 1 if ny > 1 else 1)
    vel = np.random.default_rng(order).uniform(1500.0, 6000.0, ncell)
    ierr = c_int(1)
    L.fteik_model_setCellVelocityModel64f(ncell, order, _ptr(vel), byref(ierr))
    assert ierr.value == 0
    # 2D knows orders 0 (ZX) and 1 (XZ); 2 falls back to natural order there
    want = 1.0 / O.cell_to_slowness(n, order if (ny > 1 or order < 2) else 0, vel)
    assert np.array_equal(_velocity(L, n), want)


@pytest.mark.parametrize("n", [N3, N2])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_nodal_setter_orderings(fk, n, order):
    L = fk.lib()
    _geometry(L, n)
    nz, nx, ny = n
    ngrd = nz * nx * ny
    vel = np.random.default_rng(10 + order).uniform(1500.0, 6000.0, ngrd)
    ierr = c_int(1)
    L.fteik_model_setNodalVelocityModel64f(ngrd, order, _ptr(vel), byref(ierr))
    assert ierr.value == 0
    o = order if (ny > 1 or order < 2) else 0
    got = _velocity(L, n)
    assert np.array_equal(got, 1.0 / O.nodal_to_slowness(n, o, vel, keep_defects=False))
    defective = 1.0 / O.nodal_to_slowness(n, o, vel, keep_defects=True)
    if ny > 1 and o in (0, 1):
        assert not np.allclose(got, defective)     # model.F90:353 / :386-389 not reproduced
    else:
        assert np.array_equal(got, defective)      # no defect on this path


def test_velocity_setters_32f_and_natural(fk):
    L = fk.lib()
    _geometry(L, N3)
    ncell = 6 * 5 * 4
    v32 = np.random.default_rng(3).uniform(1500.0, 6000.0, ncell).astype(np.float32)
    ierr = c_int(1)
    L.fteik_model_setVelocityModel32f(ncell, v32.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), byref(ierr))
    assert ierr.value == 0
    # model.F90:719-754: slow = 1 / DBLE(vel4)
    assert np.array_equal(_velocity(L, N3), 1.0 / (1.0 / v32.astype(np.float64)))
    v64 = v32.astype(np.float64) * 1.25
    L.fteik_model_setVelocityModel64f(ncell, _ptr(v64), byref(ierr))
    assert ierr.value == 0
    assert np.array_equal(_velocity(L, N3), 1.0 / (1.0 / v64))
    # wrong size and non-positive velocities are refused, and the model is unset
    L.fteik_model_setVelocityModel32f(ncell - 1, v32.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), byref(ierr))
    assert ierr.value == 1
    bad = v32.copy()
    bad[7] = 0.0
    L.fteik_model_setVelocityModel32f(ncell, bad.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), byref(ierr))
    assert ierr.value == 1
    nv = c_int()
    out = np.ones(ncell)
    L.fteik_model_getVelocityModel64f(ncell, byref(nv), _ptr(out), byref(ierr))
    assert ierr.value == 1 and np.all(out == 0.0)
    lis3d = c_bool(False)
    L.fteik_model_isModel3D(byref(lis3d), byref(ierr))
    assert ierr.value == 0 and lis3d.value
    L.fteik_model_free()


def _wrapper(name):
    path = os.path.join(ROOT, "oracle", "_ref", "python", name + ".bytecode")
    if not os.path.exists(path):
        pytest.skip("%s not built (oracle/ref_callers.mk needs the reference tree)" % path)
    os.environ["LD_LIBRARY_PATH"] = os.pathsep.join([os.path.dirname(fteik_lib_path()),
                                                     os.environ.get("LD_LIBRARY_PATH", "")])
    loader = SourcelessFileLoader(name, path)
    spec = importlib.util.spec_from_loader(name, loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def fteik_lib_path():
    import fteik_b200
    return fteik_b200.LIB_PATH


@pytest.mark.parametrize("name,cls", [("fteik3d", "fteik3d"), ("fteik2d", "fteik2d")])
def test_reference_python_wrappers_bind(fk, name, cls):
    """The reference's wrappers, unmodified, find libfteik_shared.so on
    LD_LIBRARY_PATH and set the argument types of every entry point they
    call: each must exist in this library (a missing one raises here)."""
    m = _wrapper(name)
    obj = getattr(m, cls)()
    lib = getattr(obj, name)
    assert os.path.samefile(lib._name, fteik_lib_path())
