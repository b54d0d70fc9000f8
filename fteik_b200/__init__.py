"""fteik_b200 -- B200 (sm_100a) implementation of fteik's eikonal solver and
grid-search locator behind the reference's C ABI.

The product is the shared library ``fteik_b200/lib/libfteik_shared.so``
(C host layer + CUDA kernels); its entry points are declared in
``include/fteik_b200.h``.  This module binds it with ctypes and mirrors the
reference's Python wrappers (python/fteik3d.py, python/fteik2d.py) so that
existing callers read the same.  There is no CPU fallback: if the library
or a CUDA device is missing, calls raise.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, byref, c_bool, c_double, c_float, c_int, c_longlong

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfteik_shared.so")
CSRC = os.path.join(_HERE, "csrc")

FTEIK_NATURAL_ORDERING = 0
FTEIK_ZXY_ORDERING = 0
FTEIK_ZX_ORDERING = 0
FTEIK_XYZ_ORDERING = 1
FTEIK_XZ_ORDERING = 1
FTEIK_ZYX_ORDERING = 2
FTEIK_HUGE = 99999.0

_lib = None

_PD = POINTER(c_double)
_PF = POINTER(c_float)
_PI = POINTER(c_int)

# name -> argtypes (restype void unless listed in _RESTYPES)
_SIGS = {
    # model.F90
    "fteik_model_initializeGeometry": [c_bool, c_int, c_int, c_int] + [c_double] * 6 + [_PI],
    "fteik_model_setGridSize": [c_bool, c_int, c_int, c_int, _PI],
    "fteik_model_setGridSpacing": [c_bool, c_double, c_double, c_double, _PI],
    "fteik_model_setOrigin3D": [c_double, c_double, c_double],
    "fteik_model_setOrigin2D": [c_double, c_double],
    "fteik_model_getGridSize": [_PI, _PI, _PI, _PI, _PI, _PI],
    "fteik_model_setVelocityModel64f": [c_int, _PD, _PI],
    "fteik_model_setNodalVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_model_setCellVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_model_setVelocityModel32f": [c_int, _PF, _PI],
    "fteik_model_getVelocityModel64f": [c_int, _PI, _PD, _PI],
    "fteik_model_isModel3D": [POINTER(c_bool), _PI],
    "fteik_model_grid2indexF": [c_int] * 5,
    "fteik_model_grid2index": [c_int] * 5,
    "fteik_model_index2gridF": [c_int, _PI, _PI, _PI, _PI],
    "fteik_model_velGrid2indexF": [c_int] * 5,
    "fteik_model_free": [],
    # source.F90
    "fteik_source_initialize64f": [c_int, _PD, _PD, _PD, c_int, _PI],
    "fteik_source_getSolverInfo64fF": [c_int, _PI, _PI, _PI, _PD, _PD, _PD, _PD, _PD, _PI],
    "fteik_source_getNumberOfSources": [_PI, _PI],
    "fteik_source_free": [],
    "fteik_source_setVerbosity": [c_int],
    # receiver.F90
    "fteik_receiver_initialize64f": [c_int, _PD, _PD, _PD, c_int, _PI],
    "fteik_receiver_getTravelTimes64f": [c_int, c_int, _PD, _PD, _PI],
    "fteik_receiver_getNumberOfReceivers": [_PI, _PI],
    "fteik_receiver_free": [],
    "fteik_receiver_setVerbosity": [c_int],
    # solver3D.F90
    "fteik_solver3d_initialize": [c_int, c_int, c_int] + [c_double] * 6 + [c_int, c_double, c_double, c_int, _PI],
    "fteik_solver3d_free": [],
    "fteik_solver3d_setVerbosity": [c_int],
    "fteik_solver3d_setConvergenceTolerance": [c_double],
    "fteik_solver3d_setNumberOfSweeps": [c_int, _PI],
    "fteik_solver3d_setSphereToCartEpsilon": [c_double, _PI],
    "fteik_solver3d_setVelocityModel64f": [c_int, _PD, _PI],
    "fteik_solver3d_setCellVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_solver3d_setNodalVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_solver3d_setSources64f": [c_int, _PD, _PD, _PD, _PI],
    "fteik_solver3d_getNumberOfSources": [_PI, _PI],
    "fteik_solver3d_setReceivers64f": [c_int, _PD, _PD, _PD, _PI],
    "fteik_solver3d_getNumberOfReceivers": [_PI, _PI],
    "fteik_solver3d_solveSourceLSM": [c_int, _PI],
    "fteik_solver3d_getTravelTimeField64f": [c_int, c_int, _PD, _PI],
    "fteik_solver3d_getTravelTimeFieldCell64f": [c_int, c_int, _PD, _PI],
    "fteik_solver3d_getTravelTimes64f": [c_int, _PD, _PI],
    "fteik_solver3d_traceRaysToReceivers": [_PI],
    "fteik_solver3d_traceRaysToPoints": [c_int, _PD, _PD, _PD, _PI],
    "fteik_solver2d_traceRaysToReceivers": [_PI],
    "fteik_solver2d_traceRaysToPoints": [c_int, _PD, _PD, _PI],
    # solver2D.F90
    "fteik_solver2d_initialize": [c_int, c_int] + [c_double] * 4 + [c_int, c_double, c_double, c_int, _PI],
    "fteik_solver2d_free": [],
    "fteik_solver2d_setVelocityModel64f": [c_int, _PD, _PI],
    "fteik_solver2d_setCellVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_solver2d_setNodalVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_solver2d_setSources64f": [c_int, _PD, _PD, _PI],
    "fteik_solver2d_setReceivers64f": [c_int, _PD, _PD, _PI],
    "fteik_solver2d_getNumberOfReceivers": [_PI, _PI],
    "fteik_solver2d_solveSourceLSM": [c_int, _PI],
    "fteik_solver2d_solveSourceFSM": [c_int, _PI],
    "fteik_solver2d_solveLSM": [_PI],
    "fteik_solver2d_getTravelTimeField64f": [c_int, c_int, _PD, _PI],
    "fteik_solver2d_getTravelTimeFieldCell64f": [c_int, c_int, _PD, _PI],
    "fteik_solver2d_getTravelTimes64f": [c_int, _PD, _PI],
    # analytic.F90
    "fteik_analytic_initialize64f": [c_int, c_int, c_int] + [c_double] * 6 + [c_int, _PI],
    "fteik_analytic_setSources64f": [c_int, _PD, _PD, _PD, _PI],
    "fteik_analytic_setReceivers64f": [c_int, _PD, _PD, _PD, _PI],
    "fteik_analytic_setConstantVelocity64f": [c_double, _PI],
    "fteik_analytic_setLinearVelocityGradient64f": [c_double, c_double, _PI],
    "fteik_analytic_solveSourceConstantVelocity64f": [c_int, _PI],
    "fteik_analytic_solveSourceLinearVelocityGradient64f": [c_int, _PI],
    "fteik_analytic_getTravelTimeField64f": [c_int, c_int, _PD, _PI],
    "fteik_analytic_getTravelTimesConstantVel64f": [c_int, _PD, _PI],
    "fteik_analytic_getTravelTimesGradientVel64f": [c_int, _PD, _PI],
    "fteik_analytic_free": [],
    "fteik_analytic_setVerbosity": [c_int],
    # locate.F90
    "locate_initialize": [c_int, c_int, c_int, _PI],
    "locate_finalize": [],
    "locate_setTravelTimeField64f": [c_int, c_int, _PD, _PI],
    "locate_setTravelTimeField32f": [c_int, c_int, _PF, _PI],
    "locate_setObservation64f": [c_int, c_int, c_bool, c_double, _PI, _PD, _PD, _PI],
    "locate_setObservation64fC": [c_int, c_int, c_bool, c_double, _PI, _PD, _PD, _PI],
    "locate_locateEvent": [c_int, _PI, _PD, _PD],
    # additions
    "fteik_b200_version": [],
    "fteik_b200_device": [],
    "fteik_b200_stream": [],
    "fteik_b200_setSpinLimit": [c_longlong, _PI],
    "fteik_b200_getSpinLimit": [POINTER(c_longlong)],
    "fteik_b200_setSlabConfig": [c_int, c_int, c_int, c_int, _PI],
    "fteik_b200_getSlabConfig": [_PI, _PI, _PI, _PI],
    "fteik_b200_solver3d_setPrecision": [c_int, _PI],
    "fteik_b200_solver3d_getSolveInfo": [_PD, _PI, _PI],
    "fteik_b200_batch3d_initialize": [c_int, _PI, _PI, _PI, _PD, _PD, _PD, c_int, c_double, c_double,
                                      c_int, c_int, _PI],
    "fteik_b200_batch3d_setVelocityModel64f": [c_int, c_int, _PD, _PI],
    "fteik_b200_batch3d_setSources64f": [c_int, c_int, _PD, _PD, _PD, _PI],
    "fteik_b200_batch3d_setReceivers64f": [c_int, c_int, _PD, _PD, _PD, _PI],
    "fteik_b200_batch3d_solve": [_PI],
    "fteik_b200_batch3d_solveAsync": [],
    "fteik_b200_batch3d_getTravelTimeField64f": [c_int, c_int, c_int, c_int, _PD, _PI],
    "fteik_b200_batch3d_getTravelTimeFields32f": [c_int, c_longlong, _PF, _PI],
    "fteik_b200_batch3d_getTravelTimeFields32fAsync": [c_int, c_longlong, _PF, _PI],
    "fteik_b200_batch3d_waitDownloads": [_PI],
    "fteik_b200_solver3d_getTravelTimeGradient64f": [c_int, _PD, _PI],
    "fteik_b200_solver2d_getTravelTimeGradient64f": [c_int, _PD, _PD, _PI],
    "fteik_rays_setODEIntegrator": [c_int, _PI],
    "fteik_b200_solver2d_getNumberOfRays": [_PI, _PI],
    "fteik_b200_solver2d_getRayTimes": [c_int, _PD, _PD, _PD, _PI, _PI],
    "fteik_b200_solver2d_getRayPath": [c_int, c_int, _PD, _PD, _PI, _PI],
    "fteik_b200_solver2d_getRayCells": [c_int, c_int, _PI, _PD, _PI, _PI],
    "fteik_b200_batch3d_getTravelTimes64f": [c_int, c_int, _PD, _PI],
    "fteik_b200_batch3d_getSolveInfo": [c_int, c_int, _PD, _PI, _PI],
    "fteik_b200_batch3d_exportToLocator": [c_int, c_int, _PI],
    "fteik_b200_batch3d_finalize": [],
    "fteik_b200_batch3d_timeSolve": [POINTER(c_float), POINTER(c_float), _PI],
    "fteik_b200_batch3d_getSlabConfig": [_PI, _PI, _PI, _PI, _PI, _PI, POINTER(c_float), POINTER(c_float), _PI, _PI],
    "fteik_b200_locate_locateEvents": [c_int, _PI, _PI, _PD, _PD, _PI],
    "fteik_b200_locate_setMethod": [c_int, _PI],
    "fteik_b200_locate_setRankingProducts": [c_int, _PI],
    "fteik_b200_locate_getRankingProducts": [_PI],
    "fteik_b200_locate_setNorm": [c_int, _PI],
    "fteik_b200_locate_setRescoreCandidates": [c_int, _PI],
    "fteik_b200_locate_debugAccumulators": [c_int, _PF, _PI],
    "fteik_b200_locate_setGeometry": [c_int, c_int, c_int, c_double, c_double, c_double, c_int, _PD, _PD,
                                      _PD, _PI],
    "fteik_b200_locate_trainSurrogate": [c_longlong, c_int, c_int, c_double, c_double,
                                         ctypes.c_ulonglong, _PD, _PI],
    "fteik_b200_locate_buildSurrogate": [c_int, c_int, c_int, _PI],
    "fteik_b200_locate_setPruning": [c_int, c_int, _PI],
    "fteik_b200_locate_getPruneInfo": [_PI, _PI, POINTER(c_longlong), _PI, _PI],
    "fteik_b200_locate_getSurrogateTable": [c_int, c_int, _PF, _PI],
    "fteik_b200_locate_setStageTiming": [c_int, _PI],
    "fteik_b200_locate_getStageTimes": [POINTER(c_float), POINTER(c_float), POINTER(c_float), _PI],
    "fteik_b200_mlp_initialize": [c_int, c_int, ctypes.c_ulonglong, _PI],
    "fteik_b200_mlp_finalize": [],
    "fteik_b200_mlp_getNumberOfWeights": [_PI, _PI],
    "fteik_b200_mlp_getWeights": [c_int, _PF, _PI],
    "fteik_b200_mlp_setWeights": [c_int, _PF, _PI],
    "fteik_b200_mlp_forward": [c_int, _PF, _PF, _PI],
    "fteik_b200_mlp_gradient": [c_int, _PF, _PF, _PD, _PF, _PI],
    "fteik_b200_mlp_train": [c_int, _PF, _PF, c_int, c_int, c_double, _PD, _PI],
    "fteik_b200_mlp_setTensorProducts": [c_int, _PI],
    "fteik_b200_mlp_getTensorProducts": [_PI],
    "fteik_b200_mlp_setTrainGraph": [c_int],
    "fteik_b200_mlp_getTrainGraph": [_PI],
    "fteik_b200_mlp_setFusedForward": [c_int],
    "fteik_b200_mlp_getFusedForward": [_PI],
    "fteik_b200_mlp_setAsyncStaging": [c_int],
    "fteik_b200_mlp_getAsyncStaging": [_PI],
    "fteik_b200_locate_l2_noalloc": [c_int, c_int, c_int, ctypes.c_void_p, c_int, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, _PI],
    "fteik_h5io_initializeF": [ctypes.c_char_p],
    "fteik_h5io_finalizeF": [],
    "fteik_h5io_writeLevelSchedulesF": [],
    "fteik_h5io_writeVelocityModelF": [ctypes.c_char_p],
    "fteik_h5io_writeTravelTimesF": [ctypes.c_char_p],
}
_RESTYPES = {
    "fteik_model_grid2indexF": c_int,
    "fteik_model_grid2index": c_int,
    "fteik_model_velGrid2indexF": c_int,
    "fteik_b200_version": ctypes.c_char_p,
    "fteik_b200_device": c_int,
    "fteik_b200_stream": ctypes.c_void_p,
    "fteik_b200_batch3d_solveAsync": c_int,
    "fteik_h5io_initializeF": c_int,
    "fteik_h5io_finalizeF": c_int,
    "fteik_h5io_writeLevelSchedulesF": c_int,
    "fteik_h5io_writeVelocityModelF": c_int,
    "fteik_h5io_writeTravelTimesF": c_int,
}


def build(quiet=True):
    """Compile libfteik_shared.so for sm_100a in-tree (nvcc + gcc)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.check_call(["make", "-C", CSRC, "-j8"], stdout=out)
    return LIB_PATH


def lib():
    """The loaded product library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libfteik_shared.so is not built; run fteik_b200.build()")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _RESTYPES.get(name, None)
    _lib = L
    return L


def exported_symbols():
    return sorted(_SIGS)


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_PD)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_PI)


class FteikError(RuntimeError):
    pass


def set_spin_limit(polls):
    """Poll limit of the 3D sweeps' bounded device-side waits (< 0: the
    default); returns the previous limit."""
    old = c_longlong(0)
    lib().fteik_b200_getSpinLimit(byref(old))
    ierr = c_int(1)
    lib().fteik_b200_setSpinLimit(int(polls), byref(ierr))
    _check(ierr, "fteik_b200_setSpinLimit")
    return old.value


def set_slab_config(staged=-1, pairs=-1, progress=-1, blocks_per_sm=-1):
    """Launch configuration of the 3D sweep kernels (-1: the library's
    choice); returns the previous (staged, pairs, progress, blocks_per_sm)."""
    old = [c_int() for _ in range(4)]
    lib().fteik_b200_getSlabConfig(*[byref(v) for v in old])
    ierr = c_int(1)
    lib().fteik_b200_setSlabConfig(int(staged), int(pairs), int(progress), int(blocks_per_sm), byref(ierr))
    _check(ierr, "fteik_b200_setSlabConfig")
    return tuple(v.value for v in old)


def set_mlp_tensor_products(products):
    """Hidden-layer GEMMs of the surrogate: 0 FP32 CUDA cores, 1 BF16
    tensor cores, 3 split-BF16 tensor cores; returns the previous value."""
    old = c_int()
    lib().fteik_b200_mlp_getTensorProducts(byref(old))
    ierr = c_int(1)
    lib().fteik_b200_mlp_setTensorProducts(int(products), byref(ierr))
    _check(ierr, "fteik_b200_mlp_setTensorProducts")
    return old.value


def set_mlp_train_graph(on):
    """Captured (1) or eager (0) training steps of trainSurrogate; returns
    the previous value."""
    old = c_int()
    lib().fteik_b200_mlp_getTrainGraph(byref(old))
    lib().fteik_b200_mlp_setTrainGraph(int(on))
    return old.value


def set_mlp_async_staging(on):
    """Asynchronous (1) or synchronous (0) operand staging of the
    tensor-core products; returns the previous value."""
    old = c_int()
    lib().fteik_b200_mlp_getAsyncStaging(byref(old))
    lib().fteik_b200_mlp_setAsyncStaging(int(on))
    return old.value


def set_mlp_fused_forward(on):
    """Fused (1) or layer-by-layer (0) inference of the surrogate; returns
    the previous value."""
    old = c_int()
    lib().fteik_b200_mlp_getFusedForward(byref(old))
    lib().fteik_b200_mlp_setFusedForward(int(on))
    return old.value


def _check(ierr, what):
    if ierr.value != 0:
        raise FteikError("%s failed (ierr=%d)" % (what, ierr.value))


class fteik3d:
    """Mirror of the reference's python/fteik3d.py class over this library."""

    def __init__(self):
        self.lib = lib()
        self.nx = self.ny = self.nz = 0
        self.nsrc = 0
        self.nrec = 0

    def free(self):
        self.lib.fteik_solver3d_free()

    def initialize(self, nx, ny, nz, dx, dy, dz, x0=0.0, y0=0.0, z0=0.0,
                   nsweep=2, eps=5.0, convTol=0.0, verbose=0, precision=4):
        ierr = c_int(1)
        self.lib.fteik_b200_solver3d_setPrecision(int(precision), byref(ierr))
        _check(ierr, "setPrecision")
        self.lib.fteik_solver3d_initialize(nz, nx, ny, z0, x0, y0, dz, dx, dy, nsweep,
                                           float(eps), float(convTol), verbose, byref(ierr))
        _check(ierr, "fteik_solver3d_initialize")
        self.nx, self.ny, self.nz = nx, ny, nz
        return 0

    def setCellSlownessNatural(self, vel_natural):
        """Cell velocities in the solver's natural order (z fastest)."""
        v, p = _d(np.ravel(vel_natural))
        ierr = c_int(1)
        self.lib.fteik_solver3d_setCellVelocityModel64f(v.size, FTEIK_NATURAL_ORDERING, p, byref(ierr))
        _check(ierr, "setCellVelocityModel64f")

    def setVelocityModel(self, vel):
        """[nz-1, ny-1, nx-1] cell or [nz, ny, nx] nodal velocities (python/fteik3d.py)."""
        vel = np.asarray(vel)
        v, p = _d(np.reshape(vel, vel.size, order="F"))
        ierr = c_int(1)
        if v.size == (self.nx - 1) * (self.ny - 1) * (self.nz - 1):
            self.lib.fteik_solver3d_setCellVelocityModel64f(v.size, FTEIK_ZYX_ORDERING, p, byref(ierr))
        else:
            self.lib.fteik_solver3d_setNodalVelocityModel64f(v.size, FTEIK_ZYX_ORDERING, p, byref(ierr))
        _check(ierr, "setVelocityModel")
        return 0

    def setSources(self, xsrc, ysrc, zsrc):
        x, px = _d(np.atleast_1d(xsrc))
        y, py = _d(np.atleast_1d(ysrc))
        z, pz = _d(np.atleast_1d(zsrc))
        ierr = c_int(1)
        self.lib.fteik_solver3d_setSources64f(x.size, pz, px, py, byref(ierr))
        _check(ierr, "setSources64f")
        self.nsrc = x.size
        return 0

    def setReceivers(self, xrec, yrec, zrec):
        x, px = _d(np.atleast_1d(xrec))
        y, py = _d(np.atleast_1d(yrec))
        z, pz = _d(np.atleast_1d(zrec))
        ierr = c_int(1)
        self.lib.fteik_solver3d_setReceivers64f(x.size, pz, px, py, byref(ierr))
        _check(ierr, "setReceivers64f")
        self.nrec = x.size
        return 0

    def solveSourceLSM(self, isrc):
        ierr = c_int(1)
        self.lib.fteik_solver3d_solveSourceLSM(int(isrc), byref(ierr))
        _check(ierr, "solveSourceLSM")

    def solveLSM(self):
        errorAll = 0
        for i in range(self.nsrc):
            ierr = c_int(1)
            self.lib.fteik_solver3d_solveSourceLSM(i + 1, byref(ierr))
            errorAll += int(ierr.value != 0)
        return errorAll

    def getTravelTimeField(self, wantCell=False, order=FTEIK_NATURAL_ORDERING):
        """Natural-order (z fastest) FP64 field as a flat array."""
        ierr = c_int(1)
        if wantCell:
            n = (self.nx - 1) * (self.ny - 1) * (self.nz - 1)
            out = np.zeros(n)
            self.lib.fteik_solver3d_getTravelTimeFieldCell64f(n, order, out.ctypes.data_as(_PD), byref(ierr))
        else:
            n = self.nx * self.ny * self.nz
            out = np.zeros(n)
            self.lib.fteik_solver3d_getTravelTimeField64f(n, order, out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "getTravelTimeField")
        return out

    def getTravelTimes(self):
        out = np.zeros(max(self.nrec, 1))
        ierr = c_int(1)
        self.lib.fteik_solver3d_getTravelTimes64f(self.nrec, out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "getTravelTimes64f")
        return out[: self.nrec]

    def getTravelTimeGradient(self):
        """(ngrd, 3) array of dT/dx, dT/dy, dT/dz of the current field
        (solver3D.F90:1249-1321), natural node order."""
        n = self.nx * self.ny * self.nz
        out = np.zeros(3 * n)
        ierr = c_int(1)
        self.lib.fteik_b200_solver3d_getTravelTimeGradient64f(n, out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "getTravelTimeGradient64f")
        return out.reshape(n, 3)

    def traceRaysToPoints(self, xp, yp, zp):
        """solver3D.F90:784-823 semantics: returns ierr."""
        x, px = _d(np.atleast_1d(xp))
        y, py = _d(np.atleast_1d(yp))
        z, pz = _d(np.atleast_1d(zp))
        ierr = c_int(1)
        self.lib.fteik_solver3d_traceRaysToPoints(x.size, pz, px, py, byref(ierr))
        return ierr.value

    def getSolveInfo(self):
        r, n, ierr = c_double(), c_int(), c_int(1)
        self.lib.fteik_b200_solver3d_getSolveInfo(byref(r), byref(n), byref(ierr))
        return r.value, n.value


class fteik2d:
    """Mirror of the reference's python/fteik2d.py class over this library."""

    def __init__(self):
        self.lib = lib()
        self.nx = self.nz = 0
        self.nsrc = self.nrec = 0

    def free(self):
        self.lib.fteik_solver2d_free()

    def initialize(self, nx, nz, dx, dz, x0=0.0, z0=0.0, nsweep=2, eps=5.0,
                   convTol=0.0, verbose=0):
        ierr = c_int(1)
        self.lib.fteik_solver2d_initialize(nz, nx, z0, x0, dz, dx, nsweep, float(eps),
                                           float(convTol), verbose, byref(ierr))
        _check(ierr, "fteik_solver2d_initialize")
        self.nx, self.nz = nx, nz
        return 0

    def setCellVelocityNatural(self, vel_natural):
        v, p = _d(np.ravel(vel_natural))
        ierr = c_int(1)
        self.lib.fteik_solver2d_setCellVelocityModel64f(v.size, FTEIK_NATURAL_ORDERING, p, byref(ierr))
        _check(ierr, "setCellVelocityModel64f")

    def setSources(self, xsrc, zsrc):
        x, px = _d(np.atleast_1d(xsrc))
        z, pz = _d(np.atleast_1d(zsrc))
        ierr = c_int(1)
        self.lib.fteik_solver2d_setSources64f(x.size, pz, px, byref(ierr))
        _check(ierr, "setSources64f")
        self.nsrc = x.size

    def setReceivers(self, xrec, zrec):
        x, px = _d(np.atleast_1d(xrec))
        z, pz = _d(np.atleast_1d(zrec))
        ierr = c_int(1)
        self.lib.fteik_solver2d_setReceivers64f(x.size, pz, px, byref(ierr))
        _check(ierr, "setReceivers64f")
        self.nrec = x.size

    def solveSourceLSM(self, isrc):
        ierr = c_int(1)
        self.lib.fteik_solver2d_solveSourceLSM(int(isrc), byref(ierr))
        _check(ierr, "solveSourceLSM")

    def solveSourceFSM(self, isrc):
        ierr = c_int(1)
        self.lib.fteik_solver2d_solveSourceFSM(int(isrc), byref(ierr))
        _check(ierr, "solveSourceFSM")

    def solveLSM(self):
        ierr = c_int(1)
        self.lib.fteik_solver2d_solveLSM(byref(ierr))
        _check(ierr, "solveLSM")

    def getTravelTimeField(self, order=FTEIK_NATURAL_ORDERING):
        n = self.nx * self.nz
        out = np.zeros(n)
        ierr = c_int(1)
        self.lib.fteik_solver2d_getTravelTimeField64f(n, order, out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "getTravelTimeField64f")
        return out

    def getTravelTimeGradient(self):
        """(gradx, gradz) of the current field (solver2D.F90:984-1032)."""
        n = self.nx * self.nz
        gx, gz = np.zeros(n), np.zeros(n)
        ierr = c_int(1)
        self.lib.fteik_b200_solver2d_getTravelTimeGradient64f(n, gx.ctypes.data_as(_PD), gz.ctypes.data_as(_PD),
                                                              byref(ierr))
        _check(ierr, "getTravelTimeGradient64f")
        return gx, gz

    def traceRaysToPoints(self, xp, zp):
        """solver2D.F90:310-350 semantics: returns ierr."""
        x, px = _d(np.atleast_1d(xp))
        z, pz = _d(np.atleast_1d(zp))
        ierr = c_int(1)
        self.lib.fteik_solver2d_traceRaysToPoints(x.size, px, pz, byref(ierr))
        return ierr.value

    def setODEIntegrator(self, integrator):
        """rays.F90:215-229: 1 Euler, 2 midpoint, 3 RK4; returns ierr."""
        ierr = c_int(1)
        self.lib.fteik_rays_setODEIntegrator(int(integrator), byref(ierr))
        return ierr.value

    def getRays(self):
        """The traced rays: list of dicts with the path (x, z), the cells
        and lengths, the times along the steps / from the field / from the
        cells, and the status."""
        n, ierr = c_int(), c_int(1)
        self.lib.fteik_b200_solver2d_getNumberOfRays(byref(n), byref(ierr))
        nr = n.value
        if nr < 1:
            return []
        ts, tf, tc = np.zeros(nr), np.zeros(nr), np.zeros(nr)
        st = np.zeros(nr, np.int32)
        self.lib.fteik_b200_solver2d_getRayTimes(nr, ts.ctypes.data_as(_PD), tf.ctypes.data_as(_PD),
                                                 tc.ctypes.data_as(_PD), st.ctypes.data_as(_PI), byref(ierr))
        _check(ierr, "getRayTimes")
        rays = []
        for r in range(1, nr + 1):
            npts, nseg = c_int(), c_int()
            self.lib.fteik_b200_solver2d_getRayPath(r, 0, None, None, byref(npts), byref(ierr))
            x, z = np.zeros(npts.value), np.zeros(npts.value)
            self.lib.fteik_b200_solver2d_getRayPath(r, npts.value, x.ctypes.data_as(_PD), z.ctypes.data_as(_PD),
                                                    byref(npts), byref(ierr))
            _check(ierr, "getRayPath")
            self.lib.fteik_b200_solver2d_getRayCells(r, 0, None, None, byref(nseg), byref(ierr))
            c, ln = np.zeros(nseg.value, np.int32), np.zeros(nseg.value)
            self.lib.fteik_b200_solver2d_getRayCells(r, nseg.value, c.ctypes.data_as(_PI), ln.ctypes.data_as(_PD),
                                                     byref(nseg), byref(ierr))
            _check(ierr, "getRayCells")
            rays.append({"x": x, "z": z, "cells": c, "lengths": ln, "t_step": ts[r - 1], "t_field": tf[r - 1],
                         "t_cell": tc[r - 1], "status": int(st[r - 1])})
        return rays

    def getTravelTimes(self):
        out = np.zeros(max(self.nrec * self.nsrc, 1))
        ierr = c_int(1)
        self.lib.fteik_solver2d_getTravelTimes64f(self.nrec, out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "getTravelTimes64f")
        return out[: self.nrec * self.nsrc].reshape(self.nsrc, self.nrec)


class Locator:
    """locate.F90's C ABI (locate_initialize ... locate_locateEvent)."""

    def __init__(self, nEvents, ntf, ngrd):
        self.lib = lib()
        ierr = c_int(1)
        self.lib.locate_initialize(nEvents, ntf, ngrd, byref(ierr))
        _check(ierr, "locate_initialize")
        self.nev, self.ntf, self.ngrd = nEvents, ntf, ngrd

    def finalize(self):
        self.lib.locate_finalize()

    def setTravelTimeField64f(self, itf, tt):
        t, p = _d(tt)
        ierr = c_int(1)
        self.lib.locate_setTravelTimeField64f(t.size, int(itf), p, byref(ierr))
        _check(ierr, "locate_setTravelTimeField64f")

    def setTravelTimeField32f(self, itf, tt):
        t = np.ascontiguousarray(tt, dtype=np.float32)
        ierr = c_int(1)
        self.lib.locate_setTravelTimeField32f(t.size, int(itf), t.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "locate_setTravelTimeField32f")

    def setObservation(self, ev, obs2tf, picks, wts, lhaveOT=False, t0=0.0):
        o, po = _i(obs2tf)
        p_, pp = _d(picks)
        w, pw = _d(wts)
        ierr = c_int(1)
        self.lib.locate_setObservation64f(int(ev), o.size, bool(lhaveOT), float(t0), po, pp, pw,
                                          byref(ierr))
        _check(ierr, "locate_setObservation64f")

    def locateEvent(self, ev):
        oi, t0, ob = c_int(), c_double(), c_double()
        self.lib.locate_locateEvent(int(ev), byref(oi), byref(t0), byref(ob))
        return oi.value, t0.value, ob.value

    def locateEvents(self, events):
        ev, pev = _i(events)
        n = ev.size
        oi = np.zeros(n, np.int32)
        t0 = np.zeros(n)
        ob = np.zeros(n)
        ierr = c_int(1)
        self.lib.fteik_b200_locate_locateEvents(n, pev, oi.ctypes.data_as(_PI), t0.ctypes.data_as(_PD),
                                                ob.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "fteik_b200_locate_locateEvents")
        return oi, t0, ob

    def setMethod(self, method):
        """0: exact FP32 search (the reference's arithmetic); 1: tensor-core
        BF16 hi+lo ranking with FP64 re-score of the best candidates."""
        ierr = c_int(1)
        self.lib.fteik_b200_locate_setMethod(int(method), byref(ierr))
        _check(ierr, "fteik_b200_locate_setMethod")

    def setRankingProducts(self, nprod):
        """BF16 products of the tensor-core ranking: 3 (hi+lo both sides)
        or 2 (the event side rounded once); returns the previous value."""
        old, ierr = c_int(), c_int(1)
        self.lib.fteik_b200_locate_getRankingProducts(byref(old))
        self.lib.fteik_b200_locate_setRankingProducts(int(nprod), byref(ierr))
        _check(ierr, "fteik_b200_locate_setRankingProducts")
        return old.value

    def setNorm(self, norm):
        """2: the reference's L2 misfit; 1: L1 with median origin time."""
        ierr = c_int(1)
        self.lib.fteik_b200_locate_setNorm(int(norm), byref(ierr))
        _check(ierr, "fteik_b200_locate_setNorm")

    def setRescoreCandidates(self, ncand):
        ierr = c_int(1)
        self.lib.fteik_b200_locate_setRescoreCandidates(int(ncand), byref(ierr))
        _check(ierr, "fteik_b200_locate_setRescoreCandidates")

    def setGeometry(self, nz, nx, ny, dz, dx, dy, zsta, xsta, ysta):
        z, pz = _d(zsta)
        x, px = _d(xsta)
        y, py = _d(ysta)
        ierr = c_int(1)
        self.lib.fteik_b200_locate_setGeometry(nz, nx, ny, float(dz), float(dx), float(dy), z.size, pz, px, py,
                                               byref(ierr))
        _check(ierr, "fteik_b200_locate_setGeometry")

    def trainSurrogate(self, nsamples=2_000_000, steps=3000, batch=4096, lr=2e-3, vref=3000.0, seed=7):
        loss, ierr = c_double(), c_int(1)
        self.lib.fteik_b200_locate_trainSurrogate(int(nsamples), int(steps), int(batch), float(lr), float(vref),
                                                  int(seed), byref(loss), byref(ierr))
        _check(ierr, "fteik_b200_locate_trainSurrogate")
        return loss.value

    def buildSurrogate(self, block=(4, 4, 4)):
        """Network travel times at the centres of blocks of bz x bx x by
        fine nodes (z, x, y)."""
        ierr = c_int(1)
        bz, bx, by = block
        self.lib.fteik_b200_locate_buildSurrogate(int(bz), int(bx), int(by), byref(ierr))
        _check(ierr, "fteik_b200_locate_buildSurrogate")

    def setPruning(self, runs=4, nodes=8):
        ierr = c_int(1)
        self.lib.fteik_b200_locate_setPruning(int(runs), int(nodes), byref(ierr))
        _check(ierr, "fteik_b200_locate_setPruning")

    def pruneInfo(self):
        """(events searched exhaustively, coarse nodes, blocks examined) of
        the last surrogate-pruned call."""
        nf, nc, nb, mb, ierr = c_int(), c_int(), c_longlong(), c_int(), c_int(1)
        self.lib.fteik_b200_locate_getPruneInfo(byref(nf), byref(nc), byref(nb), byref(mb), byref(ierr))
        self.max_blocks = mb.value
        return nf.value, nc.value, nb.value

    def stageTimes(self, enable=None):
        """With enable=True/False switch stage timing; otherwise return the
        last method-2 call's (coarse ranking, pruned re-score, copy) ms."""
        ierr = c_int(1)
        if enable is not None:
            self.lib.fteik_b200_locate_setStageTiming(int(bool(enable)), byref(ierr))
            return None
        a, b, c = c_float(), c_float(), c_float()
        self.lib.fteik_b200_locate_getStageTimes(byref(a), byref(b), byref(c), byref(ierr))
        return a.value, b.value, c.value

    def surrogateTable(self, itf, ncoarse):
        out = np.zeros(ncoarse, np.float32)
        ierr = c_int(1)
        self.lib.fteik_b200_locate_getSurrogateTable(int(itf), ncoarse, out.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "fteik_b200_locate_getSurrogateTable")
        return out

    def debugAccumulators(self, enable):
        """enable=True: record the first accumulator tiles at the next
        tensor-core search; enable=False: return them as [256, 128]."""
        ierr = c_int(1)
        if enable:
            self.lib.fteik_b200_locate_debugAccumulators(1, None, byref(ierr))
            _check(ierr, "fteik_b200_locate_debugAccumulators")
            return None
        out = np.zeros((256, 128), np.float32)
        self.lib.fteik_b200_locate_debugAccumulators(0, out.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "fteik_b200_locate_debugAccumulators")
        return out


class MLP:
    """The surrogate network (fteik_b200_mlp_*): 6 normalised inputs ->
    depth x width SiLU -> tau."""

    def __init__(self, width=256, depth=5, seed=7):
        self.lib = lib()
        ierr = c_int(1)
        self.lib.fteik_b200_mlp_initialize(int(width), int(depth), int(seed), byref(ierr))
        _check(ierr, "fteik_b200_mlp_initialize")
        self.width, self.depth = width, depth

    def nweights(self):
        n, ierr = c_int(), c_int(1)
        self.lib.fteik_b200_mlp_getNumberOfWeights(byref(n), byref(ierr))
        _check(ierr, "fteik_b200_mlp_getNumberOfWeights")
        return n.value

    def weights(self):
        w = np.zeros(self.nweights(), np.float32)
        ierr = c_int(1)
        self.lib.fteik_b200_mlp_getWeights(w.size, w.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "fteik_b200_mlp_getWeights")
        return w

    def setWeights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        ierr = c_int(1)
        self.lib.fteik_b200_mlp_setWeights(w.size, w.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "fteik_b200_mlp_setWeights")

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 6)
        out = np.zeros(x.shape[0], np.float32)
        ierr = c_int(1)
        self.lib.fteik_b200_mlp_forward(x.shape[0], x.ctypes.data_as(_PF), out.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "fteik_b200_mlp_forward")
        return out

    def gradient(self, x, y):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 6)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(self.nweights(), np.float32)
        loss, ierr = c_double(), c_int(1)
        self.lib.fteik_b200_mlp_gradient(x.shape[0], x.ctypes.data_as(_PF), y.ctypes.data_as(_PF), byref(loss),
                                         g.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "fteik_b200_mlp_gradient")
        return loss.value, g

    def train(self, x, y, steps, batch, lr):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 6)
        y = np.ascontiguousarray(y, np.float32)
        loss, ierr = c_double(), c_int(1)
        self.lib.fteik_b200_mlp_train(x.shape[0], x.ctypes.data_as(_PF), y.ctypes.data_as(_PF), int(steps),
                                      int(batch), float(lr), byref(loss), byref(ierr))
        _check(ierr, "fteik_b200_mlp_train")
        return loss.value

    def finalize(self):
        self.lib.fteik_b200_mlp_finalize()


class Batch3D:
    """Batched multi-source, multi-grid 3D solve (fteik_b200_batch3d_*)."""

    def __init__(self, grids, nsweep=2, eps=5.0, convTol=-1.0, maxPass=0, precision=4):
        """grids: list of (nz, nx, ny, dz, dx, dy)."""
        self.lib = lib()
        g = np.asarray(grids, dtype=np.float64)
        nz, pnz = _i(g[:, 0])
        nx, pnx = _i(g[:, 1])
        ny, pny = _i(g[:, 2])
        dz, pdz = _d(g[:, 3])
        dx, pdx = _d(g[:, 4])
        dy, pdy = _d(g[:, 5])
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_initialize(len(grids), pnz, pnx, pny, pdz, pdx, pdy, nsweep,
                                               float(eps), float(convTol), maxPass, precision,
                                               byref(ierr))
        _check(ierr, "fteik_b200_batch3d_initialize")
        self.grids = [tuple(int(v) for v in r[:3]) for r in g]
        self.nsrc = [0] * len(grids)
        self.precision = precision

    def finalize(self):
        self.lib.fteik_b200_batch3d_finalize()

    def setVelocityModel(self, igrid, vel_natural):
        v, p = _d(np.ravel(vel_natural))
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_setVelocityModel64f(igrid, v.size, p, byref(ierr))
        _check(ierr, "batch3d_setVelocityModel64f")

    def setSources(self, igrid, zsrc, xsrc, ysrc):
        z, pz = _d(zsrc)
        x, px = _d(xsrc)
        y, py = _d(ysrc)
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_setSources64f(igrid, z.size, pz, px, py, byref(ierr))
        _check(ierr, "batch3d_setSources64f")
        self.nsrc[igrid - 1] = z.size

    def setReceivers(self, igrid, zrec, xrec, yrec):
        z, pz = _d(zrec)
        x, px = _d(xrec)
        y, py = _d(yrec)
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_setReceivers64f(igrid, z.size, pz, px, py, byref(ierr))
        _check(ierr, "batch3d_setReceivers64f")
        self.nrec = z.size

    def solve(self):
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_solve(byref(ierr))
        _check(ierr, "batch3d_solve")

    def solveAsync(self):
        return self.lib.fteik_b200_batch3d_solveAsync()

    def field(self, igrid, isrc, order=FTEIK_NATURAL_ORDERING):
        nz, nx, ny = self.grids[igrid - 1]
        out = np.zeros(nz * nx * ny)
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_getTravelTimeField64f(igrid, isrc, out.size, order,
                                                          out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "batch3d_getTravelTimeField64f")
        return out

    def fields32(self, igrid, out=None):
        nz, nx, ny = self.grids[igrid - 1]
        n = self.nsrc[igrid - 1] * nz * nx * ny
        if out is None:
            out = np.empty(n, np.float32)
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_getTravelTimeFields32f(igrid, n, out.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "batch3d_getTravelTimeFields32f")
        return out

    def fields32Async(self, igrid, out):
        """Queue the download of fields32(igrid) into out (pinned host
        memory, untouched until waitDownloads)."""
        nz, nx, ny = self.grids[igrid - 1]
        n = self.nsrc[igrid - 1] * nz * nx * ny
        if out.dtype != np.float32 or out.size < n:
            raise ValueError("out must hold nsrc * ngrd float32 values")
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_getTravelTimeFields32fAsync(igrid, n, out.ctypes.data_as(_PF), byref(ierr))
        _check(ierr, "batch3d_getTravelTimeFields32fAsync")

    def waitDownloads(self):
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_waitDownloads(byref(ierr))
        _check(ierr, "batch3d_waitDownloads")

    def travelTimes(self, igrid):
        n = self.nsrc[igrid - 1] * self.nrec
        out = np.zeros(n)
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_getTravelTimes64f(igrid, n, out.ctypes.data_as(_PD), byref(ierr))
        _check(ierr, "batch3d_getTravelTimes64f")
        return out.reshape(self.nsrc[igrid - 1], self.nrec)

    def solveInfo(self, igrid, isrc):
        r, n, ierr = c_double(), c_int(), c_int(1)
        self.lib.fteik_b200_batch3d_getSolveInfo(igrid, isrc, byref(r), byref(n), byref(ierr))
        _check(ierr, "batch3d_getSolveInfo")
        return r.value, n.value

    def kernelTimes(self):
        a, b, ierr = c_float(), c_float(), c_int(1)
        self.lib.fteik_b200_batch3d_timeSolve(byref(a), byref(b), byref(ierr))
        _check(ierr, "batch3d_timeSolve")
        return a.value, b.value

    def slabConfig(self):
        """The launch configuration in use (tuned on the first solve of a new
        work list where left to the library)."""
        v = [c_int() for _ in range(6)]
        im, pm, runs, ierr = c_float(), c_float(), c_int(), c_int(1)
        self.lib.fteik_b200_batch3d_getSlabConfig(*[byref(x) for x in v], byref(im), byref(pm), byref(runs),
                                                  byref(ierr))
        _check(ierr, "batch3d_getSlabConfig")
        return {"staged": v[0].value, "pairs": v[1].value, "progress": v[2].value,
                "blocks_per_sm": v[3].value, "init_blocks_per_sm": v[4].value, "init_pairs": v[5].value,
                "init_ms": im.value, "pass_ms": pm.value, "tune_runs": runs.value}

    def exportToLocator(self, igrid, itf0=1):
        ierr = c_int(1)
        self.lib.fteik_b200_batch3d_exportToLocator(igrid, itf0, byref(ierr))
        _check(ierr, "batch3d_exportToLocator")
