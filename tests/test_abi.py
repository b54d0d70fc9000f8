"""The C ABI library without a GPU: it loads, exports every entry point the
public header declares, and runs its host-only logic."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import fteik_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fteik_b200.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:fteik|locate)_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(fk):
    out = subprocess.check_output(["nm", "-D", "--defined-only", fteik_b200.LIB_PATH]).decode()
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = [s for s in _declared() if s not in exported]
    assert not missing, missing
    # and nothing but the C ABI is exported
    assert all(s.startswith(("fteik_", "locate_")) for s in exported), exported
    for s in _declared():
        getattr(fk.lib(), s)


def test_header_compiles_as_c_and_links(fk, tmp_path):
    """A C caller: the public header compiles as C11 (gcc, warnings as
    errors) and every function it declares resolves against the library at
    link time.  Nothing is run."""
    names = _declared()
    src = tmp_path / "caller.c"
    src.write_text('#include "fteik_b200.h"\n#include <stdio.h>\n'
                   "int main(void)\n{\n    void (*const fns[])(void) = {\n" +
                   "".join("        (void (*)(void))%s,\n" % n for n in names) +
                   "    };\n    printf(\"%d\\n\", (int)(sizeof(fns) / sizeof(fns[0])));\n    return 0;\n}\n")
    libdir = os.path.dirname(fteik_b200.LIB_PATH)
    # the header needs nothing but the C standard library (no CUDA headers)
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(tmp_path / "caller"), "-L", libdir, "-lfteik_shared", "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_reference_python_wrapper_symbols_present(fk):
    """python/fteik3d.py, fteik2d.py and fteikAnalytic.py bind these at
    construction; every one must resolve."""
    names = ["fteik_solver3d_initialize", "fteik_solver3d_setReceivers64f",
             "fteik_solver3d_solveSourceLSM", "fteik_solver3d_getTravelTimeField64f",
             "fteik_solver3d_getTravelTimeFieldCell64f", "fteik_solver3d_setCellVelocityModel64f",
             "fteik_solver3d_setNodalVelocityModel64f", "fteik_solver3d_setSources64f",
             "fteik_solver3d_getTravelTimes64f", "fteik_solver3d_getNumberOfReceivers",
             "fteik_h5io_initializeF", "fteik_h5io_writeLevelSchedulesF",
             "fteik_h5io_writeTravelTimesF", "fteik_h5io_writeVelocityModelF",
             "fteik_h5io_finalizeF", "fteik_solver3d_free", "fteik_solver2d_initialize",
             "fteik_solver2d_setCellVelocityModel64f", "fteik_solver2d_setNodalVelocityModel64f",
             "fteik_solver2d_setReceivers64f", "fteik_solver2d_solveLSM",
             "fteik_solver2d_solveSourceLSM", "fteik_solver2d_solveSourceFSM",
             "fteik_solver2d_getTravelTimeField64f", "fteik_solver2d_getTravelTimeFieldCell64f",
             "fteik_solver2d_setSources64f", "fteik_solver2d_getTravelTimes64f",
             "fteik_solver2d_getNumberOfReceivers", "fteik_solver2d_free",
             "fteik_analytic_initialize64f", "fteik_analytic_setReceivers64f",
             "fteik_analytic_solveSourceLinearVelocityGradient64f",
             "fteik_analytic_solveSourceConstantVelocity64f",
             "fteik_analytic_setLinearVelocityGradient64f", "fteik_analytic_setConstantVelocity64f",
             "fteik_analytic_getTravelTimeField64f", "fteik_analytic_getTravelTimesConstantVel64f",
             "fteik_analytic_getTravelTimesGradientVel64f", "fteik_analytic_setSources64f",
             "fteik_analytic_free"]
    L = fk.lib()
    for n in names:
        getattr(L, n)


def test_index_round_trip(fk):
    """testing/tests.c:262-302 on 34 x 10 x 21."""
    L = fk.lib()
    ierr = ctypes.c_int(1)
    L.fteik_model_setGridSize(True, 34, 10, 21, ctypes.byref(ierr))
    assert ierr.value == 0
    i1, j1, k1 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    for k in range(1, 22):
        for j in range(1, 11):
            for i in range(1, 35):
                g = L.fteik_model_grid2indexF(i, j, k, 34, 340)
                L.fteik_model_index2gridF(g, ctypes.byref(i1), ctypes.byref(j1), ctypes.byref(k1),
                                          ctypes.byref(ierr))
                assert ierr.value == 0 and (i1.value, j1.value, k1.value) == (i, j, k)
                assert L.fteik_model_grid2index(i - 1, j - 1, k - 1, 34, 340) == g - 1
    L.fteik_model_free()


def test_host_validation(fk):
    L = fk.lib()
    ierr = ctypes.c_int(0)
    L.fteik_model_setGridSize(True, 2, 10, 10, ctypes.byref(ierr))
    assert ierr.value == 1
    L.fteik_model_initializeGeometry(True, 10, 11, 12, 0.0, 0.0, 0.0, 10.0, 10.0, 10.0, ctypes.byref(ierr))
    assert ierr.value == 0
    v = np.full(9 * 10 * 11, 2000.0)
    v[5] = -1.0
    L.fteik_model_setVelocityModel64f(v.size, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      ctypes.byref(ierr))
    assert ierr.value == 1
    z = np.array([5.0, 95.0])
    x = np.array([5.0, 100.0])
    y = np.array([5.0, 110.5])
    PD = ctypes.POINTER(ctypes.c_double)
    L.fteik_source_initialize64f(2, z.ctypes.data_as(PD), x.ctypes.data_as(PD),
                                 y.ctypes.data_as(PD), 0, ctypes.byref(ierr))
    assert ierr.value == 1          # y = 110.5 lies outside [0, 110]
    L.fteik_model_free()
    assert L.fteik_h5io_initializeF(b"x.h5") == -1     # no model: h5io.F90:110-114


def test_argument_checks_before_the_device(fk):
    """Arguments the library refuses before touching a device."""
    L = fk.lib()
    ierr = ctypes.c_int(0)
    L.locate_initialize(1, 65, 100, ctypes.byref(ierr))
    assert ierr.value == 1                       # at most 64 tables per grid point
    L.locate_initialize(0, 4, 100, ctypes.byref(ierr))
    assert ierr.value == 1
    for bad in (-1, 3):
        L.fteik_b200_locate_setMethod(bad, ctypes.byref(ierr))
        assert ierr.value == 1
    L.fteik_b200_locate_setNorm(3, ctypes.byref(ierr))
    assert ierr.value == 1
    IA = ctypes.c_int * 1
    DA = ctypes.c_double * 1
    n, h = IA(10), DA(10.0)
    args = (n, n, n, h, h, h)
    for ngrid, nsweep, prec in ((0, 2, 4), (1, 2, 3), (1, -1, 4)):
        ierr.value = 0
        L.fteik_b200_batch3d_initialize(ngrid, *args, nsweep, ctypes.c_double(5.0), ctypes.c_double(-1.0), 0,
                                        prec, ctypes.byref(ierr))
        assert ierr.value == 1, (ngrid, nsweep, prec)
    L.locate_finalize()


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the behaviour without a CUDA device")
def test_compute_fails_loudly_without_gpu(fk):
    L = fk.lib()
    ierr = ctypes.c_int(0)
    L.fteik_solver3d_initialize(10, 10, 10, 0, 0, 0, 10, 10, 10, 2, 5.0, 0.0, 0, ctypes.byref(ierr))
    assert ierr.value == 1
    L.locate_initialize(1, 4, 100, ctypes.byref(ierr))
    assert ierr.value == 1


def test_archive_levels_and_velocities(fk, tmp_path):
    """The archive entry points (h5io.F90:104-420) write the reference's
    datasets as .npy files: INT16 level schedules of the 8 sweeps
    (graph3d.F90 levels, x fastest) and INT16 velocities per cell."""
    L = fk.lib()
    ierr = ctypes.c_int(0)
    nz, nx, ny = 6, 7, 5
    L.fteik_model_initializeGeometry(True, nz, nx, ny, 0.0, 0.0, 0.0, 10.0, 20.0, 30.0, ctypes.byref(ierr))
    assert ierr.value == 0
    rng = np.random.default_rng(3)
    vel = rng.uniform(1500.0, 6000.0, (ny - 1) * (nx - 1) * (nz - 1))   # natural order, z fastest
    L.fteik_model_setVelocityModel64f(vel.size, vel.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      ctypes.byref(ierr))
    assert ierr.value == 0
    assert L.fteik_h5io_initializeF(str(tmp_path / "arch.txt").encode()) == -1   # not .h5/.hdf5
    assert L.fteik_h5io_initializeF(str(tmp_path / "sub" / "arch.h5").encode()) == 0
    d = tmp_path / "sub" / "arch.h5.d"
    assert L.fteik_h5io_writeLevelSchedulesF() == 0
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    for s in range(8):
        pz = nz - 1 - iz if s >= 4 else iz
        px = nx - 1 - ix if s % 2 else ix
        py = ny - 1 - iy if (s // 2) % 2 else iy
        got = np.load(d / "LevelSchedules" / f"Sweep_{s + 1}.npy")
        assert got.dtype == np.int16 and np.array_equal(got, pz + px + py + 1)
    assert L.fteik_h5io_writeVelocityModelF(b"model") == 0
    assert L.fteik_h5io_writeVelocityModelF(b"model") == -1                       # name taken
    got = np.load(d / "VelocityModels" / "model.npy")
    want = np.floor(1.0 / (1.0 / vel) + 0.5).astype(np.int16).reshape(ny - 1, nx - 1, nz - 1)
    assert np.array_equal(got, want.transpose(2, 0, 1))                         # x fastest
    assert L.fteik_h5io_writeTravelTimesF(b"tt") == -1                            # no times
    assert L.fteik_h5io_finalizeF() == 0
    assert L.fteik_h5io_writeVelocityModelF(b"other") == -1                      # closed
    geo = (d / "Geometry.txt").read_text().split()
    assert [int(v) for v in geo[:3]] == [nz, nx, ny]
    L.fteik_model_free()


def test_host_switches_validate_and_round_trip(fk):
    """The speed switches of the grid search and the surrogate (host-side
    state only): invalid values are refused with ierr = 1 and leave the
    setting unchanged; valid ones read back."""
    from ctypes import byref, c_int
    L = fk.lib()
    old, ierr = c_int(), c_int(0)
    L.fteik_b200_locate_getRankingProducts(byref(old))
    assert old.value == 2                       # the default: tables split, events rounded once
    for bad in (0, 1, 4):
        L.fteik_b200_locate_setRankingProducts(bad, byref(ierr))
        assert ierr.value == 1
        v = c_int()
        L.fteik_b200_locate_getRankingProducts(byref(v))
        assert v.value == old.value
    for good in (3, 2):
        L.fteik_b200_locate_setRankingProducts(good, byref(ierr))
        assert ierr.value == 0
        v = c_int()
        L.fteik_b200_locate_getRankingProducts(byref(v))
        assert v.value == good
    for name in ("AsyncStaging", "FusedForward", "TrainGraph"):
        get, put = getattr(L, "fteik_b200_mlp_get" + name), getattr(L, "fteik_b200_mlp_set" + name)
        was = c_int()
        get(byref(was))
        assert was.value == 1                   # every speed path on by default
        put(0)
        v = c_int()
        get(byref(v))
        assert v.value == 0
        put(was.value)
