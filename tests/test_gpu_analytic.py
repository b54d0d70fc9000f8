"""Analytic module (analytic.F90) on the GPU against the CPU restatement."""
import ctypes

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["const", "linear"])
def test_analytic_fields(fk, kind):
    L = fk.lib()
    PD = ctypes.POINTER(ctypes.c_double)
    ierr = ctypes.c_int(1)
    nz, nx, ny, h = 11, 13, 9, 25.0
    L.fteik_analytic_initialize64f(nz, nx, ny, 0.0, 0.0, 0.0, h, h, h, 0, ctypes.byref(ierr))
    assert ierr.value == 0
    z, x, y = np.array([55.5]), np.array([101.0]), np.array([77.0])
    L.fteik_analytic_setSources64f(1, z.ctypes.data_as(PD), x.ctypes.data_as(PD), y.ctypes.data_as(PD),
                                   ctypes.byref(ierr))
    assert ierr.value == 0
    if kind == "const":
        L.fteik_analytic_setConstantVelocity64f(3500.0, ctypes.byref(ierr))
        L.fteik_analytic_solveSourceConstantVelocity64f(1, ctypes.byref(ierr))
        ref = O.analytic_constant((nz, nx, ny), (0, 0, 0), (h, h, h), 3500.0, (55.5, 101.0, 77.0))
    else:
        L.fteik_analytic_setLinearVelocityGradient64f(3000.0, 5000.0, ctypes.byref(ierr))
        L.fteik_analytic_solveSourceLinearVelocityGradient64f(1, ctypes.byref(ierr))
        ref = O.analytic_linear((nz, nx, ny), (0, 0, 0), (h, h, h), 3000.0, 5000.0, (55.5, 101.0, 77.0))
    assert ierr.value == 0
    out = np.zeros(nz * nx * ny)
    L.fteik_analytic_getTravelTimeField64f(out.size, 0, out.ctypes.data_as(PD), ctypes.byref(ierr))
    assert ierr.value == 0
    assert np.allclose(out, ref, rtol=1e-13, atol=1e-15)
    L.fteik_analytic_free()
