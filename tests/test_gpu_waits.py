"""Bounded device-side waits of the 3D sweeps (no counterpart in the
reference, whose OpenMP barriers wait without a limit).

A slab of the persistent sweep kernels waits on its upwind slab and on its
neighbours' previous sweep with a poll limit.  With the limit set to 0 the
first wait that is not already satisfied gives up: the kernel sets its error
word and returns, the solve reports ierr = 1, and the next solve with the
default limit runs normally.  Nothing faults or hangs on the way: the waits
return, and the blocks that have not started a task stop claiming tasks once
the error word is set.
"""
import numpy as np
import pytest

import oracle_lib as O
from models import interior_source, layered_grf_cells

pytestmark = pytest.mark.gpu

# 16 slabs of 4 y-rows: a slab's first wait on its upwind neighbour cannot
# already be satisfied for every one of the 16 x 24 slab sweeps
N = (40, 70, 64)
H = (25.0, 25.0, 25.0)


def _model():
    vel = layered_grf_cells(*N, seed=4, min_cells=3)
    return vel, interior_source(N, H, 12)


def _oracle(vel, src, nsweep):
    si, sa = O.source_snap(True, N, (0, 0, 0), H, src)
    tt, _ = O.solve3d(N, H, 1.0 / np.ravel(vel), si, sa, 5.0, nsweep)
    return tt


def test_single_source_wait_runs_out_then_recovers(fk):
    vel, src = _model()
    s = fk.fteik3d()
    s.initialize(N[1], N[2], N[0], H[1], H[2], H[0], nsweep=2, eps=5.0, precision=8)
    s.setCellSlownessNatural(vel)
    s.setSources(src[1], src[2], src[0])
    old = fk.set_spin_limit(0)
    try:
        with pytest.raises(fk.FteikError):
            s.solveSourceLSM(1)
    finally:
        fk.set_spin_limit(old)
    s.solveSourceLSM(1)
    tt = s.getTravelTimeField()
    ref = _oracle(vel, src, 2)
    assert np.max(np.abs(tt - ref)) <= 1e-12 * np.max(ref)
    s.free()


def test_batch_wait_runs_out_then_recovers(fk):
    vel, _ = _model()
    rng = np.random.default_rng(3)
    z = rng.uniform(0.1, 0.9, 4) * (N[0] - 1) * H[0]
    x = rng.uniform(0.1, 0.9, 4) * (N[1] - 1) * H[1]
    y = rng.uniform(0.1, 0.9, 4) * (N[2] - 1) * H[2]
    b = fk.Batch3D([(N[0], N[1], N[2], *H)], nsweep=2, eps=5.0, precision=4)
    b.setVelocityModel(1, vel)
    b.setSources(1, z, x, y)
    b.solve()                               # graph captured with the default limit
    old = fk.set_spin_limit(0)
    try:
        with pytest.raises(fk.FteikError):
            b.solve()                       # rebuilt with limit 0
    finally:
        fk.set_spin_limit(old)
    b.solve()                               # rebuilt with the default again
    for k in range(4):
        ref = _oracle(vel, (z[k], x[k], y[k]), 2)
        got = b.field(1, k + 1)
        assert np.max(np.abs(got - ref) / np.maximum(ref, 1e-6)) <= 1e-4
    b.finalize()
