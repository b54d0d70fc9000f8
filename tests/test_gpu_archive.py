"""Travel-time datasets of the archive entry points (h5io.F90:263-347) from
fields solved on the GPU: the current 3D field in FP32 with x fastest, the
current 2D field flipped in z."""
import numpy as np
import pytest

from models import layered_grf_cells, linear_vz_cells

pytestmark = pytest.mark.gpu


def test_archive_travel_times_3d(fk, tmp_path):
    n, h = (9, 11, 8), (25.0, 25.0, 25.0)
    vel = layered_grf_cells(*n, seed=4, min_cells=2)
    s = fk.fteik3d()
    s.initialize(n[1], n[2], n[0], h[1], h[2], h[0], nsweep=2, eps=5.0, precision=8)
    s.setCellSlownessNatural(vel)
    s.setSources(101.0, 77.0, 66.0)
    L = fk.lib()
    assert L.fteik_h5io_initializeF(str(tmp_path / "a.h5").encode()) == 0
    assert L.fteik_h5io_writeTravelTimesF(b"t1") == -1          # nothing solved yet
    s.solveSourceLSM(1)
    assert L.fteik_h5io_writeTravelTimesF(b"t1") == 0
    got = np.load(tmp_path / "a.h5.d" / "TravelTimeFields" / "t1.npy")
    nat = s.getTravelTimeField().reshape(n[2], n[1], n[0])       # [y][x][z]
    assert got.dtype == np.float32 and got.shape == (n[0], n[2], n[1])
    assert np.array_equal(got, nat.transpose(2, 0, 1).astype(np.float32))
    assert L.fteik_h5io_finalizeF() == 0
    s.free()


def test_archive_travel_times_2d(fk, tmp_path):
    nz, nx, h = 21, 17, 10.0
    vel = linear_vz_cells(nz, nx, 2, h)[0]
    s = fk.fteik2d()
    s.initialize(nx, nz, h, h, nsweep=2, eps=5.0)
    s.setCellVelocityNatural(vel)
    s.setSources(55.0, 33.0)
    s.solveSourceLSM(1)
    L = fk.lib()
    assert L.fteik_h5io_initializeF(str(tmp_path / "b.hdf5").encode()) == 0
    assert L.fteik_h5io_writeTravelTimesF(b"t2") == 0
    got = np.load(tmp_path / "b.hdf5.d" / "TravelTimeFields" / "t2.npy")
    nat = s.getTravelTimeField().reshape(nx, nz)                 # [x][z]
    assert np.array_equal(got, nat.T[::-1].astype(np.float32))   # row 0 = the deepest nodes
    assert L.fteik_h5io_writeLevelSchedulesF() == -1             # 3D only, as the reference
    assert L.fteik_h5io_finalizeF() == 0
    s.free()
