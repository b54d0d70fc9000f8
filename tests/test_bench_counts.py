"""The counts behind bench.py's numbers, on the CPU.

* node updates per step (the metric's numerator) equal the oracle's count of
  the updates the reference evaluates (solver3D.F90:493-565 masked
  initialisation boxes plus nsweep full passes), source by source;
* the bench's source snap (source.F90:150-168) agrees with the oracle's;
* the algorithmic bytes of the roofline: 8 B per node and source (FP32 read
  and write) plus 4 B per cell per grid, per sweep: 27.9 GB per pass of 8
  sweeps on the 4-grid batch.
"""
import os
import sys

import numpy as np

import oracle_lib as O

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_node_updates_match_the_oracle_count():
    grids = bench.workload()
    for g in grids:
        n = (g["nz"], g["nx"], g["ny"])
        want = 0
        for k in range(bench.NSRC):
            si, _ = O.source_snap(True, n, (0.0, 0.0, 0.0), (bench.H,) * 3,
                                  (g["zs"][k], g["xs"][k], g["ys"][k]))
            assert si == (bench.snap1(n[0], bench.H, g["zs"][k]), bench.snap1(n[1], bench.H, g["xs"][k]),
                          bench.snap1(n[2], bench.H, g["ys"][k]))
            n_init, n_pass = O.count_updates3d(n, si)
            assert n_init == bench.init_updates3d(n, si)
            want += n_init + bench.NSWEEP * n_pass
        assert bench.node_updates(g) == want


def test_pass_bytes_are_the_batch_figure():
    grids = bench.workload()
    _, pass_b = bench.algorithmic_bytes(grids)
    ngrd = sum(nx * ny * nz for nx, ny, nz in bench.GRIDS)
    ncell = sum((nx - 1) * (ny - 1) * (nz - 1) for nx, ny, nz in bench.GRIDS)
    assert (ngrd, ncell) == (6758144, 6588880)
    per_pass = 8 * (8 * bench.NSRC * ngrd + 4 * ncell)
    assert per_pass == 27892201984                      # 27.9 GB
    assert pass_b == bench.NSWEEP * per_pass


def test_workload_is_the_batched_tables_configuration():
    grids = bench.workload()
    assert [(g["nx"], g["ny"], g["nz"]) for g in grids] == [(96, 96, 64), (128, 128, 80), (160, 160, 96),
                                                           (200, 120, 100)]
    for g in grids:
        assert np.all(g["zs"] == 0.0) and len(g["xs"]) == bench.NSRC
        zc = (np.arange(g["nz"] - 1) + 0.5) * bench.H
        assert np.allclose(g["vel"][0, 0, :], 3000.0 + 0.5 * zc)
