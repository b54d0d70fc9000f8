"""Launch configurations of the 3D slab sweeps (fteik_b200_setSlabConfig):
the staged FP32 pass step (16-byte cp.async groups through shared memory),
one or two sources per thread, progress every 8 or 32 steps, 1 to 4
resident blocks per SM.  Each changes only how the same node updates are
scheduled and loaded, so every configuration gives the default's FP32
fields bit for bit -- single source and batch, fixed passes and solves to
convergence -- on grids whose depth takes every leading-item offset of the
staged step's descending sweeps (nz mod 4 = 0..3), shallower and deeper than
32, deep enough to need the opt-in shared memory, and wider than one
32-column block.  No counterpart in the reference."""
import numpy as np
import pytest

from models import interior_source, layered_grf_cells

pytestmark = pytest.mark.gpu

CONFIGS = [(1, 1, -1, -1), (1, 0, 8, -1), (1, 1, 32, 2), (0, 0, 32, 1), (1, 1, 8, 4)]
SHAPES = {            # nz, nx, ny
    "nz23": (23, 19, 17),
    "nz30_wide": (30, 70, 13),
    "nz12": (12, 14, 13),
    "nz45": (45, 40, 10),
    "nz9_wide": (9, 70, 11),
    "nz150_deep": (150, 20, 9),   # rings + stage + static arrays above the default 48 KB
}


def _solve_single(fk, n, h, vel, src, cfg):
    old = fk.set_slab_config(*cfg)
    try:
        s = fk.fteik3d()
        s.initialize(n[1], n[2], n[0], h[1], h[2], h[0], nsweep=2, eps=5.0, precision=4)
        s.setCellSlownessNatural(vel)
        s.setSources(src[1], src[2], src[0])
        s.solveSourceLSM(1)
        tt = s.getTravelTimeField()
        s.free()
    finally:
        fk.set_slab_config(*old)
    return tt


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_single_source_configs_same_bits(fk, shape):
    n = SHAPES[shape]
    h = (25.0, 20.0, 30.0)
    vel = layered_grf_cells(*n, seed=sum(n), min_cells=2)
    src = interior_source(n, h, n[0])
    ref = _solve_single(fk, n, h, vel, src, (-1, -1, -1, -1))
    for cfg in CONFIGS:
        got = _solve_single(fk, n, h, vel, src, cfg)
        assert np.array_equal(got, ref), cfg


def _batch(fk, grids, srcs, vels, cfg, **kw):
    old = fk.set_slab_config(*cfg)
    try:
        b = fk.Batch3D(grids, precision=4, eps=5.0, **kw)
        for ig in range(len(grids)):
            b.setVelocityModel(ig + 1, vels[ig])
            z, x, y = srcs[ig]
            b.setSources(ig + 1, z, x, y)
        b.solve()
        out = [b.fields32(ig + 1).copy() for ig in range(len(grids))]
        info = [b.solveInfo(ig + 1, 1) for ig in range(len(grids))]
        b.finalize()
    finally:
        fk.set_slab_config(*old)
    return out, info


def _batch_case():
    grids = [(23, 40, 12, 25.0, 25.0, 25.0), (30, 17, 15, 30.0, 20.0, 25.0), (12, 33, 9, 20.0, 20.0, 20.0)]
    rng = np.random.default_rng(7)
    srcs, vels = [], []
    for ig, (nz, nx, ny, dz, dx, dy) in enumerate(grids):
        k = 3 if ig != 1 else 2                        # odd source counts walk one source alone
        z = rng.uniform(0, (nz - 1) * dz, k)
        z[0] = 0.0                                     # a surface source (the on-node nudge)
        srcs.append((z, rng.uniform(0, (nx - 1) * dx, k), rng.uniform(0, (ny - 1) * dy, k)))
        vels.append(layered_grf_cells(nz, nx, ny, seed=60 + ig, min_cells=2))
    return grids, srcs, vels


def test_batch_configs_same_bits(fk):
    grids, srcs, vels = _batch_case()
    ref, _ = _batch(fk, grids, srcs, vels, (-1, -1, -1, -1), nsweep=2)
    for cfg in CONFIGS:
        got, _ = _batch(fk, grids, srcs, vels, cfg, nsweep=2)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b), cfg


def test_batch_converged_configs_same_bits(fk):
    """Passes to convergence (the FP64 residual compiled into the pass
    kernel): the same fields and the same pass counts."""
    grids, srcs, vels = _batch_case()
    ref, rinfo = _batch(fk, grids, srcs, vels, (-1, -1, -1, -1), convTol=0.0, maxPass=25)
    for cfg in CONFIGS[:3]:
        got, info = _batch(fk, grids, srcs, vels, cfg, convTol=0.0, maxPass=25)
        assert info == rinfo, cfg
        for a, b in zip(ref, got):
            assert np.array_equal(a, b), cfg


def _timed(fk, b, k=5):
    import torch
    stream = torch.cuda.ExternalStream(fk.lib().fteik_b200_stream())
    for _ in range(2):
        b.solveAsync()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(3):
        e0.record(stream)
        for _ in range(k):
            b.solveAsync()
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / k)
    return best


@pytest.mark.parametrize("kind", ["batch", "one_grid"])
def test_tuned_configuration_not_slower_than_fixed(fk, kind, tmp_path, monkeypatch):
    """The configuration the batch picks by timing (knobs at -1) is not
    slower than the fixed configuration the library ran before it had a
    tuner (direct loads, source pairs, progress step by task count, all
    resident blocks), on a multi-grid batch and on one grid; the choice goes
    to the cache file, and a second batch of the same work list reuses it
    instead of searching again."""
    monkeypatch.setenv("FTEIK_B200_TUNE_CACHE", str(tmp_path / "tune.txt"))
    if kind == "batch":
        grids = [(48, 96, 64, 50.0, 50.0, 50.0), (64, 80, 72, 50.0, 50.0, 50.0)]
        nsrc = 16
    else:
        grids = [(64, 128, 96, 50.0, 50.0, 50.0)]
        nsrc = 1
    rng = np.random.default_rng(5)

    def make():
        b = fk.Batch3D(grids, nsweep=2, eps=5.0, precision=4)
        for ig, (nz, nx, ny, dz, dx, dy) in enumerate(grids, start=1):
            b.setVelocityModel(ig, layered_grf_cells(nz, nx, ny, seed=ig, min_cells=3))
            r = np.random.default_rng(ig)
            b.setSources(ig, np.zeros(nsrc), r.uniform(0, (nx - 1) * dx, nsrc), r.uniform(0, (ny - 1) * dy, nsrc))
        return b

    old = fk.set_slab_config(0, 1, 0, 0)
    try:
        b = make()
        b.solve()
        fixed = _timed(fk, b)
        f_fixed = [b.fields32(ig + 1).copy() for ig in range(len(grids))]
        b.finalize()
    finally:
        fk.set_slab_config(*old)
    fk.set_slab_config(-1, -1, -1, -1)
    b = make()
    b.solve()
    cfg = b.slabConfig()
    tuned = _timed(fk, b)
    assert cfg["tune_runs"] > 0
    for ig in range(len(grids)):
        assert np.array_equal(b.fields32(ig + 1), f_fixed[ig])
    b.finalize()
    assert tuned <= fixed * 1.03, (tuned, fixed, cfg)
    b = make()
    b.solve()
    again = b.slabConfig()
    b.finalize()
    assert again["tune_runs"] == 0
    assert (tmp_path / "tune.txt").read_text().count("\n") >= 1
    keys = ("staged", "pairs", "progress", "blocks_per_sm", "init_blocks_per_sm", "init_pairs")
    assert [again[k] for k in keys] == [cfg[k] for k in keys]
