"""Writes tests/golden/fteik_golden.npz, the committed golden vectors.

The reference ships no fixtures and cannot be built here (Fortran), so the
vectors come from its two restatements:

* eikonal fields (3D level-set LSM, 2D LSM): the statement-by-statement
  Python transcription of the Fortran in tests/test_oracle_levelset.py,
  which agrees bit for bit with the C oracle;
* grid-search location: the C oracle's FP32 restatement of locate.F90 (the
  reference's operation order, first-index MINLOC), its FP64 exhaustive L2
  search and its FP64 L1 (median origin time) search, on analytic
  constant-velocity tables as in testing/loctest.c:21-169.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle_lib as O                       # noqa: E402
import test_oracle_levelset as T             # noqa: E402
from models import layered_grf_cells         # noqa: E402

OUT = os.path.join(HERE, "fteik_golden.npz")

# 3D cases: (n = (nz, nx, ny), h = (dz, dx, dy), source (z, x, y), eps, nsweep, seed)
CASES3 = [
    ((12, 11, 10), (25.0, 25.0, 25.0), (141.3, 121.9, 150.2), 5.0, 2, 50),
    ((10, 12, 9), (20.0, 30.0, 25.0), (0.0, 170.5, 110.1), 3.0, 2, 51),    # surface nudge
    ((9, 9, 9), (40.0, 40.0, 40.0), (319.0, 10.0, 310.0), 2.0, 3, 52),     # last cells
    ((11, 10, 12), (30.0, 30.0, 30.0), (150.0, 120.0, 180.0), 5.0, 1, 53),  # on a node
]
# 2D cases: (n = (nz, nx), h = (dz, dx), source (z, x), eps, nsweep, seed)
CASES2 = [
    ((21, 23), (10.0, 10.0), (91.3, 123.7), 5.0, 2, 60),
    ((17, 19), (20.0, 15.0), (0.0, 140.0), 3.0, 2, 61),
    ((15, 16), (10.0, 10.0), (140.0, 150.0), 2.0, 3, 62),
]


def vel3(n, seed):
    """Layered model (3000..6000 m/s) times (1 + 0.05 GRF), cells z fastest."""
    return np.ascontiguousarray(layered_grf_cells(*n, seed=seed, min_cells=1, corr=3.0)).ravel()


def vel2(n, h, seed):
    """v = 3000 + 2 z_c m/s times (1 + 0.05 white noise), cells z fastest."""
    nz, nx = n
    rng = np.random.default_rng(seed)
    zc = (np.arange(nz - 1) + 0.5) * h[0]
    v = (3000.0 + 2.0 * zc)[:, None] * (1.0 + 0.05 * rng.standard_normal((nz - 1, nx - 1)))
    return np.ascontiguousarray(v.ravel(order="F"))


def locate_problem():
    """Constant 5 km/s medium on a 12 x 11 x 10 grid (h = 1 km), 10 surface
    stations, 12 events at grid nodes with origin times in [0, 60) s, picks
    with 0.02 s noise, one outlier pick (+-0.5 s) per event, a skipped pick
    (weight 0) in every third event, picks given in a permuted order."""
    nz, nx, ny, h, v, nsta = 12, 11, 10, 1000.0, 5000.0, 10
    rng = np.random.default_rng(70)
    sx = rng.uniform(0, (nx - 1) * h, nsta)
    sy = rng.uniform(0, (ny - 1) * h, nsta)
    iz, ix, iy = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    z = (iz * h).transpose(2, 1, 0).ravel()           # z fastest
    x = (ix * h).transpose(2, 1, 0).ravel()
    y = (iy * h).transpose(2, 1, 0).ravel()
    tables = np.stack([np.sqrt(z ** 2 + (x - sx[k]) ** 2 + (y - sy[k]) ** 2) / v
                       for k in range(nsta)]).astype(np.float32)
    nev = 12
    true = rng.integers(0, nz * nx * ny, nev)
    picks, wts, o2t = [], [], []
    for e in range(nev):
        p = tables[:, true[e]].astype(np.float64) + rng.uniform(0, 60) + rng.normal(0, 0.02, nsta)
        p[rng.integers(0, nsta)] += rng.choice([-0.5, 0.5])
        w = np.ones(nsta)
        if e % 3 == 2:
            w[rng.integers(0, nsta)] = 0.0
        perm = rng.permutation(nsta)
        picks.append(p[perm])
        wts.append(w[perm])
        o2t.append(perm + 1)
    return tables, np.array(picks), np.array(wts), np.array(o2t, np.int32), true


def reduce_event(ntf, picks, wts, o2t):
    """locate.F90:431-497: picks relative to the latest pick, FP64 per table
    (weight 0 = skipped)."""
    tepoch = np.max(picks)
    obs64, w64 = np.zeros(ntf), np.zeros(ntf)
    for i, k in enumerate(o2t - 1):
        if wts[i] > 0:
            obs64[k] = picks[i] - tepoch
            w64[k] = wts[i]
    return tepoch, obs64, w64


def main():
    out = {}
    for c, (n, h, src, eps, nsweep, seed) in enumerate(CASES3):
        v = vel3(n, seed)
        tt, _, _ = T.solve3(n, h, list(1.0 / v), src, eps, nsweep)
        out.update({f"s3_{c}_n": np.array(n), f"s3_{c}_h": np.array(h),
                    f"s3_{c}_src": np.array(src), f"s3_{c}_eps": eps, f"s3_{c}_nsweep": nsweep,
                    f"s3_{c}_vel": v, f"s3_{c}_tt": tt})
    for c, (n, h, src, eps, nsweep, seed) in enumerate(CASES2):
        v = vel2(n, h, seed)
        tt, _, _ = T.solve2(n, h, list(1.0 / v), src, eps, nsweep)
        out.update({f"s2_{c}_n": np.array(n), f"s2_{c}_h": np.array(h),
                    f"s2_{c}_src": np.array(src), f"s2_{c}_eps": eps, f"s2_{c}_nsweep": nsweep,
                    f"s2_{c}_vel": v, f"s2_{c}_tt": tt})
    tables, picks, wts, o2t, true = locate_problem()
    ntf = tables.shape[0]
    l2_32, l2_64, l1_64 = [], [], []
    for e in range(picks.shape[0]):
        tepoch, obs64, w64 = reduce_event(ntf, picks[e], wts[e], o2t[e])
        skip = (w64 <= 0).astype(np.uint8)
        # O.locate_l2 returns the reference's 1-based optIndx and FP32 t0 / misfit
        i32, t32, o32 = O.locate_l2(tables, obs64.astype(np.float32), w64.astype(np.float32), skip)
        l2_32.append((i32, float(np.float32(t32)) + tepoch, float(np.float32(o32))))
        i, t, o = O.locate_l2_best64(tables, obs64, w64)     # 0-based index
        l2_64.append((i + 1, t + tepoch, o))
        i, t, o = O.locate_l1_best64(tables, obs64, w64)
        l1_64.append((i + 1, t + tepoch, o))
    out.update({"loc_tables": tables, "loc_picks": picks, "loc_wts": wts, "loc_obs2tf": o2t,
                "loc_true": true + 1, "loc_l2_fp32": np.array(l2_32),
                "loc_l2_fp64": np.array(l2_64), "loc_l1_fp64": np.array(l1_64)})
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
