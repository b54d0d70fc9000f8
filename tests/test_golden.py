"""The C oracle against the committed golden vectors (tests/golden/).

The eikonal fields there were written by the statement-by-statement Python
transcription of the reference (test_oracle_levelset.py), the location
results by the oracle itself (tests/golden/make_golden.py).  The oracle
must reproduce the fields bit for bit and the location results exactly
(FP32 search) or to the last few ulp (FP64 searches, whose reductions
run over OpenMP threads).
"""
import os

import numpy as np
import pytest

import oracle_lib as O

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                            "fteik_golden.npz"))
N3 = len([k for k in GOLD.files if k.startswith("s3_") and k.endswith("_tt")])
N2 = len([k for k in GOLD.files if k.startswith("s2_") and k.endswith("_tt")])


def case3(c):
    g = lambda k: GOLD[f"s3_{c}_{k}"]  # noqa: E731
    return (tuple(int(v) for v in g("n")), tuple(float(v) for v in g("h")),
            tuple(float(v) for v in g("src")), float(g("eps")), int(g("nsweep")), g("vel"), g("tt"))


def case2(c):
    g = lambda k: GOLD[f"s2_{c}_{k}"]  # noqa: E731
    return (tuple(int(v) for v in g("n")), tuple(float(v) for v in g("h")),
            tuple(float(v) for v in g("src")), float(g("eps")), int(g("nsweep")), g("vel"), g("tt"))


def reduce_event(ntf, picks, wts, o2t):
    """locate.F90:431-497: picks relative to the latest pick, per table."""
    tepoch = np.max(picks)
    obs64, w64 = np.zeros(ntf), np.zeros(ntf)
    for i, k in enumerate(o2t - 1):
        if wts[i] > 0:
            obs64[k] = picks[i] - tepoch
            w64[k] = wts[i]
    return tepoch, obs64, w64


def test_fixture_counts():
    assert N3 >= 4 and N2 >= 3


@pytest.mark.parametrize("c", range(4))
def test_oracle_3d_reproduces_golden(c):
    n, h, src, eps, nsweep, vel, tt = case3(c)
    si, sa = O.source_snap(True, n, (0.0, 0.0, 0.0), h, src)
    for level_set in (False, True):
        got, _ = O.solve3d(n, h, 1.0 / vel, si, sa, eps, nsweep, level_set=level_set, nthreads=2)
        np.testing.assert_array_equal(got, tt)


@pytest.mark.parametrize("c", range(3))
def test_oracle_2d_reproduces_golden(c):
    n, h, src, eps, nsweep, vel, tt = case2(c)
    si, sa = O.source_snap(False, (n[0], n[1], 1), (0.0, 0.0, 0.0), (h[0], h[1], 1.0),
                           (src[0], src[1], 0.0))
    got, _ = O.solve2d(n, h, 1.0 / vel, si[:2], sa[:2], eps, nsweep)
    np.testing.assert_array_equal(got, tt)


def test_oracle_locate_reproduces_golden():
    tables = GOLD["loc_tables"]
    picks, wts, o2t = GOLD["loc_picks"], GOLD["loc_wts"], GOLD["loc_obs2tf"]
    ntf = tables.shape[0]
    for e in range(picks.shape[0]):
        tepoch, obs64, w64 = reduce_event(ntf, picks[e], wts[e], o2t[e])
        skip = (w64 <= 0).astype(np.uint8)
        i32, t32, o32 = O.locate_l2(tables, obs64.astype(np.float32), w64.astype(np.float32), skip)
        want = GOLD["loc_l2_fp32"][e]
        assert i32 == int(want[0])
        assert float(np.float32(t32)) + tepoch == want[1] and float(np.float32(o32)) == want[2]
        for fn, key in ((O.locate_l2_best64, "loc_l2_fp64"), (O.locate_l1_best64, "loc_l1_fp64")):
            i, t, o = fn(tables, obs64, w64)
            want = GOLD[key][e]
            assert i + 1 == int(want[0])
            assert abs(t + tepoch - want[1]) <= 1e-12 * abs(want[1])
            assert abs(o - want[2]) <= 1e-12 * abs(want[2])


def test_l1_is_robust_to_the_outlier_pick():
    """Each event has one pick off by 0.5 s: the L1 optima stay within three
    nodes of the true hypocentres (surface stations resolve depth poorly)
    and closer on average than the L2 optima, which the outlier pulls."""
    def zxy(i):
        i = int(i) - 1
        return np.array([i % 12, (i // 12) % 11, i // 132])
    d1 = [np.abs(zxy(a) - zxy(b)).max() for a, b in zip(GOLD["loc_l1_fp64"][:, 0], GOLD["loc_true"])]
    d2 = [np.abs(zxy(a) - zxy(b)).max() for a, b in zip(GOLD["loc_l2_fp64"][:, 0], GOLD["loc_true"])]
    assert max(d1) <= 3 and np.mean(d1) < 0.7 * np.mean(d2)
