"""The GPU library, through the reference-facing C ABI, against the committed
golden vectors (tests/golden/fteik_golden.npz; see tests/golden/make_golden.py
for how they were made).

* 3D and 2D fields in FP64: within 1e-12 of the largest time;
* 3D fields in FP32 (the product precision): 1e-4 relative (1e-3 for the
  source exactly on a node, where exact FP64 ties between upwind stencils
  break differently in FP32);
* locate, exact FP32 search (the drop-in default): optimum, origin time
  and misfit bit-identical;
* locate, tensor-core search: the FP64 exhaustive optimum, t0 and misfit to
  1e-9 relative for events with every pick at one weight, the exact FP32
  result for the others;
* locate, L1 norm: the FP64 exhaustive L1 optimum, t0 and misfit to 1e-9.
"""
import numpy as np
import pytest

from test_golden import GOLD, case2, case3

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [8, 4])
@pytest.mark.parametrize("c", range(4))
def test_gpu_3d_golden(fk, c, precision):
    n, h, src, eps, nsweep, vel, tt = case3(c)
    s = fk.fteik3d()
    s.initialize(n[1], n[2], n[0], h[1], h[2], h[0], nsweep=nsweep, eps=eps, precision=precision)
    s.setCellSlownessNatural(vel)
    s.setSources(src[1], src[2], src[0])
    s.solveSourceLSM(1)
    got = s.getTravelTimeField()
    s.free()
    if precision == 8:
        assert np.max(np.abs(got - tt)) <= 1e-12 * np.max(tt)
    else:
        assert np.max(np.abs(got - tt) / np.maximum(tt, 1e-6)) <= 1e-4


@pytest.mark.parametrize("c", range(3))
def test_gpu_2d_golden(fk, c):
    n, h, src, eps, nsweep, vel, tt = case2(c)
    s = fk.fteik2d()
    s.initialize(n[1], n[0], h[1], h[0], nsweep=nsweep, eps=eps)
    s.setCellVelocityNatural(vel)
    s.setSources(src[1], src[0])
    s.solveSourceLSM(1)
    got = s.getTravelTimeField()
    s.free()
    assert np.max(np.abs(got - tt)) <= 1e-12 * np.max(tt)


def _locator(fk):
    tables = GOLD["loc_tables"]
    picks, wts, o2t = GOLD["loc_picks"], GOLD["loc_wts"], GOLD["loc_obs2tf"]
    nev, ntf = picks.shape[0], tables.shape[0]
    loc = fk.Locator(nev, ntf, tables.shape[1])
    for k in range(ntf):
        loc.setTravelTimeField32f(k + 1, tables[k])
    for e in range(nev):
        loc.setObservation(e + 1, o2t[e], picks[e], wts[e])
    return loc, np.arange(1, nev + 1)


def _close(a, b, rel=1e-9):
    return abs(a - b) <= rel * max(abs(b), 1e-12)


def test_gpu_locate_exact_golden(fk):
    loc, ev = _locator(fk)
    oi, t0, ob = loc.locateEvents(ev)
    want = GOLD["loc_l2_fp32"]
    assert np.array_equal(oi, want[:, 0].astype(int))
    assert np.array_equal(t0, want[:, 1]) and np.array_equal(ob, want[:, 2])
    loc.finalize()


def test_gpu_locate_tensor_core_golden(fk):
    loc, ev = _locator(fk)
    loc.setMethod(1)
    oi, t0, ob = loc.locateEvents(ev)
    one_weight = np.all(GOLD["loc_wts"] > 0, axis=1)
    for e in range(len(ev)):
        want = GOLD["loc_l2_fp64"][e] if one_weight[e] else GOLD["loc_l2_fp32"][e]
        assert oi[e] == int(want[0]), e
        if one_weight[e]:
            assert _close(t0[e], want[1]) and _close(ob[e], want[2]), e
        else:
            assert t0[e] == want[1] and ob[e] == want[2], e
    loc.finalize()


def test_gpu_locate_l1_golden(fk):
    loc, ev = _locator(fk)
    loc.setNorm(1)
    oi, t0, ob = loc.locateEvents(ev)
    want = GOLD["loc_l1_fp64"]
    assert np.array_equal(oi, want[:, 0].astype(int))
    for e in range(len(ev)):
        assert _close(t0[e], want[e, 1]) and _close(ob[e], want[e, 2]), e
    loc.finalize()
