"""Tensor-core L2 search (locate method 1) against the CPU oracle.

* The raw accumulators equal an exact emulation of the BF16 hi+lo
  contraction (checks operand packing, swizzle and MMA descriptors).
* The located node equals the exhaustive FP64 search of the oracle, and t0 /
  misfit equal the oracle's FP64 values there.
* Events outside the tensor-core form (a skipped pick, unequal weights) fall
  back to the exact FP32 search and match it bit for bit.
"""
import numpy as np
import pytest

import oracle_lib as O
from models import station_tables, synthetic_events

pytestmark = pytest.mark.gpu


def _bf16(x32):
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    b = np.ascontiguousarray(x32, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def _split(d64):
    hi = _bf16(d64.astype(np.float32))
    lo = _bf16((d64 - hi.astype(np.float64)).astype(np.float32))
    return hi.astype(np.float64), lo.astype(np.float64)


def _locator(fk, tables, picks, wts=None):
    ntf, ngrd = tables.shape
    nev = picks.shape[0]
    loc = fk.Locator(nev, ntf, ngrd)
    for k in range(ntf):
        loc.setTravelTimeField32f(k + 1, tables[k])
    o2t = np.arange(1, ntf + 1)
    for e in range(nev):
        w = np.ones(ntf) if wts is None else wts[e]
        loc.setObservation(e + 1, o2t, picks[e], w)
    return loc


def _reduced(picks):
    return picks - picks.max(axis=1, keepdims=True)


@pytest.mark.parametrize("nprod,rank_tol", [(3, 4e-5), (2, 4e-3)])
def test_accumulators_match_bf16_emulation(fk, nprod, rank_tol):
    """The accumulator of event e at grid point g is the ranking score
    q(g) - 2 sum_i o'_i T'_i(g), formed from the bf16 splits: the products
    hi*hi + hi*lo + lo*hi (3), or hi*hi + hi*lo with the event side rounded
    to bf16 once (2, the default; its ranking error is the event side's
    rounding, about 2^-9 of the scale)."""
    tables = station_tables(16, 24, 20, 100.0, 64, seed=3)
    _, picks = synthetic_events(tables, 300, seed=4)
    loc = _locator(fk, tables, picks)
    loc.setMethod(1)
    old = loc.setRankingProducts(nprod)
    loc.debugAccumulators(True)
    loc.locateEvents(np.arange(1, 301))
    acc = loc.debugAccumulators(False).astype(np.float64)
    # CTA 0's first tile: events 0..255 x grid points 0..127
    T = tables[:, :128].astype(np.float64)
    Tp = T - T.mean(axis=0, keepdims=True)
    q = (Tp ** 2).sum(axis=0)
    q1 = _bf16(q.astype(np.float32)).astype(np.float64)
    q2 = _bf16((q - q1).astype(np.float32)).astype(np.float64)
    q3 = _bf16((q - q1 - q2).astype(np.float32)).astype(np.float64)
    o = _reduced(picks)[:256]
    op = -2.0 * (o - o.mean(axis=1, keepdims=True))
    ah, al = _split(op)
    bh, bl = _split(Tp.T)
    want = ah @ bh.T + ah @ bl.T + (al @ bh.T if nprod == 3 else 0.0) + (q1 + q2 + q3)[None, :]
    scale = np.abs(ah) @ np.abs(bh).T + q[None, :] + 1e-6
    err = np.abs(acc - want) / scale
    assert err.max() < 2e-6, f"max scaled error {err.max():.3g}"
    # the score ranks like the FP64 misfit: p + s = 2 obj (unit weights)
    p = (o - o.mean(axis=1, keepdims=True)) ** 2
    obj2 = p.sum(axis=1)[:, None] + acc
    res = o[:, :, None] - T[None, :, :]
    t0 = res.mean(axis=1, keepdims=True)
    want_obj2 = ((res - t0) ** 2).sum(axis=1)
    assert (np.abs(obj2 - want_obj2) / scale).max() < rank_tol
    loc.setRankingProducts(old)
    loc.finalize()


@pytest.mark.parametrize("shape,ntf,nev", [((16, 24, 20), 64, 300), ((13, 17, 11), 20, 37)])
def test_tc_matches_fp64_exhaustive(fk, shape, ntf, nev):
    tables = station_tables(*shape, 100.0, ntf, seed=7)
    _, picks = synthetic_events(tables, nev, seed=8)
    loc = _locator(fk, tables, picks)
    loc.setMethod(1)
    oi, t0, ob = loc.locateEvents(np.arange(1, nev + 1))
    red = _reduced(picks)
    tep = picks.max(axis=1)
    w = np.ones(ntf)
    miss = 0
    for e in range(nev):
        gi, gt0, gob = O.locate_l2_best64(tables, red[e], w)
        if oi[e] - 1 != gi:
            # only an exact FP64 tie may pick a different node
            _, _, ob_here = O.locate_l2_best64(tables[:, [oi[e] - 1]], red[e], w)
            if abs(ob_here - gob) > 1e-12 * max(gob, 1e-30):
                # report whether the miss repeats and how many events it hits
                oi2, _, ob2 = loc.locateEvents(np.arange(1, nev + 1))
                best = [O.locate_l2_best64(tables, red[k], w)[0] for k in range(nev)]
                bad = [k for k in range(nev) if oi[k] - 1 != best[k]]
                bad2 = [k for k in range(nev) if oi2[k] - 1 != best[k]]
                raise AssertionError(f"event {e}: got node {oi[e] - 1} (misfit {ob[e]!r}, oracle there "
                                     f"{ob_here!r}), oracle optimum {gi} ({gob!r}); events off: {bad}; "
                                     f"second call: node {oi2[e] - 1} ({ob2[e]!r}), events off {bad2}")
            miss += 1
            continue
        assert abs(t0[e] - (gt0 + tep[e])) <= 1e-9 * max(1.0, abs(gt0 + tep[e]))
        assert abs(ob[e] - gob) <= 1e-10 * max(gob, 1e-12)
    assert miss <= nev // 100
    loc.finalize()


def test_ineligible_events_use_exact_search(fk):
    tables = station_tables(12, 16, 14, 100.0, 32, seed=9)
    _, picks = synthetic_events(tables, 20, seed=10)
    wts = np.ones_like(picks)
    wts[3, 5] = 0.0          # a skipped pick
    wts[7, :] = 2.0          # uniform but not 1: still eligible
    wts[9, 2] = 0.5          # unequal weights
    loc = _locator(fk, tables, picks, wts)
    ev = np.arange(1, 21)
    oi0, t00, ob0 = loc.locateEvents(ev)
    loc.setMethod(1)
    oi1, t01, ob1 = loc.locateEvents(ev)
    for e in (3, 9):
        assert oi1[e] == oi0[e] and t01[e] == t00[e] and ob1[e] == ob0[e]
    red = _reduced(picks)
    gi, _, gob = O.locate_l2_best64(tables, red[7], wts[7])
    assert oi1[7] - 1 == gi and abs(ob1[7] - gob) <= 1e-10 * gob
    loc.finalize()


def test_tc_single_event_and_rescore_count(fk):
    tables = station_tables(10, 12, 9, 100.0, 16, seed=12)
    _, picks = synthetic_events(tables, 3, seed=13)
    loc = _locator(fk, tables, picks)
    loc.setMethod(1)
    loc.setRescoreCandidates(1)
    a = loc.locateEvent(2)
    loc.setRescoreCandidates(32)
    b = loc.locateEvent(2)
    gi, gt0, gob = O.locate_l2_best64(tables, _reduced(picks)[1], np.ones(16))
    assert b[0] - 1 == gi
    assert a[2] >= b[2]
    with pytest.raises(RuntimeError):
        loc.setMethod(5)
    loc.finalize()
