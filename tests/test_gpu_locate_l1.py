"""L1 grid search (locate norm 1) against the FP64 exhaustive L1 search of the
CPU oracle.  The reference has no L1 misfit (parity is measured against the FP64
search only)."""
import numpy as np
import pytest

import oracle_lib as O
from models import station_tables, synthetic_events

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ntf", [12, 32, 64])
def test_l1_matches_fp64_exhaustive(fk, ntf):
    tables = station_tables(14, 18, 16, 100.0, ntf, seed=ntf)
    nev = 24
    _, picks = synthetic_events(tables, nev, seed=ntf + 1)
    wts = np.full(picks.shape, 2.0)
    wts[3, 1] = 0.0                     # skipped picks
    wts[5, :4] = 0.0
    loc = fk.Locator(nev, ntf, tables.shape[1])
    for k in range(ntf):
        loc.setTravelTimeField32f(k + 1, tables[k])
    o2t = np.arange(1, ntf + 1)
    for e in range(nev):
        loc.setObservation(e + 1, o2t, picks[e], wts[e])
    loc.setNorm(1)
    oi, t0, ob = loc.locateEvents(np.arange(1, nev + 1))
    for e in range(nev):
        red = picks[e] - picks[e].max()
        gi, gt0, gob = O.locate_l1_best64(tables, red, wts[e])
        # the GPU ranks in FP32: a different node only within FP32 rounding of the minimum
        _, t_here, ob_here = O.locate_l1_best64(tables[:, [oi[e] - 1]], red, wts[e])
        assert ob_here <= gob * (1 + 2e-6) + 1e-9, (e, oi[e] - 1, gi, ob_here, gob)
        assert abs(ob[e] - ob_here) <= 1e-9 * max(ob_here, 1e-12)
        assert abs(t0[e] - (t_here + picks[e].max())) <= 1e-9 * max(1.0, abs(t0[e]))
    loc.finalize()


def test_l1_rejects_unequal_weights(fk):
    tables = station_tables(8, 9, 10, 100.0, 8, seed=4)
    _, picks = synthetic_events(tables, 2, seed=5)
    loc = fk.Locator(2, 8, tables.shape[1])
    for k in range(8):
        loc.setTravelTimeField32f(k + 1, tables[k])
    w = np.ones(8)
    w[2] = 3.0
    loc.setObservation(1, np.arange(1, 9), picks[0], w)
    loc.setObservation(2, np.arange(1, 9), picks[1], np.ones(8))
    loc.setNorm(1)
    assert loc.locateEvent(2)[0] > 0
    with pytest.raises(RuntimeError):
        loc.locateEvents(np.array([1, 2]))
    loc.finalize()
