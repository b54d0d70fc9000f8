"""Grid-search location on the GPU against the FP32 CPU restatement of
locate.F90 (bit-identical optimum, origin time and misfit)."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


def _problem(seed, ntf=12, ngrd=40000, nev=5):
    rng = np.random.default_rng(seed)
    tables = rng.uniform(0.5, 12.0, size=(ntf, ngrd)).astype(np.float32)
    true = rng.integers(0, ngrd, nev)
    events = []
    for e in range(nev):
        t0 = rng.uniform(0, 60)
        picks = tables[:, true[e]].astype(np.float64) + t0 + rng.normal(0, 0.02, ntf)
        wts = np.ones(ntf)
        wts[rng.integers(0, ntf)] = 0.0                      # a skipped pick
        order = rng.permutation(ntf)                         # obs2tf mapping
        events.append((order + 1, picks[order], wts[order]))
    return tables, events


def _oracle_event(tables, obs2tf, picks, wts):
    ntf = tables.shape[0]
    tepoch = np.max(picks)
    obs = np.zeros(ntf, np.float32)
    w = np.zeros(ntf, np.float32)
    skip = np.ones(ntf, np.uint8)
    for i, k in enumerate(obs2tf - 1):
        if wts[i] > 0:
            obs[k] = np.float32(picks[i] - tepoch)
            w[k] = np.float32(wts[i])
            skip[k] = 0
    idx, t0, obj = O.locate_l2(tables, obs, w, skip)
    return idx, float(t0) + tepoch, float(obj)


def test_locate_matches_oracle_bitwise(fk):
    tables, events = _problem(1)
    loc = fk.Locator(len(events), tables.shape[0], tables.shape[1])
    for k in range(tables.shape[0]):
        if k % 2:
            loc.setTravelTimeField32f(k + 1, tables[k])
        else:
            loc.setTravelTimeField64f(k + 1, tables[k].astype(np.float64))
    for e, (o2t, picks, wts) in enumerate(events, start=1):
        loc.setObservation(e, o2t, picks, wts)
    oi, t0, ob = loc.locateEvents(np.arange(1, len(events) + 1))
    for e, (o2t, picks, wts) in enumerate(events, start=1):
        want = _oracle_event(tables, o2t, picks, wts)
        single = loc.locateEvent(e)
        assert single[0] == want[0] and oi[e - 1] == want[0]
        assert single[1] == want[1] and t0[e - 1] == want[1]
        assert single[2] == want[2] and ob[e - 1] == want[2]
    loc.finalize()


def test_locate_ties_take_first_index(fk):
    tables = np.tile(np.linspace(1, 2, 8, dtype=np.float32)[:, None], (1, 1000))
    loc = fk.Locator(1, 8, 1000)
    for k in range(8):
        loc.setTravelTimeField32f(k + 1, tables[k])
    loc.setObservation(1, np.arange(1, 9), tables[:, 0].astype(np.float64) + 3.0, np.ones(8))
    assert loc.locateEvent(1)[0] == 1
    loc.finalize()


def test_batch_tables_hand_off_to_locator(fk):
    nz, nx, ny, h = 12, 13, 11, 50.0
    from models import linear_vz_cells
    vel = linear_vz_cells(nz, nx, ny, h)
    b = fk.Batch3D([(nz, nx, ny, h, h, h)], nsweep=2, precision=4)
    b.setVelocityModel(1, vel)
    rng = np.random.default_rng(3)
    zs = np.zeros(6)
    xs = rng.uniform(0, (nx - 1) * h, 6)
    ys = rng.uniform(0, (ny - 1) * h, 6)
    b.setSources(1, zs, xs, ys)
    b.solve()
    ngrd = nz * nx * ny
    loc = fk.Locator(1, 6, ngrd)
    b.exportToLocator(1, 1)
    f32 = b.fields32(1).reshape(6, ngrd)
    true = 777
    picks = f32[:, true].astype(np.float64) + 10.0
    loc.setObservation(1, np.arange(1, 7), picks, np.ones(6))
    idx, t0, obj = loc.locateEvent(1)
    want = O.locate_l2(f32, (picks - picks.max()).astype(np.float32), np.ones(6, np.float32),
                       np.zeros(6, np.uint8))
    assert idx == want[0] == true + 1
    b.finalize()
    loc.finalize()
