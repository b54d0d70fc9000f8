"""The allocation-free grid search (fteik_b200_locate_l2_noalloc) against the
library's regular locator, through the C ABI.

Callers that cannot let a library allocate device memory pass their own
device buffers; the entry point keeps its per-event scratch in a fixed
device array.  The test runs it twice in a row on different events (the
array keeps the previous call's contents, which must not leak into the next
call) and checks the optimum index, origin time and misfit against the
regular entry point, which must agree exactly (same FP32 arithmetic).
This file is named to run last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(seed, ntf, ngrd, nev):
    rng = np.random.default_rng(seed)
    tables = rng.uniform(0.5, 12.0, size=(ntf, ngrd)).astype(np.float32)
    picks = np.empty((nev, ntf))
    wts = np.ones((nev, ntf))
    for e in range(nev):
        g = rng.integers(0, ngrd)
        picks[e] = tables[:, g] + rng.uniform(0, 60) + rng.normal(0, 0.02, ntf)
        wts[e, rng.integers(0, ntf)] = 0.0
    return tables, picks, wts


def test_noalloc_matches_locator(fk):
    import torch
    lib = fk.lib()
    ntf, ngrd = 16, 30011
    tables, picks, wts = _problem(11, ntf, ngrd, 40)
    # the regular entry point on all events
    loc = fk.Locator(picks.shape[0], ntf, ngrd)
    for k in range(ntf):
        loc.setTravelTimeField32f(k + 1, tables[k])
    for e in range(picks.shape[0]):
        loc.setObservation(e + 1, np.arange(1, ntf + 1), picks[e], wts[e])
    want_i, want_t0, want_obj = loc.locateEvents(np.arange(1, picks.shape[0] + 1))
    loc.finalize()
    # the allocation-free entry point on device buffers owned by the caller
    tepoch = picks.max(axis=1)
    obs = np.where(wts > 0, picks - tepoch[:, None], 0.0).astype(np.float32)
    w32 = wts.astype(np.float32)
    dev = torch.device("cuda", 0)
    t_tab = torch.from_numpy(tables).to(dev)
    for lo, hi in ((0, 25), (25, 40)):       # two calls in a row
        n = hi - lo
        t_obs = torch.from_numpy(obs[lo:hi].copy()).to(dev)
        t_w = torch.from_numpy(w32[lo:hi].copy()).to(dev)
        o_i = torch.full((n,), -1, dtype=torch.int32, device=dev)
        o_t0 = torch.zeros(n, dtype=torch.float32, device=dev)
        o_obj = torch.zeros(n, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        ierr = ctypes.c_int(1)
        lib.fteik_b200_locate_l2_noalloc(ngrd, ngrd, ntf, t_tab.data_ptr(), n, t_obs.data_ptr(),
                                         t_w.data_ptr(), o_i.data_ptr(), o_t0.data_ptr(),
                                         o_obj.data_ptr(), None, ctypes.byref(ierr))
        assert ierr.value == 0
        torch.cuda.synchronize()
        got_i = o_i.cpu().numpy() + 1
        got_t0 = o_t0.cpu().numpy().astype(np.float64) + tepoch[lo:hi]
        got_obj = o_obj.cpu().numpy().astype(np.float64)
        assert np.array_equal(got_i, want_i[lo:hi])
        assert np.array_equal(got_t0, want_t0[lo:hi])
        assert np.array_equal(got_obj, want_obj[lo:hi])


def test_noalloc_rejects_too_many_events(fk):
    ierr = ctypes.c_int(0)
    fk.lib().fteik_b200_locate_l2_noalloc(10, 10, 2, 1, 65537, 1, 1, 1, 1, 1, None, ctypes.byref(ierr))
    assert ierr.value == 1
