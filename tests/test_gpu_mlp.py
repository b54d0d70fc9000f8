"""Surrogate network on the GPU against the FP64 CPU oracle
(oracle/mlp_oracle.py), and the surrogate-pruned grid search (locate
method 2) against the exhaustive tensor-core search (method 1), its reference."""
import os
import sys

import numpy as np
import pytest

from models import linear_gradient_tables, synthetic_events

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


# hidden-layer products: FP32 CUDA cores (0), split BF16 on the tensor cores
# (3, about FP32 accuracy) and plain BF16 on the tensor cores (1); the
# tolerances are relative to the FP64 oracle
PRODUCTS = [(0, 2e-4, 1e-5), (3, 2e-4, 1e-5), (1, 2e-2, 5e-3)]


@pytest.mark.parametrize("products,gtol,ftol", PRODUCTS)
@pytest.mark.parametrize("width,depth,n", [(32, 3, 64), (256, 5, 300), (256, 5, 4096), (256, 5, 16384),
                                           (102, 3, 301)])
def test_gradient_matches_oracle(fk, width, depth, n, products, gtol, ftol):
    """The hidden layers reach the tensor cores when their width is 64 or
    more (width 256); the width-32 network checks the CUDA-core path; width
    102 with 301 rows (extents not multiples of 4 or 64) the fallbacks:
    plain-load staging with ragged K blocks, the scalar epilogue, the
    one-column thin-layer kernels and the separate column sums."""
    old = fk.set_mlp_tensor_products(products)
    try:
        _gradient_case(fk, width, depth, n, gtol, ftol)
    finally:
        fk.set_mlp_tensor_products(old)


def _gradient_case(fk, width, depth, n, gtol, ftol):
    net = fk.MLP(width, depth, seed=3)
    rng = np.random.default_rng(1)
    w = net.weights()
    x = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
    y = rng.uniform(0.6, 1.1, n).astype(np.float32)
    loss, g = net.gradient(x, y)
    wl, gw = M.loss_and_grad(w.astype(np.float64), width, depth, x, y)
    assert abs(loss - wl) <= max(ftol, 1e-5) * 10 * wl + 1e-9
    off = 0
    for o, i in M.layer_shapes(width, depth):
        for size in (o * i, o):
            a, b = g[off:off + size].astype(np.float64), gw[off:off + size]
            assert np.linalg.norm(a - b) <= gtol * np.linalg.norm(b) + 1e-9
            off += size
    tau = net.forward(x)
    want = M.forward(w.astype(np.float64), width, depth, x)[0]
    assert np.max(np.abs(tau - want)) <= ftol * (1 + np.max(np.abs(want)))
    net.finalize()


def test_training_reduces_loss(fk):
    net = fk.MLP(64, 3, seed=5)
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (20000, 6)).astype(np.float32)
    y = (0.8 + 0.1 * np.sin(2 * x[:, 0]) * x[:, 3] + 0.05 * x[:, 1] ** 2).astype(np.float32)
    l0, _ = net.gradient(x[:4096], y[:4096])
    net.train(x, y, steps=1500, batch=1024, lr=3e-3)
    l1, _ = net.gradient(x[:4096], y[:4096])
    assert l1 < l0 / 50
    net.finalize()


def _prune_problem(fk, nev, seed_ev=21, grad=0.5):
    nz, nx, ny, h = 24, 40, 36, 100.0
    tables, (sz, sx, sy) = linear_gradient_tables(nz, nx, ny, h, 64, grad=grad, seed=20)
    _, picks = synthetic_events(tables, nev, seed=seed_ev)
    loc = fk.Locator(nev, 64, tables.shape[1])
    for k in range(64):
        loc.setTravelTimeField32f(k + 1, tables[k])
    o2t = np.arange(1, 65)
    for e in range(nev):
        loc.setObservation(e + 1, o2t, picks[e], np.ones(64))
    loc.setGeometry(nz, nx, ny, h, h, h, sz, sx, sy)
    return loc


def test_pruned_search_matches_exhaustive(fk):
    nev = 600
    loc = _prune_problem(fk, nev)
    ev = np.arange(1, nev + 1)
    loc.setMethod(1)
    ref = loc.locateEvents(ev)
    fk.MLP(256, 5, seed=7)                     # fresh network
    loss = loc.trainSurrogate(nsamples=400_000, steps=1500, batch=4096, lr=2e-3, vref=3000.0, seed=7)
    assert loss < 1e-4                          # tau ~ 0.9: about 1 % rms
    loc.buildSurrogate((4, 4, 4))
    loc.setMethod(2)
    got = loc.locateEvents(ev)
    nfb, ncoarse, nblk = loc.pruneInfo()
    agree = np.mean(got[0] == ref[0])
    assert agree >= 0.995, (agree, nfb)
    same = got[0] == ref[0]
    assert np.all(np.abs(got[2][same] - ref[2][same]) <= 1e-9 * np.abs(ref[2][same]) + 1e-12)
    assert nfb <= nev // 100
    assert nblk / (nev - nfb) <= 16       # about 1k of the 34,560 fine nodes per event
    loc.finalize()


def test_rebuild_keeps_block_copy_only_while_tables_unchanged(fk):
    """buildSurrogate keeps the exact tables' block copy across rebuilds
    with the same tables and block shape (the same located events), and
    rebuilds it when a table changes (the pruned search then follows the
    new tables: it agrees with the exhaustive search on them)."""
    nev = 300
    loc = _prune_problem(fk, nev)
    ev = np.arange(1, nev + 1)
    fk.MLP(256, 5, seed=7)
    loc.trainSurrogate(nsamples=400_000, steps=600, batch=4096, lr=2e-3, vref=3000.0, seed=7)
    loc.setMethod(2)
    loc.buildSurrogate((4, 4, 4))
    first = loc.locateEvents(ev)
    loc.buildSurrogate((4, 4, 4))                    # same tables and shape: the copy is kept
    again = loc.locateEvents(ev)
    assert np.array_equal(first[0], again[0]) and np.array_equal(first[2], again[2])
    # move one station's table: the copy must follow it
    nz, nx, ny, h = 24, 40, 36, 100.0
    tables, _ = linear_gradient_tables(nz, nx, ny, h, 64, grad=0.5, seed=20)
    shifted = tables[5] + np.float32(0.35)
    loc.setTravelTimeField32f(6, shifted)
    loc.buildSurrogate((4, 4, 4))
    got = loc.locateEvents(ev)
    loc.setMethod(1)
    ref = loc.locateEvents(ev)
    assert np.mean(got[0] == ref[0]) >= 0.995
    same = got[0] == ref[0]
    assert np.all(np.abs(got[2][same] - ref[2][same]) <= 1e-9 * np.abs(ref[2][same]) + 1e-12)
    loc.finalize()


@pytest.mark.parametrize("n", [20_000, 20_001, 85_537])
def test_fused_forward_matches_layer_by_layer(fk, n):
    """The one-kernel forward pass (BF16 products, activations kept on the
    SM) gives the layer-by-layer path's outputs bit for bit, full and
    ragged last tiles included (sizes at which the layer-by-layer products
    are not split over K: at least 148 row tiles per 65,536-row chunk)."""
    old_p = fk.set_mlp_tensor_products(1)
    try:
        net = fk.MLP(256, 5, seed=11)
        rng = np.random.default_rng(n)
        net.setWeights(net.weights() * rng.uniform(0.5, 1.5, net.nweights()).astype(np.float32))
        x = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
        outs = []
        for fused in (1, 0):
            old = fk.set_mlp_fused_forward(fused)
            try:
                outs.append(net.forward(x))
            finally:
                fk.set_mlp_fused_forward(old)
        assert np.array_equal(outs[0], outs[1])
        net.finalize()
    finally:
        fk.set_mlp_tensor_products(old_p)


@pytest.mark.parametrize("products", [1, 3])
@pytest.mark.parametrize("n", [300, 4096, 16384])
def test_async_staging_matches_synchronous(fk, products, n):
    """The tensor-core products staged by asynchronous copies (FP32 ring,
    then BF16 conversion) give the synchronous staging's loss, gradient and
    outputs bit for bit: forward, input-gradient and split-K weight-gradient
    products with their fused column sums."""
    old_p = fk.set_mlp_tensor_products(products)
    try:
        net = fk.MLP(256, 5, seed=13)
        rng = np.random.default_rng(n + products)
        x = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
        y = rng.uniform(0.6, 1.1, n).astype(np.float32)
        out = []
        for on in (1, 0):
            old = fk.set_mlp_async_staging(on)
            try:
                old_f = fk.set_mlp_fused_forward(0)
                try:
                    loss, g = net.gradient(x, y)
                    out.append((loss, g, net.forward(x)))
                finally:
                    fk.set_mlp_fused_forward(old_f)
            finally:
                fk.set_mlp_async_staging(old)
        gd = np.flatnonzero(out[0][1] != out[1][1])
        fd = np.flatnonzero(out[0][2] != out[1][2])
        assert out[0][0] == out[1][0], (out[0][0], out[1][0])
        assert gd.size == 0, ("gradient entries differ", gd[:10], gd.size)
        assert fd.size == 0, ("outputs differ", fd[:10], fd.size)
        net.finalize()
    finally:
        fk.set_mlp_tensor_products(old_p)


def test_retraining_from_restored_weights_is_reproducible(fk):
    """setWeights restores a network's starting state (weights, Adam
    moments and step count): training again from the initial weights gives
    the first run's weights and loss bit for bit (the bench times a run
    after an untimed warm-up run this way)."""
    loc = _prune_problem(fk, 40)
    net = fk.MLP(256, 5, seed=7)
    w0 = net.weights()
    loss_a = loc.trainSurrogate(nsamples=200_000, steps=30, batch=4096, lr=2e-3, vref=3000.0, seed=7)
    wa = net.weights()
    net.setWeights(w0)
    loss_b = loc.trainSurrogate(nsamples=200_000, steps=30, batch=4096, lr=2e-3, vref=3000.0, seed=7)
    assert loss_a == loss_b
    assert np.array_equal(wa, net.weights())
    assert not np.array_equal(wa, w0)
    loc.finalize()


def test_captured_training_steps_match_eager(fk):
    """trainSurrogate replays one captured step (step number, learning rate
    and bias corrections from device memory): the same weights and loss as
    launching every kernel of every step."""
    loc = _prune_problem(fk, 40)
    out = []
    for graph in (1, 0):
        old = fk.set_mlp_train_graph(graph)
        try:
            net = fk.MLP(256, 5, seed=7)
            loss = loc.trainSurrogate(nsamples=200_000, steps=80, batch=4096, lr=2e-3, vref=3000.0, seed=7)
            out.append((loss, net.weights()))
        finally:
            fk.set_mlp_train_graph(old)
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    loc.finalize()


def test_training_is_what_makes_pruning_work(fk):
    """Same pipeline with an untrained network (tau = 1 + noise: straight rays
    at v_ref) in a strong gradient (v = 3000 + 2 z m/s, up to ~7600 m/s): its
    coarse ranking is biased in depth, so the descent over blocks has much
    more to do than with the trained network; both end at the exhaustive
    search's answer."""
    nev = 300
    loc = _prune_problem(fk, nev, seed_ev=22, grad=2.0)
    ev = np.arange(1, nev + 1)
    loc.setMethod(1)
    ref = loc.locateEvents(ev)
    loc.setPruning(4, 8)

    def run(steps):
        fk.MLP(256, 5, seed=7)
        loc.trainSurrogate(nsamples=400_000, steps=steps, batch=4096, lr=2e-3 if steps > 1 else 1e-12,
                           vref=3000.0, seed=7)
        loc.buildSurrogate((4, 4, 4))
        loc.setMethod(2)
        got = loc.locateEvents(ev)
        nfb, _, nblk = loc.pruneInfo()
        extra = nblk - 8 * (nev - nfb) + 540 * nfb   # an exhaustive search ~ 540 blocks
        return got, extra

    got_u, extra_u = run(1)
    got_t, extra_t = run(1500)
    assert np.mean(got_t[0] == ref[0]) >= 0.99
    assert extra_u >= 3 * max(extra_t, 10), (extra_u, extra_t)
    loc.finalize()
