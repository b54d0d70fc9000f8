"""CPU FP64 oracle of the travel-time surrogate network (test infrastructure
only: imported by tests/ and nothing on the product path).

The network has no counterpart in the reference, so this oracle is pinned by
finite differences of its own loss (tests/test_oracle.py), not by reference
outputs.  It restates, in numpy and FP64, the GPU network of fteik_b200:

    x_0 = inputs [B, 6]
    z_l = x_l W_l^T + b_l            l = 0 .. L-1 (W_l [out, in])
    x_{l+1} = silu(z_l)              l < L-1,   silu(z) = z / (1 + exp(-z))
    tau = z_{L-1}[:, 0]
    loss = mean((tau - y)^2)

Parameters are one flat vector: for each layer W_l (row-major [out, in]),
then b_l.
"""
import numpy as np


def layer_shapes(width, depth, nin=6):
    dims = [nin] + [width] * depth + [1]
    return [(dims[l + 1], dims[l]) for l in range(len(dims) - 1)]


def unpack(w, width, depth):
    w = np.asarray(w, np.float64)
    out, off = [], 0
    for o, i in layer_shapes(width, depth):
        W = w[off:off + o * i].reshape(o, i)
        off += o * i
        b = w[off:off + o]
        off += o
        out.append((W, b))
    assert off == w.size
    return out


def forward(w, width, depth, x):
    layers = unpack(w, width, depth)
    a = np.asarray(x, np.float64)
    zs, xs = [], [a]
    for l, (W, b) in enumerate(layers):
        z = a @ W.T + b
        zs.append(z)
        if l < len(layers) - 1:
            a = z / (1.0 + np.exp(-z))
            xs.append(a)
    return zs[-1][:, 0], zs, xs


def loss_and_grad(w, width, depth, x, y):
    layers = unpack(w, width, depth)
    tau, zs, xs = forward(w, width, depth, x)
    y = np.asarray(y, np.float64)
    n = tau.size
    loss = np.mean((tau - y) ** 2)
    dz = (2.0 * (tau - y) / n)[:, None]
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = dz.T @ xs[l]
        gb = dz.sum(axis=0)
        grads[l] = (gW, gb)
        if l > 0:
            da = dz @ W
            z = zs[l - 1]
            s = 1.0 / (1.0 + np.exp(-z))
            dz = da * s * (1.0 + z * (1.0 - s))
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
