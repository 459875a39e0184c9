"""CPU checker for the learned-chemistry MLP (test infrastructure only).

The model has no counterpart in the reference; this numpy restatement of its
forward pass, mean-squared-error loss and backward pass is what the GPU
kernels' outputs and gradients are compared with. It rounds to bf16 at the
same points as the device code (inputs, weights, hidden activations and the
gradients fed to the next GEMM) and accumulates in float64, so the remaining
difference from the device is fp32 accumulation order.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), kept as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unflatten(params, sizes):
    """Split one member's flat parameters (W out x in, then b, per layer)."""
    out, off = [], 0
    for n_in, n_out in sizes:
        W = params[off:off + n_in * n_out].reshape(n_out, n_in)
        off += n_in * n_out
        b = params[off:off + n_out]
        off += n_out
        out.append((W.astype(np.float64), b.astype(np.float64)))
    return out, off


def layer_sizes(n_in, width, hidden, n_out):
    dims = [n_in] + [width] * hidden + [n_out]
    return list(zip(dims[:-1], dims[1:]))


def loss_and_grads(params, X, T, n_in, width, hidden, n_out, in_shift, in_scale, out_shift, out_scale):
    """MSE of normalised outputs and its gradient, flattened like the parameters."""
    layers, _ = unflatten(params, layer_sizes(n_in, width, hidden, n_out))
    n = X.shape[0]
    x = bf16((X - in_shift) * in_scale).astype(np.float64)
    t = ((T - out_shift) * out_scale).astype(np.float64)
    Wb = [bf16(W).astype(np.float64) for W, _ in layers]
    acts, pres = [x], []
    h = x
    for l in range(hidden):
        z = h @ Wb[l].T + layers[l][1]
        pres.append(z)
        h = bf16(silu(z)).astype(np.float64)
        acts.append(h)
    y = h @ Wb[hidden].T + layers[hidden][1]
    d = y - t
    loss = float(np.mean(d * d))
    dy = bf16(2.0 * d / (n * n_out)).astype(np.float64)
    grads = [None] * (hidden + 1)
    grads[hidden] = (dy.T @ acts[hidden], dy.sum(axis=0))
    dz_b = None
    g_up = dy
    for l in range(hidden - 1, -1, -1):
        dh = g_up @ Wb[l + 1]
        dz = (dh.astype(np.float32) * silu_grad(pres[l].astype(np.float32))).astype(np.float64)
        dz_b = bf16(dz).astype(np.float64)
        grads[l] = (dz_b.T @ acts[l], dz.sum(axis=0))
        g_up = dz_b
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat


def predict(params, X, n_in, width, hidden, n_out, in_shift, in_scale, out_shift, out_scale):
    """Physical outputs of one member."""
    layers, _ = unflatten(params, layer_sizes(n_in, width, hidden, n_out))
    h = bf16((X - in_shift) * in_scale).astype(np.float64)
    for l in range(hidden):
        h = bf16(silu(h @ bf16(layers[l][0]).astype(np.float64).T + layers[l][1])).astype(np.float64)
    y = h @ bf16(layers[hidden][0]).astype(np.float64).T + layers[hidden][1]
    return y / out_scale + out_shift
