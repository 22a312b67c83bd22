"""TEST INFRASTRUCTURE ONLY: numpy restatement of the learned reduced forecast network.

The reference has no learned model (its reduced forecast is the Galerkin ROM of
src/reduced.cpp:137-209), so this checker is **parity unpinned**: it is pinned instead by a
central finite-difference check of its own gradients (the reference's gradient-check pattern,
src/main.cpp:259-270 and tests/verification.cpp:255-261), and the device kernels are checked
against it.

Network (x = (a, xi): r coefficients then q noise amplitudes):
    h1 = gelu(W1 (x / s_in) + b1),  h2 = gelu(W2 h1 + b2),  y = a + s_out * (W3 h2 + b3)
gelu is the tanh form.  Loss = mean over batch and r of (y - target)^2.

``emulate=True`` reproduces the device's rounding points: the scaled input, the hidden
activations, the weight matrices and the back-propagated deltas are rounded to BF16 (round to
nearest even) where the device feeds them to a BF16 tensor-core product; sums are FP64 here
and FP32 on the device.  ``emulate=False`` is the exact FP64 function (for the finite-difference
check).  Only ``tests/`` imports this module.
"""
from __future__ import annotations

import numpy as np

K0 = 0.7978845608028654
K1 = 0.044715


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) through FP32; returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K0 * (x + K1 * x ** 3)))


def gelu_grad(x):
    th = np.tanh(K0 * (x + K1 * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * K0 * (1.0 + 3.0 * K1 * x * x)


def layout(r: int, q: int, hidden: int) -> dict:
    i, h = r + q, hidden
    shapes = [("W1", (h, i)), ("W2", (h, h)), ("W3", (r, h)), ("b1", (h,)), ("b2", (h,)),
              ("b3", (r,))]
    out, off = {}, 0
    for name, shp in shapes:
        out[name] = (off, shp)
        off += int(np.prod(shp))
    return out


def unpack(flat, r: int, q: int, hidden: int) -> dict:
    flat = np.asarray(flat, np.float64)
    return {k: flat[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in layout(r, q, hidden).items()}


def pack(parts: dict, r: int, q: int, hidden: int) -> np.ndarray:
    lay = layout(r, q, hidden)
    flat = np.zeros(sum(int(np.prod(s)) for _, s in lay.values()))
    for k, (o, s) in lay.items():
        flat[o:o + int(np.prod(s))] = np.asarray(parts[k], np.float64).ravel()
    return flat


def forward(P: dict, x, s_in, s_out, r: int, emulate: bool = True):
    """Returns (y, cache) for a batch x [B][r+q]."""
    rnd = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    x = np.asarray(x, np.float64)
    if emulate:   # the device divides in FP32 before rounding
        xs = rnd((x.astype(np.float32) / np.asarray(s_in, np.float32)))
    else:
        xs = x / np.asarray(s_in, np.float64)
    W1, W2, W3 = rnd(P["W1"]), rnd(P["W2"]), rnd(P["W3"])
    pre1 = xs @ W1.T + P["b1"]
    h1 = rnd(gelu(pre1))
    pre2 = h1 @ W2.T + P["b2"]
    h2 = rnd(gelu(pre2))
    res = h2 @ W3.T + P["b3"]
    y = x[:, :r] + np.asarray(s_out, np.float64) * res
    return y, dict(xs=xs, pre1=pre1, h1=h1, pre2=pre2, h2=h2, res=res, W1=W1, W2=W2, W3=W3)


def loss_and_grads(P: dict, x, target, s_in, s_out, r: int, emulate: bool = True):
    """Mean squared error and its gradient with respect to every parameter."""
    rnd = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    y, c = forward(P, x, s_in, s_out, r, emulate)
    d = y - np.asarray(target, np.float64)
    B = x.shape[0]
    loss = float(np.mean(d * d))
    dr = np.asarray(s_out, np.float64) * 2.0 * d / (B * r)
    drb = rnd(dr)
    g = {"W3": drb.T @ c["h2"], "b3": dr.sum(0)}
    dpre2 = (drb @ c["W3"]) * gelu_grad(c["pre2"])
    dpre2b = rnd(dpre2)
    g["W2"] = dpre2b.T @ c["h1"]
    g["b2"] = dpre2.sum(0)
    dpre1 = (dpre2b @ c["W2"]) * gelu_grad(c["pre1"])
    dpre1b = rnd(dpre1)
    g["W1"] = dpre1b.T @ c["xs"]
    g["b1"] = dpre1.sum(0)
    return loss, g


def adam(p, g, m, v, t: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba, Algorithm 1) on flat arrays; returns (p, m, v)."""
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** t)
    vh = v / (1 - beta2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
