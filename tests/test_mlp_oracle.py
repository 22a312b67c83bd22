"""The numpy restatement of the learned-forecast network (oracle/mlp.py): its analytic
gradients against central finite differences in FP64 (the reference's gradient-check
pattern, src/main.cpp:259-270), the BF16 rounding helper, and the Adam step."""
from __future__ import annotations

import numpy as np

from oracle import mlp


def _setup(r=3, q=2, h=8, B=5, seed=0):
    rng = np.random.default_rng(seed)
    flat = rng.normal(0, 0.5, sum(int(np.prod(s)) for _, s in mlp.layout(r, q, h).values()))
    x = rng.normal(0, 1, (B, r + q))
    t = rng.normal(0, 1, (B, r))
    s_in = rng.uniform(0.5, 2.0, r + q)
    s_out = rng.uniform(0.1, 1.0, r)
    return flat, x, t, s_in, s_out


def test_gradients_match_central_differences():
    r, q, h = 3, 2, 8
    flat, x, t, s_in, s_out = _setup(r, q, h)
    loss, g = mlp.loss_and_grads(mlp.unpack(flat, r, q, h), x, t, s_in, s_out, r, emulate=False)
    gflat = mlp.pack(g, r, q, h)
    eps = 1e-6
    fd = np.zeros_like(flat)
    for i in range(flat.size):
        up, dn = flat.copy(), flat.copy()
        up[i] += eps
        dn[i] -= eps
        lu, _ = mlp.loss_and_grads(mlp.unpack(up, r, q, h), x, t, s_in, s_out, r, emulate=False)
        ld, _ = mlp.loss_and_grads(mlp.unpack(dn, r, q, h), x, t, s_in, s_out, r, emulate=False)
        fd[i] = (lu - ld) / (2 * eps)
    assert loss > 0
    np.testing.assert_allclose(gflat, fd, rtol=1e-6, atol=1e-9)


def test_bf16_rounding():
    one = 1.0
    ulp = 2.0 ** -7
    vals = np.array([one, one + ulp / 2, one + 1.5 * ulp, one + 0.75 * ulp, -3.0, 0.0])
    np.testing.assert_array_equal(mlp.bf16(vals),
                                  [one, one, one + 2 * ulp, one + ulp, -3.0, 0.0])


def test_emulated_forward_is_close_to_exact():
    r, q, h = 3, 2, 8
    flat, x, t, s_in, s_out = _setup(r, q, h)
    P = mlp.unpack(flat, r, q, h)
    ye, _ = mlp.forward(P, x, s_in, s_out, r, emulate=True)
    yx, _ = mlp.forward(P, x, s_in, s_out, r, emulate=False)
    assert np.max(np.abs(ye - yx)) < 0.05 * np.max(np.abs(yx))


def test_adam_first_step_is_signed_learning_rate():
    g = np.array([1e-3, -2.0, 5.0])
    p, m, v = mlp.adam(np.zeros(3), g, np.zeros(3), np.zeros(3), 1, 1e-3)
    np.testing.assert_allclose(p, -1e-3 * np.sign(g), rtol=1e-4)
    np.testing.assert_allclose(m, 0.1 * g)
    np.testing.assert_allclose(v, 0.001 * g * g)
