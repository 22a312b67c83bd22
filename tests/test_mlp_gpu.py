"""The learned-forecast network on the B200 (hzlb_mlp_*: BF16 tcgen05 forward and backward,
Adam) against the numpy restatement oracle/mlp.py with the device's BF16 rounding points
emulated.  Tolerances: forward residual and every gradient tensor within 1e-2 relative L2 (FP32
accumulation order and BF16 rounding ties differ from the FP64 oracle); Adam to 1e-5."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp as om

pytestmark = pytest.mark.gpu

R, Q, H = 64, 8, 512


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _data(B, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (B, R + Q)).astype(np.float32) * rng.uniform(0.2, 3.0, R + Q).astype(np.float32)
    t = (x[:, :R] + 0.3 * rng.normal(0, 1, (B, R))).astype(np.float32)
    s_in = np.abs(x).mean(0).astype(np.float32) + 0.1
    s_out = rng.uniform(0.05, 0.5, R).astype(np.float32)
    return x, t, s_in, s_out


def _net(hzlb, B, seed=1):
    net = hzlb.Mlp(R, Q, H, B, seed=seed)
    rng = np.random.default_rng(seed + 100)
    p = net.params()
    parts = net.unpack(p.copy())
    parts["b1"] = rng.normal(0, 0.1, H)
    parts["b2"] = rng.normal(0, 0.1, H)
    parts["b3"] = rng.normal(0, 0.1, R)
    parts["W3"] = rng.normal(0, 1 / np.sqrt(H), (R, H))   # nontrivial output layer
    net.set_params(net.pack(parts))
    return net


@pytest.mark.parametrize("B", [300, 1024])
def test_forward_matches_oracle(hzlb, B):
    import torch
    x, _, s_in, s_out = _data(B, B)
    net = _net(hzlb, B)
    net.set_scales(s_in, s_out)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    P = om.unpack(net.params(), R, Q, H)
    yo, c = om.forward(P, x, s_in, s_out, R, emulate=True)
    # compare the learned increment, not the identity part
    assert _rel((y - x[:, :R]) / s_out, c["res"]) < 1e-2


@pytest.mark.parametrize("B", [200, 1024])
def test_gradients_match_oracle(hzlb, B):
    import torch
    x, t, s_in, s_out = _data(B, 7 + B)
    net = _net(hzlb, B, seed=3)
    net.set_scales(s_in, s_out)
    loss = net.train_step(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), 0.0)
    p, g = net.params(grads=True)
    lo, go = om.loss_and_grads(om.unpack(p, R, Q, H), x, t, s_in, s_out, R, emulate=True)
    assert abs(loss - lo) / lo < 1e-3
    gd = net.unpack(g)
    for k in ("W1", "W2", "W3", "b1", "b2", "b3"):
        assert _rel(gd[k], go[k]) < 1e-2, k
    # lr = 0 leaves the parameters unchanged
    np.testing.assert_array_equal(net.params(), p)


def test_adam_step_matches_oracle(hzlb):
    import torch
    B = 256
    x, t, s_in, s_out = _data(B, 11)
    net = _net(hzlb, B, seed=5)
    net.set_scales(s_in, s_out)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    p0 = net.params().astype(np.float64)
    m = np.zeros_like(p0)
    v = np.zeros_like(p0)
    p = p0
    for step in (1, 2, 3):
        net.train_step(xd, td, 1e-3)
        _, g = net.params(grads=True)
        p, m, v = om.adam(p, g.astype(np.float64), m, v, step, 1e-3)
        np.testing.assert_allclose(net.params(), p, rtol=1e-5, atol=1e-7)


def test_training_fits_a_smooth_map(hzlb):
    import torch
    B = 2048
    rng = np.random.default_rng(0)
    x = rng.normal(0, 1, (B, R + Q)).astype(np.float32)
    A = rng.normal(0, 1 / np.sqrt(R + Q), (R, R + Q))
    t = (x[:, :R] + 0.2 * np.tanh(x @ A.T)).astype(np.float32)
    net = hzlb.Mlp(R, Q, H, B, seed=2)
    net.set_scales(np.ones(R + Q, np.float32), np.full(R, 0.2, np.float32))
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = net.train_step(xd, td, 1e-3)
    for _ in range(300):
        last = net.train_step(xd, td, 1e-3)
    assert last < first / 20, (first, last)


def test_invalid_shapes(hzlb):
    import torch
    with pytest.raises(hzlb.HzlbInvalidArgument):
        hzlb.Mlp(R, Q, 500, 16)
    net = hzlb.Mlp(R, Q, H, 16)
    x = torch.zeros(32, R + Q, device="cuda")
    with pytest.raises(hzlb.HzlbInvalidArgument):
        net.forward(x)
    with pytest.raises(ValueError):
        net.forward(torch.zeros(8, R, device="cuda"))
