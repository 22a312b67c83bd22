"""POD on the device and the learned forecast window built on it.

* hzlb_fit_pod (the reference's fit_pod, src/reduced.cpp:36-136) against the committed golden
  vectors, the rank-2 analytic case (tests/verification.cpp:273-282) and the reference library
  itself: singular values and captured variance to 1e-10, modes with their signs to 1e-8.
* hzlb_pod_fit (compact FP32 snapshots) against an FP64 numpy eigendecomposition of the
  weighted snapshot Gram matrix (the reference's inner product): eigenvalues to 1e-4 relative,
  modes spanning the same space, both by Jacobi (<= 256 snapshots) and by subspace iteration.
* Projection against numpy, noise-mode amplitudes against the oracle's Philox draws, and the
  learned forecast window with networks whose output is known.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def _full_fields(hzlb, n, m, rank, seed, decay=0.7, noise=1e-3):
    """m real fields (reference layout) of approximate rank `rank` with decaying amplitudes."""
    base = np.array([hzlb.grf_spectrum(n, seed, j) for j in range(rank + 1)])
    rng = np.random.default_rng(seed)
    amp = rng.normal(size=(m, rank)) * decay ** np.arange(rank)
    x = np.einsum("ij,jab->iab", amp, base[:rank]) + 0.3 * base[rank][None]
    x += noise * np.einsum("i,ab->iab", rng.normal(size=m), base[0])
    return x


def test_fit_pod_golden_and_analytic(hzlb):
    g = np.load(GOLDEN / "pod_n16.npz")
    out = hzlb.fit_pod(g["snapshots"], 4, 0.9999999)
    np.testing.assert_allclose(out["mean"].reshape(g["mean"].shape), g["mean"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(out["singular_values"], g["singular_values"], rtol=1e-10)
    np.testing.assert_allclose(np.abs(out["modes"].reshape(g["modes"].shape)), np.abs(g["modes"]),
                               atol=1e-9)
    assert abs(out["captured"] - float(g["captured"])) < 1e-10
    t = 2 * np.pi * np.arange(30) / 30
    snaps = np.stack([1 + np.sin(t), 2 + 2 * np.cos(t), np.full(30, 3.0)], axis=1).astype(complex)
    out = hzlb.fit_pod(snaps, 3, 1.0)
    assert len(out["modes"]) == 2
    gram = np.real(np.conj(out["modes"]) @ out["modes"].T)
    np.testing.assert_allclose(gram, np.eye(2), atol=1e-12)


@pytest.mark.parametrize("n,m,rank,fraction", [(16, 40, 6, 0.9999), (32, 200, 12, 0.999999)])
def test_fit_pod_matches_reference(hzlb, reference, n, m, rank, fraction):
    snaps = _full_fields(hzlb, n, m, 10, 17)
    ref_mean, ref_modes, ref_sv, ref_cap = reference.fit_pod(snaps, rank, fraction)
    got = hzlb.fit_pod(snaps, rank, fraction)
    assert len(got["modes"]) == len(ref_modes)
    np.testing.assert_allclose(got["singular_values"], ref_sv, rtol=1e-10)
    assert abs(got["captured"] - ref_cap) < 1e-10
    np.testing.assert_allclose(got["mean"].ravel(), ref_mean, rtol=0, atol=1e-13)
    np.testing.assert_allclose(got["modes"].reshape(len(ref_modes), -1), ref_modes, atol=1e-8)


def test_fit_pod_rejects_like_the_reference(hzlb):
    with pytest.raises(hzlb.HzlbInvalidArgument):
        hzlb.fit_pod(np.zeros((1, 4, 4), complex), 2)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        hzlb.fit_pod(np.ones((513, 2, 2), complex), 2)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        hzlb.fit_pod(np.ones((4, 2, 2), complex), 2)   # no variance
    bad = np.ones((4, 2, 2), complex)
    bad[1, 0, 0] = np.nan
    with pytest.raises(hzlb.HzlbInvalidArgument):
        hzlb.fit_pod(bad, 2)


def _weights(n):
    k = (n - 1) // 3
    ld = 2 * k + 1
    w = np.where(np.arange(k + 1) > 0, np.sqrt(2.0), 1.0)
    return np.repeat(np.repeat(w, ld), 2)   # per real entry of a compact member


def _numpy_pod(x, n, rank):
    w = _weights(n)
    xc = (x - x.mean(axis=0)) * w
    G = xc @ xc.T
    ev, vec = np.linalg.eigh(G)
    order = np.argsort(ev)[::-1][:rank]
    modes_w = (vec[:, order] / np.sqrt(ev[order])).T @ xc
    return ev[order], modes_w / w, np.trace(G)


@pytest.mark.parametrize("m,rank,data_rank", [(120, 8, 24), (600, 16, 24), (400, 8, 10)])
def test_compact_pod_matches_numpy(hzlb, m, rank, data_rank):
    """(400, 8, 10): the data span fewer directions than the 32 iteration vectors, so the
    orthonormalisation meets dependent columns and must replace them."""
    import torch
    n = 32
    full = _full_fields(hzlb, n, m, data_rank, 5, decay=0.8)
    x = hzlb.full_to_compact(full, n).astype(np.complex64).view(np.float32)
    pod = hzlb.Pod(n, torch.from_numpy(x).cuda(), rank, oversample=24, iterations=80, seed=1)
    info = pod.info()
    ev, modes_ref, trace = _numpy_pod(x.astype(np.float64), n, rank)
    np.testing.assert_allclose(info["eigenvalues"], ev, rtol=1e-4)
    assert abs(info["captured"] - ev.sum() / trace) < 1e-5
    assert info["residual"] < 1e-4
    modes, mean = pod.modes()
    np.testing.assert_allclose(mean, x.mean(axis=0), rtol=0, atol=1e-5 * np.abs(x).max())
    w = _weights(n)
    gram = (modes * w) @ (modes * w).T
    np.testing.assert_allclose(gram, np.eye(rank), atol=2e-5)
    # same space as the FP64 modes: the projection of each reference mode is kept
    overlap = (modes * w) @ (modes_ref * w).T
    np.testing.assert_allclose(np.linalg.svd(overlap, compute_uv=False), np.ones(rank), atol=1e-3)
    # projection of states against numpy
    states = torch.from_numpy(x[:50]).cuda()
    a = pod.project(states).cpu().numpy()
    expect = ((x[:50].astype(np.float64) - mean) * w) @ (modes.astype(np.float64) * w).T
    np.testing.assert_allclose(a, expect, rtol=0, atol=1e-5 * np.abs(expect).max())


def test_noise_amplitudes_match_philox(hzlb, oracle):
    import torch
    cfg = hzlb.Config(n=64, members=5, precision=4, noise_sigma=0.05, noise_kmax=4, seed=77,
                      member_base=3)
    dt, first, steps = 5e-4, 40, 20
    out = torch.zeros((5, 10), dtype=torch.float32, device="cuda")
    hzlb.noise_amplitudes(cfg, dt, first, steps, 5, out)
    got = out.cpu().numpy()
    scale = 0.05 * np.sqrt(dt) / np.sqrt(2.0)
    x1, x2 = C.c_double(), C.c_double()
    for m in range(5):
        for q, (kx, ky) in enumerate([(1, 0), (0, 1), (1, 1), (1, -1)]):
            code = oracle.lib.ho_mode_code(kx, ky)
            sr = si = 0.0
            for s in range(first, first + steps):
                oracle.lib.ho_philox_normal_pair(77, 3 + m, s, code, C.byref(x1), C.byref(x2))
                sr += scale * x1.value
                si += scale * x2.value
            np.testing.assert_allclose(got[m, 2 * q:2 * q + 2], [sr, si], rtol=1e-6, atol=1e-9)
    assert np.all(got[:, 8:] == 0)


def _learned_setup(hzlb, n=32, members=64, rank=8, noise=0.0):
    import torch
    cfg = hzlb.Config(n=n, members=members, precision=4, nu=1e-3, noise_sigma=noise, noise_kmax=4)
    e = hzlb.Ensemble(cfg)
    full = _full_fields(hzlb, n, members, 12, 9, decay=0.8)
    e.set_state(full)
    x = torch.from_numpy(e.get_state_compact().view(np.float32).reshape(members, -1).copy()).cuda()
    pod = hzlb.Pod(n, x, rank, seed=2)
    net = hzlb.Mlp(rank, 8, 64, members, seed=4)
    return cfg, e, pod, net


def test_learned_forecast_with_known_networks(hzlb):
    cfg, e, pod, net = _learned_setup(hzlb)
    r = pod.rank
    modes, _ = pod.modes()
    parts = net.unpack(net.params())
    # zero output layer: the window changes nothing but the clock
    parts["W3"][:] = 0
    parts["b3"][:] = 0
    net.set_params(net.pack(parts))
    before = e.get_state_compact()
    t0, s0 = e.time()
    e.learned_forecast(pod, net, 5e-4, 20)
    np.testing.assert_array_equal(e.get_state_compact(), before)
    t1, s1 = e.time()
    assert s1 == s0 + 20 and abs(t1 - (t0 + 20 * 5e-4)) < 1e-15
    # constant output bias c: every member moves by sum_j c_j mode_j
    c = np.linspace(-0.2, 0.3, r).astype(np.float32)
    parts["b3"][:] = c
    net.set_params(net.pack(parts))
    e.learned_forecast(pod, net, 5e-4, 20)
    diff = (e.get_state_compact() - before).view(np.float32).reshape(before.shape[0], -1)
    expect = c.astype(np.float64) @ modes.astype(np.float64)
    np.testing.assert_allclose(diff, np.broadcast_to(expect, diff.shape), rtol=0,
                               atol=2e-6 * np.abs(before.view(np.float32)).max())


def test_learned_forecast_rejects_mismatched_network(hzlb):
    cfg, e, pod, _ = _learned_setup(hzlb)
    wrong = hzlb.Mlp(pod.rank + 1, 8, 64, 64)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.learned_forecast(pod, wrong, 5e-4, 20)
    small = hzlb.Mlp(pod.rank, 8, 64, 16)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.learned_forecast(pod, small, 5e-4, 20)


def test_learned_forecast_adds_the_window_noise(hzlb):
    """With the network output off, a window adds exactly the window's noise increments, and
    those equal the sums of the increments the spectral step would add (Philox restated)."""
    import torch
    cfg, e, pod, net = _learned_setup(hzlb, noise=0.05)
    parts = net.unpack(net.params())
    parts["W3"][:] = 0
    parts["b3"][:] = 0
    net.set_params(net.pack(parts))
    e.set_time(0.0, 100)
    before = e.get_state_compact()
    copy = torch.from_numpy(before.view(np.float32).copy()).cuda()
    hzlb.add_window_noise(cfg, 5e-4, 100, 20, cfg.members, copy.data_ptr())
    e.learned_forecast(pod, net, 5e-4, 20)
    after = e.get_state_compact()
    np.testing.assert_array_equal(after.view(np.float32), copy.cpu().numpy())
    changed = np.flatnonzero(np.any(after != before, axis=0))
    k = (cfg.n - 1) // 3
    ld = 2 * k + 1
    kx, j = changed // ld, changed % ld
    ky = np.where(j <= k, j, j - ld)
    k2 = kx ** 2 + ky ** 2
    assert len(changed) == 28 and k2.min() >= 1 and k2.max() <= 16


def test_window_noise_matches_philox(hzlb, oracle):
    import torch
    cfg = hzlb.Config(n=32, members=3, precision=4, noise_sigma=0.05, noise_kmax=4, seed=5,
                      member_base=7)
    k = (cfg.n - 1) // 3
    ld = 2 * k + 1
    x = torch.zeros((3, 2 * (k + 1) * ld), dtype=torch.float32, device="cuda")
    hzlb.add_window_noise(cfg, 1e-3, 10, 4, 3, x.data_ptr())
    got = x.cpu().numpy().view(np.complex64).reshape(3, k + 1, ld)
    scale = 0.05 * np.sqrt(1e-3) / np.sqrt(2.0)
    x1, x2 = C.c_double(), C.c_double()
    for m in range(3):
        for kx, ky in [(1, -2), (0, 3), (0, -3), (4, 0)]:
            rep = kx > 0 or ky > 0
            code = oracle.lib.ho_mode_code(kx, ky if rep else -ky)
            sr = si = 0.0
            for s in range(10, 14):
                oracle.lib.ho_philox_normal_pair(5, 7 + m, s, code, C.byref(x1), C.byref(x2))
                sr += scale * x1.value
                si += scale * (x2.value if rep else -x2.value)
            np.testing.assert_allclose(got[m, kx, ky % ld], sr + 1j * si, rtol=1e-6, atol=1e-9)
