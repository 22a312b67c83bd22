"""Batched tangent and adjoint drifts (hzlb_linearized_drift / hzlb_adjoint_drift) against the
reference library's own hzl::Solver::linearized_drift and Solver::adjoint_drift
(src/solver.cpp:264-324) on the same projected fields, FP64: relative L2 <= 1e-12 per pair, and
the transpose identity <l, J d> = <J^T l, d> (Re sum conj(a) b over the spectrum, the reference's
own) on the device results."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_l2
from oracle.oracle import params6

pytestmark = pytest.mark.gpu

P = (0.02, 0.1, 0.2, 0.5, 2, 3)


def _fields(n, count, seed, scale=1.0):
    """Spectra of random real fields, projected onto the active modes (forward / n^2)."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n, 1 / n).astype(int)
    mask = (3 * np.abs(k)[None, :] < n) & (3 * np.abs(k)[:, None] < n)
    mask[0, 0] = False
    return np.stack([scale * np.fft.fft2(rng.normal(size=(n, n))) / n ** 2 * mask
                     for _ in range(count)])


def _ip(a, b):
    return float(np.real(np.vdot(a, b)))


@pytest.mark.parametrize("n,count", [(16, 3), (64, 5), (128, 2), (256, 1)])
def test_linearized_drift_matches_reference(hzlb, reference, n, count):
    w, d = _fields(n, count, 1), _fields(n, count, 2, 0.1)
    got = hzlb.linearized_drift(n, hzlb.Parameters(*P), w, d)
    s = reference.solver(n, params6(*P), 5)
    for i in range(count):
        assert rel_l2(got[i], s.linearized_drift(w[i], d[i])) <= 1e-12


@pytest.mark.parametrize("n,count", [(16, 3), (64, 5), (128, 2), (256, 1)])
def test_adjoint_drift_matches_reference(hzlb, reference, n, count):
    w, lam = _fields(n, count, 3), _fields(n, count, 4, 10.0)
    got = hzlb.adjoint_drift(n, hzlb.Parameters(*P), w, lam)
    s = reference.solver(n, params6(*P), 5)
    for i in range(count):
        assert rel_l2(got[i], s.adjoint_drift(w[i], lam[i])) <= 1e-12


def test_adjoint_is_the_transpose_of_the_tangent(hzlb):
    n, count = 64, 4
    p = hzlb.Parameters(*P)
    w, d, lam = _fields(n, count, 5), _fields(n, count, 6), _fields(n, count, 7)
    jd = hzlb.linearized_drift(n, p, w, d)
    jtl = hzlb.adjoint_drift(n, p, w, lam)
    for i in range(count):
        a, b = _ip(lam[i], jd[i]), _ip(jtl[i], d[i])
        assert abs(a - b) <= 1e-12 * max(abs(a), abs(b))


def test_solver_states_and_large_batches(hzlb, reference):
    """States of a running reference solver (not random fields), 40 pairs in one call."""
    n = 32
    s = reference.solver(n, params6(*P), 9)
    s.initialize("multimode")
    states = []
    for _ in range(40):
        s.step(0.01, 3)
        states.append(s.coefficients())
    w = np.stack(states)
    d = _fields(n, 40, 8)
    got_t = hzlb.linearized_drift(n, hzlb.Parameters(*P), w, d)
    got_a = hzlb.adjoint_drift(n, hzlb.Parameters(*P), w, d)
    for i in (0, 17, 39):
        assert rel_l2(got_t[i], s.linearized_drift(w[i], d[i])) <= 1e-12
        assert rel_l2(got_a[i], s.adjoint_drift(w[i], d[i])) <= 1e-12


def test_invalid_arguments(hzlb):
    p = hzlb.Parameters(*P)
    w = _fields(16, 1, 1)
    with pytest.raises(hzlb.HzlbInvalidArgument, match="power of two"):
        hzlb.linearized_drift(12, p, np.zeros((1, 12, 12)), np.zeros((1, 12, 12)))
    with pytest.raises(hzlb.HzlbInvalidArgument, match="size mismatch"):
        hzlb.adjoint_drift(16, p, w, np.zeros((2, 16, 16)))
    bad = w.copy()
    bad[0, 1, 1] = np.nan
    with pytest.raises(hzlb.HzlbInvalidArgument, match="nonfinite"):
        hzlb.linearized_drift(16, p, bad, w)


def _deterministic_dataset(reference, n=16, steps=30, every=10, seed=271):
    p6 = params6(0.03, 0.1, 0.0, 0.5, 2, 3)
    return reference.synthetic_observations(n, 0.01, steps, every, p6, 0.05, seed)


@pytest.mark.parametrize("stride", [1, 7, 20])
def test_likelihood_adjoint_matches_reference(hzlb, reference, stride):
    """Value, gradient and counters of the reference's likelihood_adjoint for several
    parameter vectors in one call (src/adjoint.cpp:43-161)."""
    ds = _deterministic_dataset(reference)
    qs = np.array([[np.log(0.03), np.log(0.1)], [np.log(0.05), np.log(0.2)],
                   [np.log(0.01), np.log(0.05)], [-0.5, -3.0]])
    got = hzlb.likelihood_adjoint(ds, qs, stride)
    for q, g in zip(qs, got):
        ref = reference.likelihood_adjoint(ds, q, stride)
        assert abs(g["value"] - ref["value"]) <= 1e-11 * abs(ref["value"])
        np.testing.assert_allclose(g["gradient"], ref["gradient"], rtol=1e-9, atol=1e-12)
        for key in ("checkpoint_fields", "peak_block_fields", "replayed_steps"):
            assert g[key] == ref[key], key


def test_likelihood_adjoint_gradient_by_differences(hzlb, reference):
    """The gradient is the derivative of the device objective (central differences)."""
    ds = _deterministic_dataset(reference, n=32, steps=40, every=10)
    q = np.array([np.log(0.02), np.log(0.08)])
    h = 1e-5
    pts = [q, q + [h, 0], q - [h, 0], q + [0, h], q - [0, h]]
    res = hzlb.likelihood_adjoint(ds, np.array(pts), 10)
    fd = [(res[1]["value"] - res[2]["value"]) / (2 * h), (res[3]["value"] - res[4]["value"]) / (2 * h)]
    np.testing.assert_allclose(res[0]["gradient"], fd, rtol=1e-5)


def test_likelihood_adjoint_exits(hzlb, reference):
    ds = _deterministic_dataset(reference)
    got = hzlb.likelihood_adjoint(ds, [[0.5, -1.0], [-1.0, np.nan], [-13.0, -1.0]], 5)
    for g in got:
        assert g["value"] == np.inf and list(g["gradient"]) == [0, 0]
        assert reference.likelihood_adjoint(ds, [0.5, -1.0], 5)["value"] == np.inf
    # past the explicit diffusion bound
    big = dict(ds, dt=1.0)
    assert hzlb.likelihood_adjoint(big, [[-1.0, -1.0]], 5)[0]["value"] == np.inf
    assert reference.likelihood_adjoint(big, [-1.0, -1.0], 5)["value"] == np.inf
    with pytest.raises(hzlb.HzlbInvalidArgument, match="positive checkpoint stride"):
        hzlb.likelihood_adjoint(ds, [[-1.0, -1.0]], 0)
    with pytest.raises(hzlb.HzlbInvalidArgument, match="deterministic data"):
        hzlb.likelihood_adjoint(dict(ds, stochastic=1), [[-1.0, -1.0]], 5)
