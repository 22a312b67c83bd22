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
