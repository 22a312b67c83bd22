"""The Galerkin reduced model (hzlb_galerkin_*) against the reference's own GalerkinModel
(src/reduced.cpp:137-209, through oracle/_ref): right-hand sides and RK4 trajectories to 1e-9
relative, on a POD basis of deterministic 16^2 and 32^2 runs; the reference's rejection of a
stochastic forcing; symmetry of the quadratic tensor."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import params6

pytestmark = pytest.mark.gpu


def _snapshots(hzlb, n, nu, alpha):
    e = hzlb.Ensemble(hzlb.Config(n=n, members=6, precision=8, nu=nu, alpha=alpha))
    e.set_state(np.array([hzlb.grf_spectrum(n, 21, m) for m in range(6)]))
    snaps = [e.get_state()]
    for _ in range(5):
        e.step(0.01, 4)
        snaps.append(e.get_state())
    e.close()
    return np.concatenate(snaps)


@pytest.mark.parametrize("n,rank", [(16, 4), (32, 6)])
def test_galerkin_matches_reference(hzlb, reference, n, rank):
    nu, alpha = 0.01, 0.1
    snaps = _snapshots(hzlb, n, nu, alpha)
    mean, modes, sv, _ = reference.fit_pod(snaps, rank, 0.999999)
    modes = modes.reshape(len(modes), n, n)
    p = hzlb.Parameters(nu, alpha, 0.0, 0.5, 2, 3)
    g = hzlb.GalerkinModel(n, p, mean.reshape(n, n), modes)
    rng = np.random.default_rng(3)
    a = rng.normal(size=(5, len(modes))) * sv[: len(modes)]
    ref_rhs, ref_step = reference.galerkin(n, params6(nu, alpha, 0.0, 0.5, 2, 3), mean, modes, a,
                                           0.01, 5)
    got_rhs = g.rhs(a)
    scale = np.abs(ref_rhs).max()
    np.testing.assert_allclose(got_rhs, ref_rhs, rtol=1e-9, atol=1e-9 * scale)
    got_step = g.step(a, 0.01, 5)
    np.testing.assert_allclose(got_step, ref_step, rtol=1e-9, atol=1e-9 * np.abs(ref_step).max())
    c, A, Q = g.coefficients()
    np.testing.assert_array_equal(Q, Q.transpose(0, 2, 1))


def test_galerkin_rejects_stochastic_forcing(hzlb):
    n = 16
    mean = np.zeros((n, n), complex)
    modes = np.zeros((1, n, n), complex)
    modes[0, 1, 2] = modes[0, n - 1, n - 2] = 0.5
    with pytest.raises(hzlb.HzlbInvalidArgument):
        hzlb.GalerkinModel(n, hzlb.Parameters(0.01, 0.1, 0.2, 0.5, 2, 3), mean, modes)
