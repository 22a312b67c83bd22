"""The drop-in drivers for hzl::ensemble, hzl::bootstrap_filter and
hzl::ensemble_kalman_filter against the reference's own CPU library on the same inputs
(FP64 path).  These reuse the reference's own test scenarios (tests/verification.cpp:141-239)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_l2
from oracle.oracle import params6

pytestmark = pytest.mark.gpu


def _p6(p):
    return params6(p.viscosity, p.friction, p.forcing_sigma, p.forcing_tau, p.forcing_min,
                   p.forcing_max)


def test_ensemble_matches_reference(hzlb, reference):
    """hzl::ensemble(16, {}, 0.01, 4, 6, workers, 77) (verification.cpp:160-163) and a 64^2
    case: every diagnostic of every member agrees with the reference's CPU ensemble."""
    for n, steps, count, seed in ((16, 4, 6, 77), (64, 10, 5, 42)):
        p = hzlb.Parameters()
        got = hzlb.ensemble(n, p, 0.01, steps, count, seed)
        ref = reference.ensemble(n, _p6(p), 0.01, steps, count, 3, seed)
        np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=1e-15)
        np.testing.assert_allclose(got[:, 1:5], ref[:, 1:5], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(got[:, 5], ref[:, 5], rtol=1e-11)


def test_ensemble_fp32_error(hzlb, reference):
    p = hzlb.Parameters()
    got = hzlb.ensemble(32, p, 0.01, 10, 4, 5, precision=4)
    ref = reference.ensemble(32, _p6(p), 0.01, 10, 4, 2, 5)
    np.testing.assert_allclose(got[:, 1:3], ref[:, 1:3], rtol=1e-5)


def _dataset(reference, sigma):
    p = params6(0.03, 0.1, sigma, 0.5, 2, 3)
    return reference.synthetic_observations(16, 0.01, 30, 10, p, 0.2, 987), p


def test_particle_filter_deterministic_limit(hzlb, reference):
    """verification.cpp:184-197: sigma = 0, identical particles, no resampling."""
    ds, p6 = _dataset(reference, 0.0)
    p = hzlb.Parameters(0.03, 0.1, 0.0, 0.5, 2, 3)
    got = hzlb.bootstrap_filter(ds, p, 8, 555)
    ref = reference.bootstrap_filter(ds, p6, 8, 555)
    assert got["resampling_events"] == 0 == ref["resampling_events"]
    assert abs(got["log_likelihood"] - ref["log_likelihood"]) < 1e-10
    np.testing.assert_allclose(got["records"], ref["records"], rtol=1e-11)
    for g, r in zip(got["means"], ref["means"]):
        assert rel_l2(g, r) < 1e-12


def test_particle_filter_stochastic_matches_reference(hzlb, reference):
    """sigma = 0.2 with resampling: same log-likelihood, ESS history, resampling events and
    weighted mean fields as the reference's bootstrap_filter (verification.cpp:211-218)."""
    ds, p6 = _dataset(reference, 0.2)
    p = hzlb.Parameters(0.03, 0.1, 0.2, 0.5, 2, 3)
    for particles, seed in ((32, 555), (64, 7)):
        got = hzlb.bootstrap_filter(ds, p, particles, seed)
        ref = reference.bootstrap_filter(ds, p6, particles, seed)
        assert got["resampling_events"] == ref["resampling_events"]
        assert abs(got["log_likelihood"] - ref["log_likelihood"]) < 1e-9 * abs(ref["log_likelihood"])
        np.testing.assert_allclose(got["records"], ref["records"], rtol=1e-9)
        for rec in got["records"]:
            assert 1 - 1e-10 <= rec[2] <= particles + 1e-10
        for g, r in zip(got["means"], ref["means"]):
            assert rel_l2(g, r) < 1e-10


def test_enkf_deterministic_limit_equals_particle_mean(hzlb, reference):
    """verification.cpp:204-210: in the deterministic limit the EnKF mean equals the particle
    filter mean and the spread vanishes."""
    ds, p6 = _dataset(reference, 0.0)
    p = hzlb.Parameters(0.03, 0.1, 0.0, 0.5, 2, 3)
    kal = hzlb.ensemble_kalman_filter(ds, p, 8, 555)
    pf = hzlb.bootstrap_filter(ds, p, 8, 555)
    assert len(kal["records"]) == len(pf["records"])
    for a, b, rec in zip(kal["means"], pf["means"], kal["records"]):
        assert rel_l2(a, b) < 1e-12
        assert rec[2] < 1e-12


@pytest.mark.parametrize("options", [dict(), dict(inflation=1.02, localization_radius=4.0,
                                                  forecast_steps=2, forecast_every=1)])
def test_enkf_matches_reference(hzlb, reference, options):
    """Stochastic serial EnKF with and without inflation/localisation/forecast against the
    reference ensemble_kalman_filter (verification.cpp:219-224 scenario)."""
    ds, p6 = _dataset(reference, 0.2)
    p = hzlb.Parameters(0.03, 0.1, 0.2, 0.5, 2, 3)
    got = hzlb.ensemble_kalman_filter(ds, p, 12, 99, **options)
    ref = reference.enkf(ds, p6, 12, 99, options.get("inflation", 1.0),
                         options.get("localization_radius", 0.0),
                         options.get("forecast_steps", 0), options.get("forecast_every", 1))
    assert got["records"].shape == ref["records"].shape
    np.testing.assert_array_equal(got["records"][:, 0], ref["records"][:, 0])
    np.testing.assert_array_equal(got["records"][:, 3], ref["records"][:, 3])
    np.testing.assert_allclose(got["records"][:, 1:3], ref["records"][:, 1:3], rtol=1e-9)
    for g, r in zip(got["means"], ref["means"]):
        assert rel_l2(g, r) < 1e-10
