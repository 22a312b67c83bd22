"""hzl::particle_log_likelihood and hzl::averaged_particle_log_likelihood (src/filter.cpp:141-165)
against the reference's own CPU library on the reference's synthetic stochastic dataset.

The host-side exits (prior support, explicit diffusion bound, replicate count) need no GPU; the
likelihood values themselves come from the batched ensemble of replicates x particles members
and run on the device."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.oracle import params6

TRUE_Q = np.log([0.03, 0.1, 0.2, 0.5])


def _dataset(reference):
    p6 = params6(0.03, 0.1, 0.2, 0.5, 2, 3)
    return reference.synthetic_observations(16, 0.01, 30, 10, p6, 0.2, 987)


@pytest.mark.parametrize("q", [
    [0.5, np.log(0.1), np.log(0.2), np.log(0.5)],       # log nu above the prior's support
    [np.log(0.03), -11.0, np.log(0.2), np.log(0.5)],    # log alpha below it
    [np.log(0.03), np.log(0.1), 2.5, np.log(0.5)],      # log sigma above it
    [np.log(0.03), np.log(0.1), np.log(0.2), np.nan],   # nonfinite
])
def test_outside_prior_is_minus_infinity(hzlb, reference, q):
    ds = _dataset(reference)
    assert hzlb.particle_log_likelihood(ds, q, 16, 5) == -math.inf
    assert reference.particle_log_likelihood(ds, q, 16, 5) == -math.inf
    assert hzlb.averaged_particle_log_likelihood(ds, q, 16, 3, 5) == -math.inf
    assert reference.particle_log_likelihood(ds, q, 16, 5, replicates=3) == -math.inf


def test_diffusion_bound_is_minus_infinity(hzlb, reference):
    """dt (2 nu K^2 + alpha) > 2.5 rejects the parameters before any member is stepped."""
    ds = dict(_dataset(reference), dt=5.0)
    assert hzlb.particle_log_likelihood(ds, TRUE_Q, 16, 5) == -math.inf
    assert reference.particle_log_likelihood(ds, TRUE_Q, 16, 5) == -math.inf
    assert hzlb.averaged_particle_log_likelihood(ds, TRUE_Q, 16, 2, 5) == -math.inf


def test_argument_errors(hzlb, reference):
    ds = _dataset(reference)
    with pytest.raises(hzlb.HzlbInvalidArgument, match="at least one replicate"):
        hzlb.averaged_particle_log_likelihood(ds, TRUE_Q, 16, 0, 5)
    with pytest.raises(Exception, match="at least one replicate"):
        reference.particle_log_likelihood(ds, TRUE_Q, 16, 5, replicates=0)
    with pytest.raises(hzlb.HzlbInvalidArgument, match="log\\(nu\\)"):
        hzlb.particle_log_likelihood(ds, TRUE_Q[:3], 16, 5)


@pytest.mark.gpu
@pytest.mark.parametrize("particles,seed", [(32, 555), (64, 7)])
def test_particle_log_likelihood_matches_reference(hzlb, reference, particles, seed):
    ds = _dataset(reference)
    got = hzlb.particle_log_likelihood(ds, TRUE_Q, particles, seed)
    ref = reference.particle_log_likelihood(ds, TRUE_Q, particles, seed)
    assert math.isfinite(ref)
    assert abs(got - ref) < 1e-9 * abs(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("particles,replicates,seed", [(32, 4, 11), (16, 8, 3)])
def test_averaged_particle_log_likelihood_matches_reference(hzlb, reference, particles,
                                                            replicates, seed):
    """Every replicate of the batched ensemble reproduces the reference's sequential
    bootstrap_filter(data, p, particles, stream_seed(seed, r)), so the log-mean-exp agrees."""
    ds = _dataset(reference)
    got = hzlb.averaged_particle_log_likelihood(ds, TRUE_Q, particles, replicates, seed)
    ref = reference.particle_log_likelihood(ds, TRUE_Q, particles, seed, replicates=replicates)
    assert math.isfinite(ref)
    assert abs(got - ref) < 1e-9 * abs(ref)


@pytest.mark.gpu
def test_single_replicate_is_the_plain_likelihood(hzlb, reference):
    ds = _dataset(reference)
    q = np.log([0.05, 0.2, 0.3, 0.4])
    one = hzlb.averaged_particle_log_likelihood(ds, q, 24, 1, 99)
    plain = hzlb.particle_log_likelihood(ds, q, 24, reference.stream_seed(99, 0))
    assert abs(one - plain) < 1e-12 * abs(plain)
    assert abs(plain - reference.particle_log_likelihood(ds, q, 24, reference.stream_seed(99, 0))) \
        < 1e-9 * abs(plain)
