"""hzl::synthetic_observations (src/inference.cpp:258-288) with the truth run on the device,
against the reference library's own function and its CPU Solver on the same inputs: the same
observation sites, steps and uncertainties, values equal to FP64 roundoff (the noise draws are
the reference's NormalStream exactly), and truth fields equal to the reference Solver's
physical vorticity."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_l2
from oracle.oracle import params6

pytestmark = pytest.mark.gpu

CASES = [
    # n, dt, steps, every, (nu, alpha, sigma, tau, kmin, kmax), noise, seed
    (16, 0.01, 150, 10, (0.03, 0.1, 0.2, 0.5, 2, 3), 0.02, 314159),   # the reference's default
    (64, 0.005, 60, 20, (0.01, 0.1, 0.2, 0.5, 2, 4), 0.05, 7),
    (32, 0.01, 40, 10, (0.02, 0.1, 0.0, 0.5, 2, 3), 0.1, 3),           # deterministic truth
]


@pytest.mark.parametrize("case", CASES)
def test_matches_reference(hzlb, reference, case):
    n, dt, steps, every, p, noise, seed = case
    got = hzlb.synthetic_observations(n, hzlb.Parameters(*p), dt, steps, every, noise, seed)
    ref = reference.synthetic_observations(n, dt, steps, every, params6(*p), noise, seed)
    for key in ("n", "stochastic", "forcing_min", "forcing_max"):
        assert int(got[key]) == int(ref[key]), key
    assert got["dt"] == ref["dt"]
    assert len(got["steps"]) == 8 * (steps // every)
    for key in ("steps", "x", "y", "sd"):
        np.testing.assert_array_equal(got[key], ref[key])
    np.testing.assert_allclose(got["value"], ref["value"], rtol=0, atol=1e-11)


def test_truth_fields_match_reference_solver(hzlb, reference):
    n, dt, steps, every, p, noise, seed = CASES[1]
    ds, fields = hzlb.synthetic_observations(n, hzlb.Parameters(*p), dt, steps, every, noise,
                                             seed, truth_fields=True)
    solver = reference.solver(n, params6(*p), reference.stream_seed(seed, 0))
    solver.initialize("multimode")
    for g in range(steps // every):
        solver.step(dt, every)
        truth = np.real(solver.physical_vorticity()).reshape(n, n)
        assert rel_l2(fields[g], truth) <= 1e-12
        # the observations sit on the truth field plus noise
        idx = slice(8 * g, 8 * g + 8)
        resid = ds["value"][idx] - truth[ds["y"][idx], ds["x"][idx]]
        assert np.all(np.abs(resid) < 6 * noise)


def test_round_trip_through_a_dataset_file(hzlb, reference, tmp_path):
    n, dt, steps, every, p, noise, seed = CASES[0]
    ds = hzlb.synthetic_observations(n, hzlb.Parameters(*p), dt, steps, every, noise, seed)
    hzlb.save_dataset(ds, tmp_path / "obs.csv")
    back = reference.dataset_load(tmp_path / "obs.csv")
    np.testing.assert_array_equal(back["value"], ds["value"])
    np.testing.assert_array_equal(back["steps"], ds["steps"])


@pytest.mark.parametrize("steps,every,noise", [(10, 0, 0.1), (5, 10, 0.1), (20, 10, 0.0),
                                               (20, 10, float("nan"))])
def test_invalid_experiment(hzlb, reference, steps, every, noise):
    p = (0.03, 0.1, 0.2, 0.5, 2, 3)
    with pytest.raises(hzlb.HzlbInvalidArgument) as ours:
        hzlb.synthetic_observations(16, hzlb.Parameters(*p), 0.01, steps, every, noise, 1)
    with pytest.raises(Exception) as theirs:
        reference.synthetic_observations(16, 0.01, steps, every, params6(*p), noise, 1)
    assert str(ours.value) == str(theirs.value)
