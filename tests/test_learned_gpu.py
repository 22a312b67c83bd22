"""The learned reduced forecast end to end at a reduced size (64^2, 128 members): transitions
generated by the solver, POD, network training, and the EnKF twin experiment.

* the trained network predicts the one-window drift of the POD coefficients far better than
  persistence (what the method does without the network) on held-out windows;
* every forecast variant keeps the filter finite and consistent, and the hybrid (spectral
  mean, learned anomalies) stays close to the spectral filter;
* in the complement variant (the network moves every POD coefficient, the spectral step of the
  mean supplies only the motion outside the POD space) switching the network off makes the
  filter worse: the network carries the forecast there;
* with an innovation-statistic limit below every statistic, the learned filter falls back to
  the spectral forecast on every cycle and then reproduces the spectral filter exactly.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small():
    from hzl_stochasticflowinference_b200 import learned
    return learned, learned.TwinConfig(
        n=64, nu=1e-3, dt=1e-3, window=10, spinup_steps=500, snapshots=400, snapshot_members=20,
        rank=16, hidden=128, train_members=512, train_windows=20, epochs=15, batch=256,
        members=128, obs_stride=4, cycles=10)


@pytest.fixture(scope="module")
def experiment(hzlb):
    learned, tc = _small()
    return tc, learned.run(tc)


def test_network_beats_persistence(experiment):
    tc, out = experiment
    assert out["transitions"] == tc.train_members * tc.train_windows
    assert out["pod"]["captured"] > 0.8 and out["pod"]["residual"] < 1e-6
    t = out["training"]
    assert t["val_mse_network"] < 0.5 * t["val_mse_persistence"], t


def test_twin_variants_are_consistent(experiment):
    tc, out = experiment
    spectral = out["spectral"]
    assert np.all(np.isfinite(spectral["rmse"]))
    assert spectral["mean_rmse"] < 0.5 * spectral["initial_rmse"]
    for mode in ("learned", "hybrid", "complement", "persistence", "hybrid_persistence",
                 "complement_persistence"):
        o = out[mode]
        assert np.all(np.isfinite(o["rmse"])) and len(o["rmse"]) == tc.cycles
        assert 0 <= o["fallback_cycles"] <= tc.cycles
        assert np.all(np.asarray(o["nis"]) > 0)
    assert out["hybrid"]["mean_rmse"] < 1.25 * spectral["mean_rmse"]
    assert out["complement"]["mean_rmse"] < out["complement_persistence"]["mean_rmse"]
    assert out["rmse_ratio"] == out["complement"]["rmse_ratio"]


def test_fallback_on_every_cycle_reproduces_the_spectral_filter(hzlb, experiment):
    import dataclasses
    learned, _ = _small()
    tc, _out = experiment
    strict = dataclasses.replace(tc, cycles=4, nis_limit=1e-12, epochs=1, train_members=256,
                                 train_windows=4)
    base = learned.spinup(strict)
    truth = learned.truth_run(strict, base)
    import torch
    snaps = learned.snapshots(strict, base)
    pod = hzlb.Pod(strict.n, snaps, strict.rank, seed=1)
    X, Y = learned.transitions(strict, base, pod)
    net, _ = learned.train(strict, X, Y)
    spec = learned.twin(strict, base, truth, "spectral")
    fb = learned.twin(strict, base, truth, "learned", pod, net)
    assert fb["fallback_cycles"] == strict.cycles
    assert fb["rmse"] == spec["rmse"]
    assert fb["nis"] == spec["nis"]
