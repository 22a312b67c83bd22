"""Device analysis primitives through the C ABI: observation operator, particle weights and
systematic resampling (bit-exact with the oracle given identical weights and uniform), member
gather, inflation, and the batched perturbed-observation EnKF analysis (equal to the
reference's serial scalar update for one observation; equal to the ensemble-space FP64 formula
for many)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import device_synthetic, enkf_weight_matrix, rel_l2
from oracle.oracle import params6

pytestmark = pytest.mark.gpu


def _ensemble(hzlb, n, members, precision=8, seed=3):
    e = hzlb.Ensemble(hzlb.Config(n=n, members=members, precision=precision, nu=1e-3))
    w = np.array([hzlb.grf_spectrum(n, seed, m) for m in range(members)])
    e.set_state(w)
    return e, w


def test_observe_matches_oracle(hzlb, oracle):
    n, members = 32, 4
    e, w = _ensemble(hzlb, n, members)
    xs, ys = np.array([0, 3, 31, 17]), np.array([5, 0, 31, 9])
    got = e.observe(xs, ys)
    for m in range(members):
        phys = oracle.fft(w[m], inverse=True).real
        np.testing.assert_allclose(got[m], phys[ys, xs], rtol=0, atol=1e-14)


def test_device_resampling_bit_exact(hzlb, oracle):
    e, _ = _ensemble(hzlb, 16, 2048, precision=4)
    rng = np.random.default_rng(11)
    for count in (2048,):
        w = rng.random(count) ** 6
        w /= w.sum()
        for u in (0.0, 0.123456789, 1 - 2 ** -53):
            np.testing.assert_array_equal(e.resample(w, u), oracle.systematic_resample(w, u))


def test_pf_weights_on_device_match_oracle(hzlb, oracle):
    e, _ = _ensemble(hzlb, 16, 2)
    rng = np.random.default_rng(3)
    for count in (2, 257, 4096):
        logs = rng.normal(-50, 10, count)
        logs[count // 3] = -np.inf
        w, inc, ess, mw = e.pf_weights(logs)
        w2, inc2, ess2, mw2 = oracle.pf_weights(logs)
        np.testing.assert_allclose(w, w2, rtol=1e-13, atol=0)
        np.testing.assert_allclose([inc, ess, mw], [inc2, ess2, mw2], rtol=1e-13)
    with pytest.raises(hzlb.HzlbError) as err:
        e.pf_weights(np.array([-np.inf, -np.inf]))
    assert err.value.code == hzlb.HZLB_ERUNTIME
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.resample(np.array([0.5, 0.5]), 1.5)


def _pf_reference(oracle, phys, xs, ys, vals, sd, prior):
    """Log-weights in the reference's order (filter.cpp:65-75) from host physical fields."""
    logs = np.where(prior > 0, np.log(np.where(prior > 0, prior, 1)), -np.inf)
    half = 0.5 * np.log(2 * np.pi)
    for o in range(len(xs)):
        r = (phys[:, ys[o], xs[o]] - vals[o]) / sd[o]
        logs = logs - (0.5 * r * r + np.log(sd[o]) + half)
    return logs


@pytest.mark.parametrize("precision", [8, 4])
def test_pf_assimilate_matches_oracle(hzlb, oracle, precision):
    """Device weights, records, resampling and gather of two 24-particle filters against the
    reference's formulas (weights rtol 1e-12; ancestors bit-exact given the device weights)."""
    n, P, S = 32, 24, 2
    M = P * S
    e, w = _ensemble(hzlb, n, M, precision)
    phys = e.physical()
    xs, ys = np.array([1, 7, 30, 12]), np.array([3, 4, 0, 29])
    vals, sd = np.array([0.1, -0.2, 0.05, 0.3]), np.array([0.05, 0.08, 0.1, 0.02])
    e.pf_reset(P)
    before = e.get_state_compact()
    r = e.pf_assimilate(xs, ys, vals, sd, weighted_mean=True)   # no resampling
    logs = _pf_reference(oracle, phys, xs, ys, vals, sd, np.full(M, 1 / P))
    got_w = e.pf_get_weights()
    for s in range(S):
        w2, inc2, ess2, mw2 = oracle.pf_weights(logs[s * P:(s + 1) * P])
        np.testing.assert_allclose(got_w[s * P:(s + 1) * P], w2, rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose([r["increment"][s], r["ess"][s], r["max_weight"][s]],
                                   [inc2, ess2, mw2], rtol=1e-12)
        mean = (got_w[s * P:(s + 1) * P, None] * before[s * P:(s + 1) * P]).sum(axis=0)
        np.testing.assert_allclose(r["mean"][s], mean, rtol=1e-12, atol=1e-14 * np.abs(mean).max())
    assert not r["resampled"].any() and not r["collapsed"].any()
    np.testing.assert_array_equal(r["ancestors"], np.arange(M))
    np.testing.assert_array_equal(e.get_state_compact(), before)
    # the same time again from the same state and weights, now allowed to resample segment 0
    # only: the kernels are deterministic, so the weights equal those above bit for bit
    e.set_state(w)
    e.pf_reset(P)
    u = np.array([0.37, -1.0])
    r2 = e.pf_assimilate(xs, ys, vals, sd, u=u)
    np.testing.assert_array_equal(r2["increment"], r["increment"])
    resampled = r2["ess"] < P / 2
    assert resampled[0], "the test observations must collapse the weights of segment 0"
    np.testing.assert_array_equal(r2["resampled"], [1, 0])
    anc = r2["ancestors"]
    np.testing.assert_array_equal(anc[:P], oracle.systematic_resample(got_w[:P], 0.37))
    np.testing.assert_array_equal(anc[P:], np.arange(P, M))
    np.testing.assert_array_equal(e.get_state_compact(), before[anc])
    np.testing.assert_array_equal(e.pf_get_weights()[:P], np.full(P, 1 / P))
    np.testing.assert_array_equal(e.pf_get_weights()[P:], got_w[P:])
    # an inactive segment is left alone; the other carries its weights into the next time
    r3 = e.pf_assimilate(xs, ys, vals, sd, u=np.array([-1.0, -1.0]), active=[0, 1])
    np.testing.assert_array_equal(e.pf_get_weights()[:P], np.full(P, 1 / P))
    logs3 = _pf_reference(oracle, phys, xs, ys, vals, sd, got_w)[P:]
    _, inc3, ess3, _ = oracle.pf_weights(logs3)
    np.testing.assert_allclose([r3["increment"][1], r3["ess"][1]], [inc3, ess3], rtol=1e-12)


def test_pf_assimilate_collapse(hzlb):
    e, _ = _ensemble(hzlb, 16, 4)
    e.pf_reset(2)
    before = e.get_state_compact()
    # an observation no member can explain makes every log-weight -inf in FP64
    r = e.pf_assimilate([0], [0], [1e300], [1e-300], u=[0.5, 0.5])
    assert r["collapsed"].all() and not r["resampled"].any()
    assert np.isneginf(r["increment"]).all()
    np.testing.assert_array_equal(e.get_state_compact(), before)


def test_gather_members(hzlb):
    n, members = 16, 5
    e, w = _ensemble(hzlb, n, members)
    before = e.get_state_compact()
    anc = np.array([4, 4, 0, 2, 1], np.uint32)
    e.gather(anc)
    np.testing.assert_array_equal(e.get_state_compact(), before[anc])


def test_pf_loglik_matches_reference_formula(hzlb, oracle):
    n, members = 32, 3
    e, w = _ensemble(hzlb, n, members)
    xs, ys = np.array([1, 2]), np.array([3, 4])
    vals, sd = np.array([0.1, -0.2]), np.array([0.3, 0.5])
    lw = e.pf_loglik(xs, ys, vals, sd, np.log(np.full(members, 1 / members)))
    for m in range(members):
        phys = oracle.fft(w[m], inverse=True).real
        v = np.log(1 / members)
        for o in range(2):
            r = (phys[ys[o], xs[o]] - vals[o]) / sd[o]
            v -= 0.5 * r * r + np.log(sd[o]) + 0.5 * np.log(2 * np.pi)
        assert abs(lw[m] - v) < 1e-12 * abs(v)


def test_inflation(hzlb):
    n, members = 16, 6
    e, w = _ensemble(hzlb, n, members)
    c = e.get_state_compact()
    e.inflate(1.05)
    mean = c.mean(axis=0)
    np.testing.assert_allclose(e.get_state_compact(), mean + 1.05 * (c - mean), rtol=1e-13,
                               atol=1e-16)


def test_enkf_single_observation_equals_serial_update(hzlb, oracle):
    """One scalar observation: the batched analysis equals the reference's serial update
    (filter.cpp:265-321), restated by the oracle, given the same perturbations."""
    n, members = 32, 16
    e, w = _ensemble(hzlb, n, members)
    xs, ys = np.array([7]), np.array([11])
    value, sd = np.array([0.05]), np.array([0.2])
    eps = np.random.default_rng(2).normal(size=(members, 1))
    pred = e.observe(xs, ys)[:, 0]
    solvers = []
    for m in range(members):
        s = oracle.solver(n, params6(1e-3, 0.0, 0.0, 0.5, 2, 3), 0)
        s.set_state(w[m], np.zeros((n, n), np.complex128))
        solvers.append(s)
    import ctypes as C
    arr = (C.c_void_p * members)(*[s.h.value for s in solvers])
    pred_c = np.ascontiguousarray(pred)
    eps_c = np.ascontiguousarray(eps[:, 0])
    oracle.check(oracle.lib.ho_enkf_scalar_update(members, arr, pred_c.ctypes.data_as(C.POINTER(C.c_double)),
                                                  float(value[0]), float(sd[0]),
                                                  eps_c.ctypes.data_as(C.POINTER(C.c_double))))
    e.enkf_analysis(xs, ys, value, sd, eps)
    got = e.get_state()
    for m in range(members):
        assert rel_l2(got[m], solvers[m].state()[0]) < 1e-12


@pytest.mark.parametrize("members,p", [(48, 64), (150, 200), (70, 333)])
@pytest.mark.parametrize("precision,tol", [(8, 1e-11), (4, 2e-5)])
def test_enkf_batch_many_observations(hzlb, precision, tol, members, p):
    """p observations at once against X + A W with W from the FP64 ensemble-space formula
    (one, several and ragged Cholesky blocks of 64)."""
    n = 64
    e, w = _ensemble(hzlb, n, members, precision=precision)
    rng = np.random.default_rng(9)
    xs, ys = rng.integers(0, n, p), rng.integers(0, n, p)
    vals, sd = rng.normal(0, 0.1, p), np.full(p, 0.1)
    eps = rng.normal(size=(members, p))
    hx = e.observe(xs, ys)
    x = e.get_state_compact().astype(np.complex128)
    W = enkf_weight_matrix(hx, vals, sd, eps)
    expect = x + ((x - x.mean(axis=0)).T @ W).T
    e.enkf_analysis(xs, ys, vals, sd, eps)
    got = e.get_state_compact().astype(np.complex128)
    assert rel_l2(got, expect) < tol
    # the analysis pulls the ensemble mean towards the observations
    after = e.observe(xs, ys).mean(axis=0)
    assert np.linalg.norm(after - vals) < np.linalg.norm(hx.mean(axis=0) - vals)


def _nis_reference(hx, vals, sd):
    M = hx.shape[0]
    ha = hx - hx.mean(axis=0)
    S = ha.T @ ha / (M - 1) + np.diag(sd ** 2)
    d = vals - hx.mean(axis=0)
    return float(d @ np.linalg.solve(S, d) / len(vals))


def test_innovation_statistic_and_rejection(hzlb):
    """The normalised innovation statistic against numpy; above the limit the state is left
    unchanged."""
    n, members, p = 64, 96, 150
    e, w = _ensemble(hzlb, n, members, precision=8)
    rng = np.random.default_rng(4)
    xs, ys = rng.integers(0, n, p), rng.integers(0, n, p)
    sd = np.full(p, 0.1)
    eps = rng.normal(size=(members, p))
    for scale in (0.0, 5.0):
        hx = e.observe(xs, ys)
        vals = hx.mean(axis=0) + scale * rng.normal(size=p)
        expect = _nis_reference(hx, vals, sd)
        before = e.get_state_compact()
        nis, applied = e.enkf_analysis_nis(xs, ys, vals, sd, eps, nis_limit=3.0)
        assert abs(nis - expect) < 1e-9 * max(1.0, expect)
        if expect > 3.0:
            assert not applied
            np.testing.assert_array_equal(e.get_state_compact(), before)
        else:
            assert applied


@pytest.mark.parametrize("precision,tol", [(8, 1e-11), (4, 2e-5)])
def test_device_perturbations_match_philox(hzlb, oracle, precision, tol):
    """Perturbations drawn on the device equal the Philox draws restated by the oracle, so the
    analysis equals the host-perturbation analysis with those draws."""
    import ctypes as C
    n, members, p = 32, 40, 70
    seed, cycle = 1234, 7
    a, w = _ensemble(hzlb, n, members, precision=precision)
    b, _ = _ensemble(hzlb, n, members, precision=precision)
    rng = np.random.default_rng(5)
    xs, ys = rng.integers(0, n, p), rng.integers(0, n, p)
    vals, sd = rng.normal(0, 0.1, p), np.full(p, 0.2)
    eps = np.zeros((members, p))
    x1, x2 = C.c_double(), C.c_double()
    for m in range(members):
        for o in range(0, p, 2):
            oracle.lib.ho_philox_normal_pair(seed, m, cycle ^ (0x454E4B46 << 32), o >> 1,
                                             C.byref(x1), C.byref(x2))
            eps[m, o] = x1.value
            if o + 1 < p:
                eps[m, o + 1] = x2.value
    na, _ = a.enkf_analysis_nis(xs, ys, vals, sd, None, seed=seed, cycle=cycle)
    nb_, _ = b.enkf_analysis_nis(xs, ys, vals, sd, eps)
    assert abs(na - nb_) < 1e-12 * max(1.0, abs(nb_))
    assert rel_l2(a.get_state_compact().astype(np.complex128),
                  b.get_state_compact().astype(np.complex128)) < tol


@pytest.mark.parametrize("precision", [4, 8])
@pytest.mark.parametrize("points", ["sparse", "scattered", "strided", "all rows"])
def test_observation_rows_equal_the_physical_field(hzlb, precision, points):
    """The observation operator transforms only the row pairs its points lie in; every value
    is the full physical field's, bit for bit, for any point set."""
    n, members = 64, 5
    e = device_synthetic(hzlb, n, members, precision, 1e-3, 0.05, 3)
    e.step(1e-3, 3)
    rng = np.random.default_rng(4)
    if points == "sparse":
        xs, ys = np.array([3, 17, 63]), np.array([0, 0, 63])
    elif points == "scattered":
        xs, ys = rng.integers(0, n, 40), rng.integers(0, n, 40)
    elif points == "strided":
        g = np.arange(0, n, 8)
        xs, ys = np.tile(g, len(g)), np.repeat(g, len(g))
    else:
        xs, ys = rng.integers(0, n, 3 * n), np.arange(3 * n) % n
    got = e.observe(xs, ys)
    phys = e.physical()
    assert np.array_equal(got, phys[:, ys, xs])
    e.close()
