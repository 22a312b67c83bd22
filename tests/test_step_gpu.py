"""Parity of the batched B200 RK4 step with the CPU oracle (through the C ABI).

Bars: FP64 relative L2 <= 1e-12 on the vorticity spectrum against the FP64 oracle; the FP32
path's error against the same oracle is bounded explicitly below.  The reference-physics
cases (OU forcing uploaded per step, friction) follow the reference's own GPU parity method
(src/cuda_benchmark.cpp:37-80: host ShellForcing midpoint forcing, rel-L2 gate 1e-9)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import device_synthetic, oracle_synthetic_run, rel_l2
from oracle.oracle import params6

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


@pytest.mark.parametrize("n", [8, 16, 32, 64, 128, 256])
def test_fp64_synthetic_parity(hzlb, oracle, n):
    members, steps, dt, nu, sigma, seed = 3, 6, 1e-3, 1e-3, 0.05, 7
    kmax = min(4, (n - 1) // 3)
    ref, _ = oracle_synthetic_run(oracle, n, members, steps, dt, nu, sigma, seed,
                                  wavenumber=kmax, noise_kmax=kmax)
    e = device_synthetic(hzlb, n, members, 8, nu, sigma, seed, wavenumber=kmax, noise_kmax=kmax)
    e.step(dt, steps)
    assert e.status() == 0
    got = e.get_state()
    for m in range(members):
        assert rel_l2(got[m], ref[m]) <= FP64_TOL, (n, m, rel_l2(got[m], ref[m]))


def test_fp64_512_parity(hzlb, oracle):
    n, steps, dt, nu, sigma, seed = 512, 2, 5e-4, 2e-4, 0.05, 3
    ref, _ = oracle_synthetic_run(oracle, n, 1, steps, dt, nu, sigma, seed)
    e = device_synthetic(hzlb, n, 1, 8, nu, sigma, seed)
    e.step(dt, steps)
    assert rel_l2(e.get_state()[0], ref[0]) <= FP64_TOL


def test_config0_fp64_1000_steps(hzlb, oracle):
    """N=64, nu=1e-3, Kolmogorov 0.1 sin(4y), sigma=0.05 EM noise on 1<=|k|<=4, dt=1e-3,
    1000 steps, GRF initial field: final vorticity and the energy/enstrophy series."""
    n, steps, dt, nu, sigma, seed = 64, 1000, 1e-3, 1e-3, 0.05, 42
    ref, series = oracle_synthetic_run(oracle, n, 1, steps, dt, nu, sigma, seed)
    e = device_synthetic(hzlb, n, 1, 8, nu, sigma, seed)
    got_series = []
    for i in range(steps):
        e.step(dt, 1)
        if i % 100 == 99:
            d = e.diagnostics()[0]
            got_series.append((d[1], d[2]))
    assert e.status() == 0
    assert rel_l2(e.get_state()[0], ref[0]) <= FP64_TOL
    np.testing.assert_allclose(np.array(got_series), series[99::100], rtol=1e-12)


# Config 1 (256 members at 128^2, nu = dt = 5e-4, 2000 steps): the FP32-against-FP64 maxima
# over the 256 members after 2000 steps measured 1.67e-6 (relative L2) and 1.31e-6 (enstrophy
# drift) on a B200, growing about linearly in time; the bounds asserted here leave 3x margin.
CONFIG1_L2_BOUND = 5e-6
CONFIG1_ENSTROPHY_BOUND = 5e-6


def _config1(hzlb, precision, members=256):
    e = device_synthetic(hzlb, 128, members, precision, 5e-4, 0.05, 42)
    return e


def test_config1_fp64_2000_steps_against_reference(hzlb, reference):
    """The FP64 path over config 1's 2000 steps equals the reference's own CPU Solver driven
    with the same forcing, noise and initial fields (its update_latent_state + step) within
    1e-12 relative L2, for the first four members of the 256-member ensemble."""
    n, steps, dt, nu = 128, 2000, 5e-4, 5e-4
    e = _config1(hzlb, 8)
    e.step(dt, steps)
    assert e.status() == 0
    got = e.get_state()
    e.close()
    ref = reference.synthetic_ensemble(n, nu, dt, steps, 4, 4, 42)
    for m in range(4):
        assert rel_l2(got[m], ref[m]) <= FP64_TOL, (m, rel_l2(got[m], ref[m]))


def test_config1_fp32_error_statement(hzlb):
    """Config 1 in FP32 against the same run in FP64 (identical fields and Philox noise): every
    member's relative L2 error and enstrophy drift after 2000 steps stay within the stated
    bounds, and both grow with time (no step leaves a jump)."""
    steps, every, dt = 2000, 500, 5e-4
    a, b = _config1(hzlb, 4), _config1(hzlb, 8)
    K = (128 - 1) // 3
    w = np.full(b.compact_size, 2.0)
    w[:2 * K + 1] = 1.0
    worst = []
    for _ in range(steps // every):
        a.step(dt, every)
        b.step(dt, every)
        x = a.get_state_compact().astype(np.complex128)
        y = b.get_state_compact()
        zx, zy = (w * np.abs(x) ** 2).sum(axis=1), (w * np.abs(y) ** 2).sum(axis=1)
        err = np.sqrt((w * np.abs(x - y) ** 2).sum(axis=1) / zy)
        worst.append((err.max(), np.abs(zx / zy - 1).max()))
    assert a.status() == 0 and b.status() == 0
    a.close()
    b.close()
    print("config1 FP32 vs FP64 (max rel L2, max enstrophy drift) per 500 steps:", worst)
    assert worst[-1][0] < CONFIG1_L2_BOUND
    assert worst[-1][1] < CONFIG1_ENSTROPHY_BOUND
    assert worst[-1][0] >= worst[0][0] * 0.5


@pytest.mark.parametrize("precision", [4, 8])
def test_checked_step_leaves_state_on_cfl_violation(hzlb, precision):
    """hzlb_step_checked: a step whose stage-1 velocities break the CFL limit is undone
    (state, clock, noise counter), and the next step equals a fresh ensemble's."""
    n, members, seed = 64, 3, 5
    a = device_synthetic(hzlb, n, members, precision, 1e-3, 0.05, seed)
    b = device_synthetic(hzlb, n, members, precision, 1e-3, 0.05, seed)
    before = a.get_state_compact()
    rate = a.diagnostics()[:, 5].max()
    with pytest.raises(hzlb.HzlbError) as err:
        a.step_checked(0.75 / rate)
    assert err.value.code == hzlb.HZLB_ERUNTIME and "CFL" in str(err.value)
    np.testing.assert_array_equal(a.get_state_compact(), before)
    assert a.status() == 0
    a.step_checked(0.1 / rate)
    b.step(0.1 / rate, 1)
    np.testing.assert_array_equal(a.get_state_compact(), b.get_state_compact())
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [4, 8])
def test_bounded_wait_runs_out_and_the_context_stays_usable(hzlb, precision):
    """Failure detection without a GPU fault: the test hook leaves one block's first tile copy
    unissued, so its mbarrier never completes with nothing in flight; the bounded wait gives up
    after about a second, the step reports STATUS_TIMEOUT, and the same context then steps
    exactly as a fresh ensemble does."""
    import time
    n, members, seed, dt = 64, 8, 3, 1e-3
    a = device_synthetic(hzlb, n, members, precision, 1e-3, 0.05, seed)
    a.inject_wait_timeout()
    t0 = time.perf_counter()
    a.step(dt, 1)
    status = a.status()
    assert status & hzlb.STATUS_TIMEOUT, status
    assert time.perf_counter() - t0 < 30
    assert a.status() == 0   # read and cleared
    # the ensemble that timed out, restarted, and a fresh one agree bit for bit
    a.set_state(np.array([hzlb.grf_spectrum(n, seed, m) for m in range(members)]))
    a.set_time(0.0, 0)
    b = device_synthetic(hzlb, n, members, precision, 1e-3, 0.05, seed)
    a.step(dt, 3)
    b.step(dt, 3)
    assert a.status() == 0 and b.status() == 0
    np.testing.assert_array_equal(a.get_state_compact(), b.get_state_compact())
    a.close()
    b.close()


def test_fp32_error_against_fp64_oracle(hzlb, oracle):
    """FP32 path (complex64 spectra): stated error bound against the FP64 oracle."""
    n, members, steps, dt, nu, sigma, seed = 128, 2, 100, 5e-4, 5e-4, 0.05, 11
    ref, _ = oracle_synthetic_run(oracle, n, members, steps, dt, nu, sigma, seed)
    e = device_synthetic(hzlb, n, members, 4, nu, sigma, seed)
    e.step(dt, steps)
    got = e.get_state()
    for m in range(members):
        err = rel_l2(got[m], ref[m])
        assert err < 2e-5, err
        z_ref = np.sum(np.abs(ref[m]) ** 2)
        z_got = np.sum(np.abs(got[m]) ** 2)
        assert abs(z_got / z_ref - 1) < 2e-5


@pytest.mark.parametrize("precision", [4, 8])
def test_reference_physics_ou_forcing(hzlb, oracle, reference, precision):
    """Reference physics (nu, alpha, OU shell forcing frozen at the midpoint) with the forcing
    generated by the reference's own ShellForcing and uploaded per step, against the
    reference Solver (cuda_benchmark.cpp:41-80 method)."""
    n, steps, dt = 32, 10, 0.005
    p = params6(0.01, 0.1, 0.2, 0.5, 2, 3)
    solver = reference.solver(n, p, 0)
    solver.initialize("multimode")
    initial = solver.coefficients()
    sf = reference.shell_forcing(n, p, 0)
    cfg = hzlb.Config(n=n, members=1, precision=precision, nu=0.01, alpha=0.1, forcing_kmax=3,
                      forcing_per_member=True)
    e = hzlb.Ensemble(cfg)
    e.set_state(initial[None])
    for _ in range(steps):
        e.set_forcing(sf.midpoint_step(dt)[None])
        e.step(dt, 1)
    cpu = reference.solver(n, p, 0)
    cpu.initialize("multimode")
    # The reference's CPU Solver draws its own OU path from the same seed (Solver(n, p, 0) and
    # ShellForcing(n, p, 0) share NormalStream(0), tests/verification.cpp:334-350).
    cpu.step(dt, steps)
    tol = 1e-12 if precision == 8 else 1e-5
    assert rel_l2(e.get_state()[0], cpu.coefficients()) <= tol


def test_deterministic_gpu_step_matches_cuda_solver_semantics(hzlb, reference):
    """CudaSolver::step(dt) with sigma = 0 (cuda_solver.cu:173-183): no forcing."""
    n, steps, dt = 64, 20, 0.005
    p = params6(0.001, 0.1, 0.0, 0.5, 2, 3)
    cpu = reference.solver(n, p, 0)
    cpu.initialize("multimode")
    e = hzlb.Ensemble(hzlb.Config(n=n, members=1, precision=8, nu=0.001, alpha=0.1))
    e.set_state(cpu.coefficients()[None])
    e.step(dt, steps)
    cpu.step(dt, steps)
    assert rel_l2(e.get_state()[0], cpu.coefficients()) <= FP64_TOL


def test_fourier_normalisation_and_physical(hzlb, oracle):
    """tests/verification.cpp:28-43 on the device observation operator: the physical field of
    the spectrum of sin(3x) + 0.7 cos(2y) is that field."""
    n = 32
    x = np.arange(n)
    field = (np.sin(3 * 2 * np.pi * x / n)[None, :] + 0.7 * np.cos(2 * 2 * np.pi * x / n)[:, None])
    spec = oracle.fft(field.astype(np.complex128), inverse=False)
    assert abs(spec[0, 3] - (0 - 0.5j)) < 1e-14
    e = hzlb.Ensemble(hzlb.Config(n=n, members=2, precision=8))
    e.set_state(np.array([spec, 2 * spec]))
    phys = e.physical()
    np.testing.assert_allclose(phys[0], field, atol=1e-14)
    np.testing.assert_allclose(phys[1], 2 * field, atol=1e-14)
    xs, ys = np.array([0, 5, 31]), np.array([0, 7, 30])
    np.testing.assert_allclose(e.observe(xs, ys), phys[:, ys, xs], rtol=0, atol=0)


def test_taylor_green_decay_order(hzlb, oracle):
    """tests/verification.cpp:44-65: Taylor-Green decays as exp(-2 (nu k^2 ... )) exactly;
    RK4 error ratios > 14 when dt halves."""
    n = 16
    nu, alpha = 0.7, 0.6
    s = oracle.solver(n, params6(nu, alpha, 0.0, 0.5, 2, 3), 1)
    s.initialize("taylor-green")
    w0 = s.state()[0]
    exact = w0 * np.exp(-2.0 * 0.4)
    errors = []
    for dt in (0.04, 0.02, 0.01):
        e = hzlb.Ensemble(hzlb.Config(n=n, members=1, precision=8, nu=nu, alpha=alpha))
        e.set_state(w0[None])
        e.step(dt, int(round(0.4 / dt)))
        errors.append(rel_l2(e.get_state()[0], exact))
        d = e.diagnostics()[0]
        assert abs(d[1] / (np.pi ** 2 * np.exp(-4.0 * 0.4)) - 1) < 1e-6
        assert abs(d[3] - 2 * nu * d[2]) < 1e-13
    assert errors[0] / errors[1] > 14 and errors[1] / errors[2] > 14


@pytest.mark.parametrize("precision,tol", [(8, 1e-9), (4, 2e-5)])
def test_inviscid_conservation(hzlb, oracle, precision, tol):
    """tests/verification.cpp:86-108: inviscid multimode flow at N=32 conserves energy and
    enstrophy (1e-9 in FP64)."""
    n = 32
    s = oracle.solver(n, params6(0.0, 0.0, 0.0, 0.5, 2, 3), 1)
    s.initialize("multimode")
    e = hzlb.Ensemble(hzlb.Config(n=n, members=1, precision=precision, nu=0.0, alpha=0.0))
    e.set_state(s.state()[0][None])
    before = e.diagnostics()[0]
    e.step(0.005, 100)
    after = e.diagnostics()[0]
    assert abs(after[1] / before[1] - 1) < tol
    assert abs(after[2] / before[2] - 1) < tol


def test_diagnostics_match_oracle(hzlb, oracle):
    n = 64
    w = oracle.grf(n, 5, 0)
    f = oracle.kolmogorov(n)
    s = oracle.solver(n, params6(1e-3, 0.0, 0.0, 0.5, 1, 4), 0)
    s.set_state(w, f)
    ref = s.diagnostics()
    e = hzlb.Ensemble(hzlb.Config(n=n, members=1, precision=8, nu=1e-3, forcing_kmax=0))
    e.set_state(w[None])
    e.set_forcing(f[None])
    got = e.diagnostics()[0]
    np.testing.assert_allclose(got[1:], ref[1:], rtol=1e-12)


def test_batch_composition_independence(hzlb):
    """A member's trajectory does not depend on which other members share the batch
    (the analogue of the reference's worker-count independence, verification.cpp:160-163)."""
    n, dt, seed = 64, 1e-3, 9
    big = device_synthetic(hzlb, n, 6, 4, 1e-3, 0.05, seed)
    big.step(dt, 5)
    cfg = hzlb.Config(n=n, members=2, precision=4, nu=1e-3, forcing_kmax=0, noise_sigma=0.05,
                      seed=seed, member_base=4)
    small = hzlb.Ensemble(cfg)
    small.set_state(np.array([hzlb.grf_spectrum(n, seed, m) for m in (4, 5)]))
    small.set_forcing(hzlb.kolmogorov_forcing(n)[None])
    small.set_time(0.0, 0)
    small.step(dt, 5)
    np.testing.assert_array_equal(small.get_state_compact(), big.get_state_compact(4, 2))


@pytest.mark.parametrize("precision,members", [(4, 2048), (8, 512)])
def test_batch_independence_at_benchmark_size(hzlb, precision, members):
    """At the benchmark's own size (256^2, 2048 FP32 members; 512 in FP64) the first, a middle
    and the last two members are bit-identical with the same members stepped alone in a
    two-member ensemble (member_base selects their noise streams): the whole-ensemble column
    groups, state windows and velocity rows address every member correctly."""
    n, dt, seed = 256, 2.5e-4, 42
    ctype = np.complex64 if precision == 4 else np.complex128
    w0 = hzlb.full_to_compact(hzlb.grf_spectrum(n, seed, 0), n)[0].astype(ctype)

    def run(count, base):
        cfg = hzlb.Config(n=n, members=count, precision=precision, nu=2.5e-4, alpha=0.0,
                          forcing_kmax=0, noise_sigma=0.05, noise_kmax=4, seed=seed,
                          member_base=base)
        e = hzlb.Ensemble(cfg)
        e.set_state_compact(np.repeat(w0[None], count, 0))
        e.set_forcing(hzlb.kolmogorov_forcing(n)[None])
        e.set_time(0.0, 0)
        e.step(dt, 3)
        return e

    big = run(members, 0)
    assert big.status() == 0
    for first in (0, members // 2 - 1, members - 2):
        small = run(2, first)
        np.testing.assert_array_equal(small.get_state_compact(), big.get_state_compact(first, 2))
        small.close()
    # the members differ (their noise does), so the comparison is not of copies of one field
    assert not np.array_equal(big.get_state_compact(0, 1), big.get_state_compact(members - 1, 1))
    big.close()


def test_cfl_violation_is_flagged(hzlb):
    n = 32
    e = hzlb.Ensemble(hzlb.Config(n=n, members=1, precision=8, nu=0.0))
    w = hzlb.grf_spectrum(n, 1, 0) * 200.0
    e.set_state(w[None])
    e.step(0.05, 1)
    assert e.status() & hzlb.STATUS_CFL


def test_invalid_arguments(hzlb):
    e = hzlb.Ensemble(hzlb.Config(n=32, members=2, precision=8, nu=1e-3, forcing_kmax=2))
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.step(-1.0, 1)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.step(float("nan"), 1)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.step(20.0, 1)   # diffusion limit: dt (2 nu K^2 + alpha) = 20 * 0.2 > 2.5 (K = 10)
    bad = np.zeros((1, 32, 32), np.complex128)
    bad[0, 1, 1] = np.nan
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.set_state(bad)
    asym = np.zeros((1, 32, 32), np.complex128)
    asym[0, 1, 0] = 1.0   # partner (0, -1) left at zero: not conjugate-symmetric
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.set_forcing(asym)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.get_state(1, 5)


def test_empty_step_and_single_member(hzlb, oracle):
    n = 16
    e = device_synthetic(hzlb, n, 1, 8, 1e-3, 0.0, 1)
    before = e.get_state()
    e.step(1e-3, 0)
    np.testing.assert_array_equal(e.get_state(), before)


def test_nonfinite_state_flagged(hzlb):
    n = 16
    e = hzlb.Ensemble(hzlb.Config(n=n, members=1, precision=4, nu=0.0))
    w = hzlb.grf_spectrum(n, 1, 0).astype(np.complex64)
    compact = hzlb.full_to_compact(w, n).astype(np.complex64)
    compact[0, 5] = np.inf
    e.set_state_compact(compact)
    e.step(1e-4, 1)
    assert e.status() & hzlb.STATUS_NONFINITE


@pytest.mark.parametrize("precision,n,members", [(4, 64, 300), (8, 32, 258), (4, 256, 256)])
def test_step_schedules_agree_bit_for_bit(hzlb, precision, n, members):
    """hzlb_set_step_schedule: the ensemble in two member parts on two streams (side by side, or
    the second part one row pass behind) steps exactly as the single pass does, through graph
    batches of 8 steps and single steps alike; the clock, step counter and status come back
    whole; a pending wait-timeout injection reaches the first part and is reported."""
    dt, seed = 1e-3 if n < 256 else 2.5e-4, 5
    runs = {}
    for schedule in ("single", "parts", "offset_parts"):
        e = device_synthetic(hzlb, n, members, precision, 1e-3, 0.05, seed)
        e.set_step_schedule(schedule)
        assert e.step_schedule() == schedule
        e.step(dt, 8 + 3)
        assert e.status() == 0
        runs[schedule] = (e.get_state_compact(), e.time())
        e.inject_wait_timeout()
        e.step(dt, 1)
        assert e.status() & hzlb.STATUS_TIMEOUT
        e.close()
    for schedule in ("parts", "offset_parts"):
        np.testing.assert_array_equal(runs[schedule][0], runs["single"][0])
        assert runs[schedule][1] == runs["single"][1]
    with pytest.raises(hzlb.HzlbError):
        e = device_synthetic(hzlb, 16, 4, 4, 1e-3, 0.05, seed)
        try:
            e.set_step_schedule(3)
        finally:
            e.close()
