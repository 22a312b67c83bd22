"""Generates the golden vectors in this directory from the reference's own CPU library
(oracle/_ref/libhzlref.so, compiled from the reference sources by oracle/Makefile).

Run from the repository root:  python tests/golden/make_golden.py
Every vector is produced by calling the reference through its public API (Fourier2D,
Solver, ShellForcing, bootstrap_filter, ensemble_kalman_filter, fit_pod); the seeded
synthetic workload (Kolmogorov forcing + Euler-Maruyama noise + Gaussian random initial
field) is driven through Solver::update_latent_state / Solver::step, with the noise and the
initial field from the oracle's Philox convention."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle.oracle import Oracle, Reference, params6  # noqa: E402


def fft_vectors(ref: Reference):
    rng = np.random.default_rng(2024)
    a = rng.standard_normal((16, 16)) + 1j * rng.standard_normal((16, 16))
    np.savez_compressed(HERE / "fft_n16.npz", input=a, forward=ref.fft(a, False),
                        inverse=ref.fft(a, True))


def reference_step(ref: Reference):
    """Solver(16, defaults, 123) multimode, 7 steps of 0.01 (verification.cpp:141-145)."""
    p = params6(0.01, 0.1, 0.2, 0.5, 2, 3)
    s = ref.solver(16, p, 123)
    s.initialize("multimode")
    w0 = s.coefficients()
    s.step(0.01, 7)
    np.savez_compressed(HERE / "step_ou_n16.npz", initial=w0, final=s.coefficients(),
                        forcing=s.forcing(), diagnostics=s.diagnostics(), params=p, seed=123,
                        steps=7, dt=0.01)


def config0(ref: Reference, o: Oracle):
    """N=64 seeded-synthetic workload, 1000 steps of dt=1e-3, nu=1e-3, Kolmogorov 0.1 sin(4y),
    EM noise sigma=0.05 on 1<=|k|<=4, GRF initial field (seed 42, member 0), driven through the
    reference's Solver: update_latent_state(w0, f) -> [step(dt); update_latent_state(w + xi, f)]."""
    n, steps, dt, nu, sigma, seed = 64, 1000, 1e-3, 1e-3, 0.05, 42
    p = params6(nu, 0.0, 0.0, 1e300, 4, 4)
    s = ref.solver(n, p, 0)
    forcing = o.kolmogorov(n, 0.1, 4)
    s.update_latent_state(o.grf(n, seed, 0), forcing)
    series = np.zeros((steps, 2))
    for i in range(steps):
        s.step(dt)
        w = o.add_noise(s.coefficients(), sigma, dt, 4, seed, 0, i)
        s.update_latent_state(w, s.forcing())
        d = s.diagnostics()
        series[i] = d[1], d[2]
    np.savez_compressed(HERE / "config0_n64.npz", final=s.coefficients(), series=series, n=n,
                        steps=steps, dt=dt, nu=nu, sigma=sigma, seed=seed)


def filters(ref: Reference):
    p = params6(0.03, 0.1, 0.2, 0.5, 2, 3)
    ds = ref.synthetic_observations(16, 0.01, 30, 10, p, 0.2, 987)
    pf = ref.bootstrap_filter(ds, p, 32, 555)
    kal = ref.enkf(ds, p, 12, 99, 1.02, 4.0, 2, 1)
    np.savez_compressed(HERE / "filters_n16.npz", steps=ds["steps"], x=ds["x"], y=ds["y"],
                        value=ds["value"], sd=ds["sd"], pf_loglik=pf["log_likelihood"],
                        pf_events=pf["resampling_events"], pf_records=pf["records"],
                        pf_means=pf["means"], enkf_records=kal["records"], enkf_means=kal["means"])


def pod(ref: Reference):
    p = params6(0.01, 0.1, 0.0, 0.5, 2, 3)
    s = ref.solver(16, p, 1)
    s.initialize("multimode")
    snaps = []
    for _ in range(20):
        snaps.append(s.coefficients())
        s.step(0.01)
    snaps = np.array(snaps)
    mean, modes, sv, cap = ref.fit_pod(snaps, 4, 0.9999999)
    np.savez_compressed(HERE / "pod_n16.npz", snapshots=snaps, mean=mean, modes=modes,
                        singular_values=sv, captured=cap)


if __name__ == "__main__":
    r, o = Reference(), Oracle()
    fft_vectors(r)
    reference_step(r)
    config0(r, o)
    filters(r)
    pod(r)
    print("golden vectors written to", HERE)
