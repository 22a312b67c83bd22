"""Shared test helpers: run the same seeded workload on the oracle and on the device."""
from __future__ import annotations

import numpy as np

from oracle.oracle import params6


def rel_l2(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def synthetic_params(n: int, nu: float, alpha: float = 0.0):
    """Oracle Parameters for the seeded-synthetic physics: OU forcing off (sigma = 0); the
    forcing shell only has to be valid for the grid."""
    kmax = min(4, (n - 1) // 3)
    return params6(nu, alpha, 0.0, 0.5, 1, kmax)


def oracle_synthetic_run(oracle, n, members, steps, dt, nu, sigma, seed, alpha=0.0,
                         amplitude=0.1, wavenumber=4, noise_kmax=4, init=None):
    """Runs the oracle on the seeded-synthetic workload; returns final spectra (members, n, n)
    and per-step (energy, enstrophy) of member 0."""
    forcing = oracle.kolmogorov(n, amplitude, wavenumber)
    out = []
    series = []
    for m in range(members):
        s = oracle.solver(n, synthetic_params(n, nu, alpha), 0)
        w0 = oracle.grf(n, seed, m) if init is None else init[m]
        s.set_state(w0, np.zeros((n, n), np.complex128))
        for i in range(steps):
            s.synthetic_step(dt, forcing, sigma, noise_kmax, seed, m, i)
            if m == 0:
                d = s.diagnostics()
                series.append((d[1], d[2]))
        out.append(s.state()[0])
    return np.array(out), np.array(series)


def device_synthetic(hzlb, n, members, precision, nu, sigma, seed, alpha=0.0, amplitude=0.1,
                     wavenumber=4, noise_kmax=4, init=None):
    cfg = hzlb.Config(n=n, members=members, precision=precision, nu=nu, alpha=alpha,
                      forcing_kmax=0, forcing_per_member=False, noise_sigma=sigma,
                      noise_kmax=noise_kmax, seed=seed)
    e = hzlb.Ensemble(cfg)
    w0 = np.array([hzlb.grf_spectrum(n, seed, m) for m in range(members)]) if init is None else init
    e.set_state(w0)
    e.set_forcing(hzlb.kolmogorov_forcing(n, amplitude, wavenumber)[None])
    e.set_time(0.0, 0)
    return e
