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


def enkf_weight_matrix(hx: np.ndarray, y: np.ndarray, sd: np.ndarray, eps: np.ndarray) -> np.ndarray:
    """W = HA^T (HA HA^T/(M-1) + R)^-1 (y + sd eps - HX) / (M-1), the perturbed-observation
    EnKF in ensemble space (rows: contributing member, columns: updated member), in numpy FP64:
    the formula the batched device analysis is checked against."""
    m = hx.shape[0]
    ha = hx - hx.mean(axis=0)
    p = ha.T @ ha / (m - 1) + np.diag(sd * sd)
    d = (y[None, :] + sd[None, :] * eps - hx).T
    l = np.linalg.cholesky(p)
    z = np.linalg.solve(l.T, np.linalg.solve(l, d))
    return ha @ z / (m - 1)


class HostAnalysis:
    """The analysis arithmetic of the sharded filters on the host, for CPU ranks over gloo:
    the oracle's particle weights and resampling (the reference's order) and the numpy EnKF
    formula.  Stands in for sharding.DeviceAnalysis where no GPU is present."""

    def __init__(self):
        from oracle.oracle import Oracle
        self.oracle = Oracle()

    def pf_weights(self, logs):
        return self.oracle.pf_weights(np.asarray(logs, np.float64))

    def resample(self, weights, u):
        return self.oracle.systematic_resample(np.asarray(weights, np.float64), u)

    def enkf_weights(self, hx, y, sd, eps):
        import torch
        w = enkf_weight_matrix(hx.cpu().numpy(), np.asarray(y), np.asarray(sd), eps.cpu().numpy())
        return torch.from_numpy(w).to(hx.device)

    def anomaly_products(self, anomalies, w_rows):
        return (w_rows.T @ anomalies).contiguous()
