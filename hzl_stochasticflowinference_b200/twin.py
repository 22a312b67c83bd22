"""Filtering twin experiment at 128^2: perturbed-observation EnKF and bootstrap particle filter
on the batched B200 path (FP32 forecast, FP64 analysis solve and particle weights).

A truth member is advanced with the Kolmogorov forcing and the additive noise and observed
every `obs_every` steps at the points of a regular sub-grid (stride `obs_stride`), with
Gaussian errors of standard deviation `obs_sd`.  Both filters start from independent draws of
the seeded Gaussian random field (unit enstrophy, E(k) ~ k^4 exp(-(k/6)^2)), one per member,
and advance every member with its own noise:

* EnKF: multiplicative anomaly inflation, then the batched perturbed-observation analysis of
  all observations at once (hzlb_enkf_analysis_nis with device perturbations);
* PF: Gaussian log-likelihood of every particle, FP64 weights in the reference's order
  (log-sum-exp increment, ESS), systematic resampling with a seeded uniform when the ESS falls
  below resample_fraction x particles (the reference's rule, filter.cpp:102-112), members
  copied on the device.

Analysis RMSE is the grid RMSE of the (weighted) ensemble mean against the truth.
"""
from __future__ import annotations

import time
from dataclasses import asdict, dataclass

import numpy as np

from . import (Config, Ensemble, full_to_compact, grf_spectrum, kolmogorov_forcing,
               retained_k)

TRUTH_ID = 1_000_000
PF_BASE = 2_000_000


@dataclass
class FilterTwinConfig:
    n: int = 128
    nu: float = 5e-4
    dt: float = 5e-4
    forcing_amplitude: float = 0.1
    forcing_wavenumber: int = 4
    noise_sigma: float = 0.05
    noise_kmax: int = 4
    seed: int = 42
    obs_every: int = 50
    obs_stride: int = 8              # 16 x 16 points at 128^2
    obs_sd: float = 0.1
    cycles: int = 40
    enkf_members: int = 512
    inflation: float = 1.05
    particles: int = 2048
    resample_fraction: float = 0.5

    def config(self, members: int, member_base: int) -> Config:
        return Config(n=self.n, members=members, precision=4, nu=self.nu, alpha=0.0,
                      forcing_kmax=0, noise_sigma=self.noise_sigma, noise_kmax=self.noise_kmax,
                      seed=self.seed, member_base=member_base)


def _weights(n: int) -> np.ndarray:
    k = retained_k(n)
    return np.repeat(np.where(np.arange(k + 1) > 0, 2.0, 1.0), 2 * k + 1)


def field_rmse(a, b, n: int) -> float:
    d = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
    return float(np.sqrt(np.sum(_weights(n) * np.abs(d) ** 2)))


def observation_grid(tc: FilterTwinConfig):
    g = np.arange(0, tc.n, tc.obs_stride)
    return np.tile(g, len(g)).astype(np.uint32), np.repeat(g, len(g)).astype(np.uint32)


def _ensemble(tc: FilterTwinConfig, count: int, member_base: int) -> Ensemble:
    """count members, member i from the random field of member id member_base + i."""
    e = Ensemble(tc.config(count, member_base))
    e.set_forcing(kolmogorov_forcing(tc.n, tc.forcing_amplitude, tc.forcing_wavenumber))
    chunk = 256
    for first in range(0, count, chunk):
        c = min(chunk, count - first)
        states = np.empty((c, e.compact_size), np.complex64)
        for i in range(c):
            states[i] = full_to_compact(grf_spectrum(tc.n, tc.seed, member_base + first + i), tc.n)[0]
        e.set_state_compact(states, first)
        e.synchronize()
    return e


def truth_run(tc: FilterTwinConfig):
    e = _ensemble(tc, 1, TRUTH_ID)
    xs, ys = observation_grid(tc)
    rng = np.random.default_rng(tc.seed + 3)
    states, obs = [e.get_state_compact()[0].astype(np.complex128)], []
    for _ in range(tc.cycles):
        e.step(tc.dt, tc.obs_every)
        states.append(e.get_state_compact()[0].astype(np.complex128))
        obs.append(e.observe(xs, ys)[0] + tc.obs_sd * rng.normal(size=len(xs)))
    e.close()
    return states, obs


def run_enkf(tc: FilterTwinConfig, truth, log=None) -> dict:
    import torch
    states, obs = truth
    e = _ensemble(tc, tc.enkf_members, 0)
    xs, ys = observation_grid(tc)
    sd = np.full(len(xs), tc.obs_sd)
    prior = field_rmse(e.mean_compact(), states[0], tc.n)
    rmse, nis, seconds = [], [], []
    for c in range(tc.cycles):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.step(tc.dt, tc.obs_every)
        if tc.inflation > 1:
            e.inflate(tc.inflation)
        v, _ = e.enkf_analysis_nis(xs, ys, obs[c], sd, None, seed=tc.seed + 5, cycle=c)
        e.synchronize()
        seconds.append(time.perf_counter() - t0)
        rmse.append(field_rmse(e.mean_compact(), states[c + 1], tc.n))
        nis.append(v)
        if log:
            log(f"enkf cycle {c}: rmse {rmse[-1]:.4f} nis {v:.3f} {1e3 * seconds[-1]:.1f} ms")
    e.close()
    steady = seconds[1:] if len(seconds) > 1 else seconds
    return dict(rmse=rmse, nis=nis, seconds=seconds, initial_rmse=prior,
                mean_rmse=float(np.mean(rmse)), final_rmse=rmse[-1],
                seconds_per_cycle=float(np.median(steady)))


def run_pf(tc: FilterTwinConfig, truth, log=None) -> dict:
    import torch
    states, obs = truth
    M = tc.particles
    e = _ensemble(tc, M, PF_BASE)
    xs, ys = observation_grid(tc)
    sd = np.full(len(xs), tc.obs_sd)
    if tc.resample_fraction != 0.5:
        raise ValueError("the device filter resamples when ESS < particles / 2 (filter.cpp:102)")
    rng = np.random.default_rng(tc.seed + 9)
    e.pf_reset(M)
    pending = None   # the next resampling uniform, drawn ahead and kept until used
    prior = field_rmse(e.mean_compact(), states[0], tc.n)
    rmse, ess_hist, loglik, resampled, seconds = [], [], [], [], []
    for c in range(tc.cycles):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.step(tc.dt, tc.obs_every)
        if pending is None:
            pending = float(rng.random())
        r = e.pf_assimilate(xs, ys, obs[c], sd, u=[pending], weighted_mean=True)
        did, ess, inc, mean = bool(r["resampled"][0]), r["ess"][0], r["increment"][0], r["mean"][0]
        if did:
            pending = None
        e.synchronize()
        seconds.append(time.perf_counter() - t0)
        rmse.append(field_rmse(mean, states[c + 1], tc.n))
        ess_hist.append(float(ess))
        loglik.append(float(inc))
        resampled.append(bool(did))
        if log:
            log(f"pf cycle {c}: rmse {rmse[-1]:.4f} ess {ess:.1f}{' resampled' if did else ''} "
                f"{1e3 * seconds[-1]:.1f} ms")
    e.close()
    steady = seconds[1:] if len(seconds) > 1 else seconds
    return dict(rmse=rmse, ess=ess_hist, loglik_increments=loglik, resampled=resampled,
                seconds=seconds, initial_rmse=prior, mean_rmse=float(np.mean(rmse)),
                final_rmse=rmse[-1], resampling_events=int(np.sum(resampled)),
                seconds_per_cycle=float(np.median(steady)))


def run(tc: FilterTwinConfig, log=None) -> dict:
    truth = truth_run(tc)
    return dict(config=asdict(tc), enkf=run_enkf(tc, truth, log), pf=run_pf(tc, truth, log))
