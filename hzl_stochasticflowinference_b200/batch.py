"""Mixed-resolution ensemble batch (the uneven-batching configuration): 4096 members at 64^2,
1024 at 128^2, 128 at 256^2 and 8 at 512^2, FP32, nu = 1e-3 (64 / N), Kolmogorov forcing and
the additive noise, seeded random-field initial vorticity.  Each resolution's time step is set
by the reference's CFL rule dt max(|u| + |v|) N / 2 pi = 0.5 (src/solver.cpp:213, 393-395)
with the velocity bound max(|u| + |v|) <= U = 4, i.e. dt = pi / (4 N): the random initial
fields are nearly at rest (|u| ~ 0.03), so a step set from them would be broken within a few
steps once the forcing energises the flow.  The row kernel checks the rule on the actual
velocities at every step and the run reports those status bits (0: the rule held throughout).
All resolutions advance together in one CUDA graph per batch of steps (hzlb_mixed_*); the
schedule is either serial or the autotuner's choice.
"""
from __future__ import annotations

import time

import numpy as np

from . import Config, Mixed, full_to_compact, grf_spectrum, kolmogorov_forcing, retained_k

GROUPS = ((64, 4096), (128, 1024), (256, 128), (512, 8))
SEED = 42


def bytes_per_member_step(n: int, real_bytes: int = 4) -> float:
    """Algorithmic HBM bytes of one RK4 step of one member in this design: per stage the row
    pass reads the two velocity column fields and writes the two product fields, the column pass
    reads the products, writes the next velocities and reads/writes the state arrays (4.25 on
    average over the stages)."""
    k = retained_k(n)
    c, ld = k + 1, 2 * k + 1
    cb = 2 * real_bytes
    return 4 * (4 * c * n + 4 * c * n + 4 * c * n + 4.25 * c * ld) * cb


def build(groups=GROUPS, seed: int = SEED) -> tuple[Mixed, list]:
    configs, base = [], 0
    for n, members in groups:
        configs.append(Config(n=n, members=members, precision=4, nu=1e-3 * 64 / n, alpha=0.0,
                              forcing_kmax=0, noise_sigma=0.05, noise_kmax=4, seed=seed,
                              member_base=base))
        base += members
    m = Mixed(configs)
    for g, c in zip(m.groups, configs):
        chunk = 512
        for first in range(0, c.members, chunk):
            k = min(chunk, c.members - first)
            states = np.empty((k, g.compact_size), np.complex64)
            for i in range(k):
                states[i] = full_to_compact(grf_spectrum(c.n, seed, c.member_base + first + i), c.n)[0]
            g.set_state_compact(states, first)
            g.synchronize()
        g.set_forcing(kolmogorov_forcing(c.n)[None])
    return m, configs


VELOCITY_BOUND = 4.0


def cfl_dt(n: int, bound: float = VELOCITY_BOUND) -> float:
    """dt with dt * bound * n / 2 pi = 0.5."""
    return 0.5 * 2 * np.pi / (bound * n)


def run(steps: int = 500, tune_repeats: int = 2, groups=GROUPS, log=None) -> dict:
    total_members = sum(n_m[1] for n_m in groups)
    step_bytes = sum(m_ * bytes_per_member_step(n) for n, m_ in groups)
    dts = [cfl_dt(n) for n, _ in groups]
    results = {}
    for label in ("serial", "tuned"):
        m, configs = build(groups)
        if label == "serial":
            m.set_schedule(True)
        else:
            t0 = time.perf_counter()
            results["tuner_ms_per_step"] = m.tune(dts, tune_repeats)
            results["tune_seconds"] = time.perf_counter() - t0
            results["schedule"] = m.schedule()
        m.step(dts, 8)                       # graph capture and warm-up
        t0 = time.perf_counter()
        m.step(dts, steps)                   # one graph launch per 8 steps, waited for
        el = time.perf_counter() - t0
        ms = el * 1e3 / steps
        results[label] = {"ms_per_step": ms, "member_steps_per_s": total_members * steps / el,
                          "algorithmic_gbs": step_bytes / (ms * 1e-3) / 1e9,
                          "status": [int(g.status()) for g in m.groups],
                          "enstrophy_max": [float(np.max(g.diagnostics()[:, 2])) for g in m.groups]}
        if log:
            log(f"{label}: {ms:.3f} ms per step, status {results[label]['status']}")
        m.close()
    results.update(groups=[{"n": n, "members": m_, "nu": 1e-3 * 64 / n, "dt": dt}
                           for (n, m_), dt in zip(groups, dts)],
                   steps=steps, velocity_bound=VELOCITY_BOUND,
                   algorithmic_bytes_per_step=step_bytes)
    return results
