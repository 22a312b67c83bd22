"""Learned reduced forecast and the EnKF twin experiment that judges it.

The reference has no learned model; this module builds one on the B200 path and measures it
against the full spectral forecast:

1. spin-up: one member from a seeded Gaussian random field, advanced with the Kolmogorov
   forcing and the additive noise;
2. snapshots of an ensemble started from that state plus Gaussian perturbations on the modes
   of the noise shell 1 <= |k| <= noise_kmax (the scales the stochastic forcing acts on), and
   a POD basis of them (``Pod``: tensor-core Gram, subspace iteration);
3. transitions of a larger ensemble over forecast windows: POD coefficients at the start,
   the window's noise-mode amplitudes, and the POD coefficients at the end less the
   projection of the window's own noise increments (which the learned window adds exactly,
   so the network learns the drift), all produced on the GPU;
4. the BF16 MLP (``Mlp``) trained on them with Adam on the tensor cores;
5. a twin experiment: a truth run observed on a regular sub-grid, and a perturbed-observation
   EnKF whose forecast is either the spectral solver, the learned window (with fallback to the
   spectral solver for every cycle whose normalised innovation statistic exceeds the limit),
   the hybrid of the learned window for the members' motion about their mean and the spectral
   solver for the mean itself (one extra member), the complement variant (the network advances
   every member's POD coefficients, the mean's included, and the one-member spectral step of
   the mean supplies only the motion outside the POD space, which the network cannot carry),
   or persistence through the same pipelines with the network's output switched off (what the
   method gives without the network).

Torch is used only to hold device buffers; every computation goes through libhzlb.
"""
from __future__ import annotations

import math
import time
from dataclasses import asdict, dataclass, replace

import numpy as np

from . import (Config, Ensemble, Mlp, Pod, add_window_noise, grf_spectrum, kolmogorov_forcing,
               noise_amplitudes, retained_k)

# Philox member keys of the experiment's ensembles (disjoint, so no two runs share noise)
TRUTH_ID = 1_000_000
SNAPSHOT_BASE = 2_000_000
TRAIN_BASE = 3_000_000
SPINUP_ID = 4_000_000
MEAN_ID = 5_000_000


@dataclass
class TwinConfig:
    n: int = 256
    nu: float = 2.5e-4
    dt: float = 5e-4
    window: int = 20                 # solver steps per forecast window / analysis cycle
    forcing_amplitude: float = 0.1   # f = amplitude sin(wavenumber y)
    forcing_wavenumber: int = 4
    noise_sigma: float = 0.05
    noise_kmax: int = 4
    seed: int = 42
    spinup_steps: int = 2000
    perturbation: float = 0.15       # rms vorticity of the members' initial perturbations
    snapshots: int = 2000
    snapshot_members: int = 40
    rank: int = 64
    hidden: int = 1024
    train_members: int = 2048
    train_windows: int = 98          # 2048 x 98 = 200,704 transitions
    epochs: int = 400
    batch: int = 1024
    lr: float = 1e-3                 # Adam, cosine-decayed to lr_floor * lr over the run
    lr_floor: float = 0.02
    members: int = 1024
    obs_stride: int = 8              # observations every obs_stride grid points (32 x 32 at 256)
    obs_sd: float = 0.1
    cycles: int = 40
    inflation: float = 1.0
    nis_limit: float = 3.0

    def config(self, members: int, member_base: int) -> Config:
        return Config(n=self.n, members=members, precision=4, nu=self.nu, alpha=0.0,
                      forcing_kmax=0, noise_sigma=self.noise_sigma, noise_kmax=self.noise_kmax,
                      seed=self.seed, member_base=member_base)


def _weights(n: int) -> np.ndarray:
    """Parseval weights of the compact complex entries: 1 on kx = 0, 2 on kx > 0."""
    k = retained_k(n)
    return np.repeat(np.where(np.arange(k + 1) > 0, 2.0, 1.0), 2 * k + 1)


def field_rmse(a: np.ndarray, b: np.ndarray, n: int) -> float:
    """Grid RMSE of two real fields given by compact spectra: sqrt(mean_x (a - b)^2)."""
    d = np.asarray(a, np.complex128) - np.asarray(b, np.complex128)
    return float(np.sqrt(np.sum(_weights(n) * np.abs(d) ** 2)))


def perturbation(tc: TwinConfig, member: int) -> np.ndarray:
    """Initial perturbation of one member (compact layout): independent complex Gaussian
    coefficients on the noise shell 1 <= |k|^2 <= noise_kmax^2, conjugate-symmetric on the
    kx = 0 column, scaled to an rms vorticity of tc.perturbation."""
    k = retained_k(tc.n)
    ld = 2 * k + 1
    rng = np.random.default_rng([tc.seed, member])
    out = np.zeros((k + 1, ld), np.complex128)
    km = tc.noise_kmax
    weight = 0.0
    for kx in range(0, km + 1):
        for ky in range(-km, km + 1):
            k2 = kx * kx + ky * ky
            if k2 < 1 or k2 > km * km or (kx == 0 and ky < 0):
                continue
            z = complex(rng.normal(), rng.normal()) / np.sqrt(2.0)
            out[kx, ky % ld] = z
            weight += 2.0
            if kx == 0:
                out[0, (-ky) % ld] = np.conj(z)
    return (out * (tc.perturbation / np.sqrt(weight))).ravel()


def _ensemble(tc: TwinConfig, base: np.ndarray, ids_base: int, count: int) -> Ensemble:
    """count members: base + perturbation(member id), Kolmogorov forcing and noise on."""
    e = Ensemble(tc.config(count, ids_base))
    e.set_forcing(kolmogorov_forcing(tc.n, tc.forcing_amplitude, tc.forcing_wavenumber))
    chunk = 256
    for first in range(0, count, chunk):
        c = min(chunk, count - first)
        states = np.empty((c, e.compact_size), np.complex64)
        for i in range(c):
            states[i] = base + perturbation(tc, ids_base + first + i)
        e.set_state_compact(states, first)
        e.synchronize()
    return e


def spinup(tc: TwinConfig) -> np.ndarray:
    """Compact complex state after the spin-up run."""
    e = Ensemble(tc.config(1, SPINUP_ID))
    e.set_forcing(kolmogorov_forcing(tc.n, tc.forcing_amplitude, tc.forcing_wavenumber))
    e.set_state(grf_spectrum(tc.n, tc.seed, 0)[None])
    e.step(tc.dt, tc.spinup_steps)
    e.synchronize()
    state = e.get_state_compact()[0].astype(np.complex128)
    e.close()
    return state


def snapshots(tc: TwinConfig, base: np.ndarray):
    """tc.snapshots compact FP32 states (CUDA tensor [count][2 * compact]) taken every window
    from an ensemble of tc.snapshot_members members."""
    import torch
    e = _ensemble(tc, base, SNAPSHOT_BASE, tc.snapshot_members)
    width = 2 * e.compact_size
    out = torch.empty((tc.snapshots, width), dtype=torch.float32, device="cuda")
    taken = 0
    while taken < tc.snapshots:
        e.step(tc.dt, tc.window)
        c = min(tc.snapshot_members, tc.snapshots - taken)
        e.get_state_compact_ptr(out[taken:].data_ptr(), 0, c)
        taken += c
    e.synchronize()
    e.close()
    return out


def transitions(tc: TwinConfig, base: np.ndarray, pod: Pod):
    """(X, Y): X = (coefficients, noise amplitudes) at the start of each window, Y = the
    coefficients at its end less rho = project(x + window noise) - project(x), the direct
    contribution of the window's noise; tc.train_members x tc.train_windows rows (CUDA)."""
    import torch
    r, M, W = tc.rank, tc.train_members, tc.train_windows
    e = _ensemble(tc, base, TRAIN_BASE, M)
    X = torch.empty((M * W, r + 8), dtype=torch.float32, device="cuda")
    Y = torch.empty((M * W, r), dtype=torch.float32, device="cuda")
    a = torch.empty((M, r), dtype=torch.float32, device="cuda")
    rho = torch.empty((M, r), dtype=torch.float32, device="cuda")
    scratch = torch.empty((M, 2 * e.compact_size), dtype=torch.float32, device="cuda")
    e.synchronize()
    pod.project_ptr(e.state_device(), M, a)
    for w in range(W):
        rows = slice(w * M, (w + 1) * M)
        X[rows, :r] = a
        step0 = e.time()[1]
        noise_amplitudes(e.config, tc.dt, step0, tc.window, M, X[rows, r:])
        e.get_state_compact_ptr(scratch.data_ptr(), 0, M)
        add_window_noise(e.config, tc.dt, step0, tc.window, M, scratch.data_ptr())
        pod.project_ptr(scratch.data_ptr(), M, rho)
        rho -= a
        e.step(tc.dt, tc.window)
        e.synchronize()   # the projection runs on the basis' stream
        pod.project_ptr(e.state_device(), M, a)
        Y[rows] = a - rho
    torch.cuda.synchronize()
    e.close()
    return X, Y


def train(tc: TwinConfig, X, Y, seed: int = 0, log=None) -> tuple[Mlp, dict]:
    """Adam on the mean squared coefficient error; 10% of the windows held out."""
    import torch
    r = tc.rank
    g = torch.Generator(device="cuda").manual_seed(seed)
    perm = torch.randperm(X.shape[0], device="cuda", generator=g)
    nval = X.shape[0] // 10
    val, tr = perm[:nval], perm[nval:]
    s_in = (X[tr].std(dim=0) + 1e-12).cpu().numpy()
    s_out = ((Y[tr] - X[tr, :r]).std(dim=0) + 1e-12).cpu().numpy()
    net = Mlp(r, 8, tc.hidden, max(tc.batch, tc.members), seed=seed)
    net.set_scales(s_in, s_out)
    B = tc.batch
    history = []
    t0 = time.perf_counter()
    steps = 0
    per_epoch = tr.numel() // B
    total_steps = max(1, per_epoch * tc.epochs)
    for epoch in range(tc.epochs):
        order = tr[torch.randperm(tr.numel(), device="cuda", generator=g)]
        total, count = 0.0, 0
        for i in range(0, order.numel() - B + 1, B):
            idx = order[i:i + B]
            frac = steps / total_steps
            lr = tc.lr * (tc.lr_floor + (1 - tc.lr_floor) * 0.5 * (1 + math.cos(math.pi * frac)))
            loss = net.train_step(X[idx].contiguous(), Y[idx].contiguous(), lr)
            total += loss
            count += 1
            steps += 1
        history.append(total / max(count, 1))
        if log:
            log(f"epoch {epoch}: train mse {history[-1]:.4e}")
    train_s = time.perf_counter() - t0
    metrics = evaluate(tc, net, X[val], Y[val])
    metrics.update(train_seconds=train_s, train_steps=steps, train_loss=history)
    return net, metrics


def evaluate(tc: TwinConfig, net: Mlp, X, Y) -> dict:
    """One-window coefficient error of the network and of persistence on held-out data."""
    import torch
    r, B = tc.rank, tc.batch
    err_net = err_pers = 0.0
    for i in range(0, X.shape[0], B):
        xb = X[i:i + B].contiguous()
        if xb.shape[0] < 1:
            continue
        yb = Y[i:i + B]
        pred = net.forward(xb)
        err_net += float(((pred - yb) ** 2).sum())
        err_pers += float(((xb[:, :r] - yb) ** 2).sum())
    change = float(((Y - X[:, :r]) ** 2).sum())
    return dict(val_mse_network=err_net / Y.numel(), val_mse_persistence=err_pers / Y.numel(),
                val_change_mse=change / Y.numel(),
                val_skill=1.0 - err_net / max(err_pers, 1e-300))


def zero_network(tc: TwinConfig, net: Mlp) -> Mlp:
    """A copy of `net` whose output is switched off (W3 = 0, b3 = 0): the pipeline then keeps
    the coefficients and adds only the window's noise (a random walk from the analysis)."""
    z = Mlp(tc.rank, 8, tc.hidden, max(tc.batch, tc.members), seed=1)
    parts = net.unpack(net.params())
    parts["W3"][:] = 0
    parts["b3"][:] = 0
    z.set_params(net.pack(parts))
    return z


def observation_grid(tc: TwinConfig):
    g = np.arange(0, tc.n, tc.obs_stride)
    return np.tile(g, len(g)).astype(np.uint32), np.repeat(g, len(g)).astype(np.uint32)


def truth_run(tc: TwinConfig, base: np.ndarray):
    """Truth compact states and noisy observations at the end of every cycle."""
    e = _ensemble(tc, base, TRUTH_ID, 1)
    xs, ys = observation_grid(tc)
    rng = np.random.default_rng(tc.seed + 7)
    states, obs = [], []
    for c in range(tc.cycles):
        e.step(tc.dt, tc.window)
        states.append(e.get_state_compact()[0].astype(np.complex128))
        obs.append(e.observe(xs, ys)[0] + tc.obs_sd * rng.normal(size=len(xs)))
    e.close()
    return states, obs


class ErrorSplit:
    """Splits an analysis error into its POD-subspace and complement parts (Parseval norm)."""

    def __init__(self, tc: TwinConfig, pod: Pod | None):
        self.w = np.repeat(_weights(tc.n), 2)   # per real entry
        self.modes = None
        if pod is not None:
            self.modes = pod.modes()[0].astype(np.float64)

    def __call__(self, mean: np.ndarray, truth: np.ndarray) -> tuple[float, float]:
        d = (np.asarray(mean, np.complex128) - np.asarray(truth, np.complex128)).view(np.float64)
        total = float(np.sum(self.w * d * d))
        if self.modes is None:
            return float(np.sqrt(total)), 0.0
        c = self.modes @ (self.w * d)
        inside = float(np.sum(c * c))
        return float(np.sqrt(min(inside, total))), float(np.sqrt(max(total - inside, 0.0)))


def twin(tc: TwinConfig, base: np.ndarray, truth, mode: str, pod: Pod | None = None,
         net: Mlp | None = None, log=None) -> dict:
    """EnKF twin experiment.  mode: "spectral" (full solver forecast), "learned" (learned
    window, spectral fallback when the innovation statistic exceeds tc.nis_limit), "hybrid"
    (as learned, with the ensemble mean advanced by the spectral solver on one member),
    "complement" (as learned, adding only the part of that spectral mean increment outside the
    POD space: the POD coefficients, the mean's included, move by the network alone),
    "persistence" / "hybrid_persistence" / "complement_persistence" (those pipelines with the
    network output off).
    Wall-clock per cycle covers forecast, analysis, fallback and inflation, with the GPU
    synchronised."""
    import torch
    states, obs = truth
    e = _ensemble(tc, base, 0, tc.members)
    xs, ys = observation_grid(tc)
    sd = np.full(len(xs), tc.obs_sd)
    split = ErrorSplit(tc, pod)
    if mode not in ("spectral", "learned", "hybrid", "complement", "persistence",
                    "hybrid_persistence", "complement_persistence"):
        raise ValueError(f"unknown forecast mode {mode}")
    if mode.endswith("persistence"):
        net = zero_network(tc, net)
    saved = None
    if mode != "spectral":
        saved = torch.empty((tc.members, 2 * e.compact_size), dtype=torch.float32, device="cuda")
    em = None
    complement = mode.startswith("complement")
    if complement:
        modes_t = torch.from_numpy(pod.modes()[0]).to("cuda")   # unweighted modes [r][2 compact]
        ca = torch.empty((1, tc.rank), dtype=torch.float32, device="cuda")
        cb = torch.empty_like(ca)
    if mode.startswith("hybrid") or complement:
        em = Ensemble(replace(tc.config(1, MEAN_ID), noise_sigma=0.0))
        em.set_forcing(kolmogorov_forcing(tc.n, tc.forcing_amplitude, tc.forcing_wavenumber))
        mbuf = torch.empty(2 * e.compact_size, dtype=torch.float32, device="cuda")
        fbuf = torch.empty_like(mbuf)
    rmse, rmse_pod, rmse_rest, spread_nis, fallback, seconds = [], [], [], [], [], []
    prior = [field_rmse(e.mean_compact(), states[0], tc.n)]
    for c in range(tc.cycles):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        used_fallback = False
        if mode == "spectral":
            e.step(tc.dt, tc.window)
            nis, _ = e.enkf_analysis_nis(xs, ys, obs[c], sd, None, seed=tc.seed + 11, cycle=c)
        else:
            clock = e.time()
            e.get_state_compact_ptr(saved.data_ptr(), 0, tc.members)
            inc = None
            if em is not None:
                e.mean_device(mbuf)
                em.set_state_compact_ptr(mbuf.data_ptr(), 0, 1)
                em.step(tc.dt, tc.window)
                em.get_state_compact_ptr(fbuf.data_ptr(), 0, 1)
                inc = fbuf - mbuf
                if complement:
                    # the POD part of the increment: the change of the (affine) projection
                    pod.project_ptr(mbuf.data_ptr(), 1, ca)
                    pod.project_ptr(fbuf.data_ptr(), 1, cb)
                    torch.cuda.synchronize()
                    inc = inc - ((cb - ca) @ modes_t)[0]
            e.learned_forecast(pod, net, tc.dt, tc.window, inc, centre=not complement)
            nis, applied = e.enkf_analysis_nis(xs, ys, obs[c], sd, None, seed=tc.seed + 11,
                                               cycle=c, nis_limit=tc.nis_limit)
            if not applied:
                used_fallback = True
                e.set_state_compact_ptr(saved.data_ptr(), 0, tc.members)
                e.set_time(*clock)
                e.step(tc.dt, tc.window)
                nis, _ = e.enkf_analysis_nis(xs, ys, obs[c], sd, None, seed=tc.seed + 11, cycle=c)
        if tc.inflation > 1:
            e.inflate(tc.inflation)
        e.synchronize()
        seconds.append(time.perf_counter() - t0)
        mean = e.mean_compact()
        rmse.append(field_rmse(mean, states[c], tc.n))
        inside, rest = split(mean, states[c])
        rmse_pod.append(inside)
        rmse_rest.append(rest)
        spread_nis.append(nis)
        fallback.append(used_fallback)
        if log:
            log(f"{mode} cycle {c}: rmse {rmse[-1]:.4f} nis {nis:.3f}"
                f"{' fallback' if used_fallback else ''} {1e3 * seconds[-1]:.2f} ms")
    e.close()
    if em is not None:
        em.close()
    # the first cycle pays one-time set-up (graph capture, workspace allocation)
    steady = seconds[1:] if len(seconds) > 1 else seconds
    return dict(mode=mode, rmse=rmse, rmse_pod=rmse_pod, rmse_complement=rmse_rest,
                nis=spread_nis, fallback=fallback, seconds=seconds,
                mean_rmse=float(np.mean(rmse)), final_rmse=rmse[-1],
                fallback_cycles=int(np.sum(fallback)), seconds_per_cycle=float(np.median(steady)),
                initial_rmse=prior[0])


def run(tc: TwinConfig, log=None) -> dict:
    """The whole experiment; returns every number it measured."""
    import torch
    out: dict = dict(config=asdict(tc))
    t = time.perf_counter()
    base = spinup(tc)
    out["spinup_seconds"] = time.perf_counter() - t
    t = time.perf_counter()
    snaps = snapshots(tc, base)
    torch.cuda.synchronize()
    out["snapshot_seconds"] = time.perf_counter() - t
    t = time.perf_counter()
    pod = Pod(tc.n, snaps, tc.rank, oversample=32, iterations=60, seed=tc.seed)
    out["pod_seconds"] = time.perf_counter() - t
    info = pod.info()
    out["pod"] = dict(captured=info["captured"], residual=info["residual"],
                      eigenvalues=info["eigenvalues"].tolist())
    del snaps
    t = time.perf_counter()
    X, Y = transitions(tc, base, pod)
    out["data_seconds"] = time.perf_counter() - t
    out["transitions"] = int(X.shape[0])
    net, metrics = train(tc, X, Y, seed=tc.seed, log=log)
    out["training"] = metrics
    del X, Y
    truth = truth_run(tc, base)
    modes = ("learned", "hybrid", "complement", "persistence", "hybrid_persistence",
             "complement_persistence")
    for mode in ("spectral",) + modes:
        out[mode] = twin(tc, base, truth, mode, pod, net, log=log)
    s = out["spectral"]
    for mode in modes:
        out[mode]["speedup"] = s["seconds_per_cycle"] / out[mode]["seconds_per_cycle"]
        out[mode]["rmse_ratio"] = out[mode]["mean_rmse"] / s["mean_rmse"]
    # headline: the variant whose POD coefficients move by the network alone
    out["speedup"] = out["complement"]["speedup"]
    out["rmse_ratio"] = out["complement"]["rmse_ratio"]
    return out
