"""Benchmark of the B200 ensemble forecast step: member-steps/s at 256^2, FP32.

Workload (one "step" = one RK4 time step of every member): 2048 members per GPU at N=256,
complex64 compact spectra, nu=2.5e-4, dt=2.5e-4, Kolmogorov forcing 0.1 sin(4y) and
Euler-Maruyama noise sigma=0.05 on 1<=|k|<=4 (Philox, in-kernel), seeded Gaussian-random-field
initial vorticity (unit enstrophy).  The ensemble state plus stage buffers (~2.5 GB) is far
larger than L2 (126 MB), so every step streams from HBM.

Legs:
  value        device-resident throughput (CUDA events on the library's stream, max over ranks)
  e2e          the same step through the C ABI (hzlb_step_host) with the whole ensemble
               state read from pinned host memory and written back every step, the
               copies of each member chunk overlapping the stepping of the others
  roofline     dominant kernel: algorithmic bytes per launch / mean launch duration
  cpu_baseline the reference's own CPU solver (oracle/_ref, its Solver API driven with this
               workload's forcing, noise and fields on all host threads, FP64) on a bounded
               sample of the same workload
  fp64         the same workload, members and steps in FP64 (the reference's precision), with
               its own roofline and e2e: the like-for-like comparison with the reference arm
  gpu_reference the reference's own GPU path (src/cuda_solver.cu: cuFFT Z2Z, FP64, one solver
               instance per member launched in sequence, host OU forcing), built for sm_100a by
               oracle/Makefile, through its hzl-cuda-ensemble-benchmark driver at 256^2
  config1      (1 GPU) 256 members at 128^2, nu = dt = 5e-4, 2000 steps in FP32 and FP64 from
               identical inputs: per-member relative L2 and enstrophy drift of FP32 against FP64

  filters      (1 GPU) the 128^2 filtering twin experiment: EnKF 512 members (inflation 1.05) and
               bootstrap PF 2048 particles, 16x16 observations (sigma 0.1) every 50 steps, 40
               cycles; analysis RMSE and wall-clock per cycle, beside the reference CPU filters'
               forecast cost extrapolated from a measured single-thread member-step
  mixed        (1 GPU) the uneven batch: 4096 x 64^2, 1024 x 128^2, 128 x 256^2, 8 x 512^2 FP32
               members in one CUDA graph per batch of steps, 500 steps, serial schedule and the
               autotuner's schedule
  learned      (1 GPU) the learned-forecast EnKF twin experiment at 256^2: POD from 2000
               snapshots (r=64), the 72-1024-1024-64 BF16 MLP trained on 200,704 solver
               transitions of 20 steps, 1024-member EnKF observed on 32x32 points (sigma
               0.1) every 20 steps for 40 cycles; analysis RMSE and wall-clock per cycle of
               the spectral, learned, hybrid and complement forecasts and of each pipeline
               with the network's output off (--no-learned skips it); `headline` is the
               complement variant, where the network moves every POD coefficient

`--impl reference` times only the reference CPU solver on this workload (rank 0; other ranks
exit 0).
`--case gemm|enkf|learned` times one isolated workload (1 GPU) and prints its own JSON line:
the tcgen05 GEMM at 4096^3 (TF32 and BF16), one EnKF analysis at 1024 members x 1024
observations at 256^2, one learned forecast window at 1024 members x 256^2.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N = 256
MEMBERS = 2048
NU = 2.5e-4
DT = 2.5e-4
SIGMA = 0.05
SEED = 42
METRIC = "ensemble member-steps/s at 256^2"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per member per launch, from one
# single-pass ncu capture of this benchmark's own 2048-member launches at 256^2 FP32 (the
# column figure is the mean of its four RK-stage launches, like its algorithmic bytes),
# scaled by the members processed for other ensemble sizes.
NCU_TRAFFIC_PER_MEMBER = {"row_kernel": 690983.0, "column_kernel": 1186247.0}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: let its first sample arrive (at most 3 s)
            # so that the samples cover the timed region that follows
            deadline = time.time() + 3.0
            while not self.lines and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference_sample(n: int, seconds_target: float = 15.0):
    """Times the reference's own CPU solver on this benchmark's workload: the seeded-synthetic
    physics (Kolmogorov forcing, Euler-Maruyama noise, random initial fields) driven through
    the reference's Solver API -- update_latent_state, then Solver::step with its validate_step
    -- one member per std::jthread worker on all host threads (ref_synthetic_ensemble, as
    hzl::ensemble shares members out, src/inference.cpp:555-590); FP64, its only precision.
    A bounded sample: every thread's member for as many steps as fill ~seconds_target."""
    from oracle.oracle import Reference, host_cores
    ref = Reference()
    threads = host_cores()
    # calibrate with one member-step per thread, then size the sample to ~seconds_target
    t0 = time.perf_counter()
    ref.synthetic_ensemble(n, NU, DT, 1, threads, threads, SEED, SIGMA, 4, keep=False)
    one = time.perf_counter() - t0
    steps = max(2, int(seconds_target / max(one, 1e-3)))
    t0 = time.perf_counter()
    ref.synthetic_ensemble(n, NU, DT, steps, threads, threads, SEED, SIGMA, 4, keep=False)
    el = time.perf_counter() - t0
    value = threads * steps / el
    sample = (f"reference Solver (its CPU build, -O2, FP64) on this workload through its API "
              f"(update_latent_state + step, validate_step included) at {n}^2: {threads} members "
              f"x {steps} steps on {threads} threads, {el:.1f} s including set-up")
    return value, threads, sample


def cpu_filter_extrapolation(tc) -> dict:
    """Per-cycle cost of the reference's filters at the config-2 size, extrapolated from a
    measured single-thread member-step of its CPU solver at tc.n^2 (its filters advance the
    members one after another on one thread, src/filter.cpp:38-126, 204-356; the analysis is
    not included, so these are lower bounds)."""
    from oracle.oracle import Reference, params6
    ref = Reference()
    p = params6(tc.nu, 0.1, 0.2, 0.5, 2, 3)
    t0 = time.perf_counter()
    ref.ensemble(tc.n, p, tc.dt, 20, 1, 1, SEED)
    per_step = (time.perf_counter() - t0) / 20
    return {"member_step_seconds": per_step,
            "enkf_cycle_seconds": per_step * tc.enkf_members * tc.obs_every,
            "pf_cycle_seconds": per_step * tc.particles * tc.obs_every,
            "sample": f"hzl::ensemble on 1 thread, 1 member x 20 steps at {tc.n}^2, "
                      f"extrapolated to the forecast of one cycle (analysis not included)"}


def filter_experiment(cpu: bool) -> dict:
    """The 128^2 filtering twin experiment (hzl_stochasticflowinference_b200.twin)."""
    try:
        from hzl_stochasticflowinference_b200 import twin as T
        tc = T.FilterTwinConfig()
        t0 = time.perf_counter()
        res = T.run(tc)
        keep = ("initial_rmse", "mean_rmse", "final_rmse", "seconds_per_cycle")
        out = {"workload": f"{tc.n}^2 FP32 forecast, {len(T.observation_grid(tc)[0])} point "
                           f"observations (sigma {tc.obs_sd}) every {tc.obs_every} steps of dt "
                           f"{tc.dt}, {tc.cycles} cycles; EnKF {tc.enkf_members} members, "
                           f"inflation {tc.inflation}; bootstrap PF {tc.particles} particles, "
                           f"resampling when ESS < {tc.resample_fraction} x particles",
               "seconds": time.perf_counter() - t0,
               "enkf": {k: res["enkf"][k] for k in keep},
               "pf": {k: res["pf"][k] for k in keep}}
        out["pf"]["resampling_events"] = res["pf"]["resampling_events"]
        out["pf"]["min_ess"] = min(res["pf"]["ess"])
        if cpu:
            try:
                out["reference_cpu_extrapolated"] = cpu_filter_extrapolation(tc)
            except Exception as exc:
                out["reference_cpu_extrapolated"] = {"sample": f"unavailable: {exc}"}
        return out
    except Exception as exc:   # report, never lose the main line
        return {"error": f"{type(exc).__name__}: {exc}"}


def arm_config(members: int, world: int) -> dict:
    """The workload both arms report (the reference arm times a bounded sample of it)."""
    return {"workload": f"{N}^2 ensemble RK4 step, {members} members per GPU: nu {NU}, dt {DT}, "
                        f"Kolmogorov forcing 0.1 sin(4y), Euler-Maruyama noise sigma {SIGMA} on "
                        "1<=|k|<=4 (Philox keyed by seed and member), seeded random initial fields",
            "n": N, "members_per_gpu": members, "nu": NU, "dt": DT,
            "l2": "inputs larger than L2 (state + stage buffers ~2.5 GB per GPU)",
            "parallelism": f"member shards x{world}"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    value, threads, sample = cpu_reference_sample(N, seconds_target=max(5.0, 3.0 * args.steps))
    out = {
        "metric": METRIC, "value": value, "unit": "member-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * threads / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": arm_config(args.members, world),
        "cpu_baseline": {"value": value, "unit": "member-steps/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "member-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def reference_gpu_sample(n: int, steps: int = 20, members: int = 64) -> dict:
    """The reference's own cuFFT ensemble benchmark (oracle/_ref/hzl-cuda-ensemble-benchmark):
    its GPU member-steps/s at n^2 (its parameters: nu 0.01, friction 0.1, OU shell forcing,
    FP64, sequential launches per member)."""
    exe = ROOT / "oracle" / "_ref" / "hzl-cuda-ensemble-benchmark"
    if not exe.exists():
        return {"value": None, "unit": "member-steps/s",
                "sample": "unavailable: oracle/_ref/hzl-cuda-ensemble-benchmark not built"}
    workers = os.cpu_count() or 1
    cmd = [str(exe), str(n), str(steps), "0.00025", str(members), str(workers)]
    try:
        proc = subprocess.run(cmd, capture_output=True, text=True, timeout=600, check=True)
        res = json.loads(proc.stdout.strip().splitlines()[-1])
    except Exception as exc:   # report, never lose the main line
        return {"value": None, "unit": "member-steps/s", "sample": f"unavailable: {exc}"}
    return {"value": res["gpu_member_steps_per_second"], "unit": "member-steps/s",
            "kind": "reference cuFFT build (FP64)",
            "sample": f"{' '.join(['hzl-cuda-ensemble-benchmark'] + cmd[1:])}: {members} members x "
                      f"{steps} steps at {n}^2, its own CUDA path (cuFFT Z2Z FP64, one solver per "
                      f"member, sequential launches, host OU forcing upload per step); its CPU/GPU "
                      f"energy agreement {res['maximum_relative_energy_error']:.1e}",
            "evolution_seconds": res["gpu_evolution_seconds"]}


def build_ensemble(hz, precision: int, M: int, member_base: int, device: int):
    """The benchmark ensemble: M members at N^2 of the given precision (4 or 8), the seeded
    random fields of members member_base.., Kolmogorov forcing, Philox noise."""
    cfg = hz.Config(n=N, members=M, precision=precision, nu=NU, alpha=0.0, forcing_kmax=0,
                    noise_sigma=SIGMA, noise_kmax=4, seed=SEED, member_base=member_base,
                    device=device)
    ens = hz.Ensemble(cfg)
    dtype = np.complex64 if precision == 4 else np.complex128
    init = np.zeros((M, ens.compact_size), dtype)
    for m in range(M):
        init[m] = hz.full_to_compact(hz.grf_spectrum(N, SEED, member_base + m), N)[0]
    ens.set_state_compact(init)
    ens.set_forcing(hz.kolmogorov_forcing(N)[None])
    ens.set_time(0.0, 0)
    return ens


def launches(ens, steps: int) -> int:
    """Kernels `steps` single-step hzlb_step calls launch: a row and a column pass per RK
    stage, per member part when the step schedule runs the ensemble in two parts (256 members
    and more), plus the parts' control split and join once per call."""
    if ens.step_schedule() != "single" and ens.members >= 256:
        return (2 * 8 + 2) * steps
    return 8 * steps


def measure(hz, torch, ens, precision: int, steps: int, warmup: int, world: int, barrier,
            max_over_ranks, clocks=None) -> dict:
    """value (device-resident member-steps/s, CUDA events on the library stream around
    `steps` steps, max over ranks), roofline of the dominant kernel (this design's algorithmic
    bytes per launch over the launch's mean CUDA-event duration) and e2e (the same step through
    hzlb_step_host with the whole state copied from pinned host memory and back every step)."""
    M = ens.members
    stream = torch.cuda.ExternalStream(ens.stream)
    for _ in range(warmup):
        ens.step(DT, 1)
    ens.synchronize()
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if clocks is not None:
        clocks.__enter__()
    start.record(stream)
    for _ in range(steps):
        ens.step(DT, 1)
    stop.record(stream)
    ens.synchronize()
    barrier()
    if clocks is not None:
        clocks.__exit__(None, None, None)
    ms = max_over_ranks(start.elapsed_time(stop))
    status = ens.status()
    value = world * M * steps / (ms / 1e3)

    # roofline: per-launch events on the library stream
    row_ms, col_ms = ens.step_profiled(DT, max(2, steps // 4))
    K = (N - 1) // 3
    C, LD = K + 1, 2 * K + 1
    cb = 8 if precision == 4 else 16   # complex bytes
    # per launch: the row kernel reads the 2 velocity column fields and writes the 2 product
    # fields; the column kernel reads the 2 product fields, writes the 2 velocity fields and
    # reads/writes the compact state, stage input and accumulator (3, 5, 5, 4 entries per mode
    # on stages 1-4: 4.25 on average)
    row_bytes = M * (2 * C * N + 2 * C * N) * cb
    col_bytes = int(M * (2 * C * N + 2 * C * N + 4.25 * C * LD) * cb)
    row_gbs = row_bytes / (row_ms * 1e-3) / 1e9
    col_gbs = col_bytes / (col_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    dom = ("column_kernel", col_gbs, col_bytes, col_ms) if col_ms >= row_ms else \
        ("row_kernel", row_gbs, row_bytes, row_ms)
    traffic = NCU_TRAFFIC_PER_MEMBER[dom[0]] * M if precision == 4 else None
    model_bytes = (32 * 8 * N * (N // 2 + 1) + 16 * 8 * N * N) * (1 if precision == 4 else 2)
    roofline = {"bound": "hbm", "kernel": dom[0], "achieved": dom[1], "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": dom[1] / peak,
                "traffic": traffic, "algorithmic_bytes": dom[2], "launch_ms": dom[3],
                "row_kernel": {"ms": row_ms, "gbs": row_gbs, "frac": row_gbs / peak},
                "column_kernel": {"ms": col_ms, "gbs": col_gbs, "frac": col_gbs / peak},
                # the whole-step byte model of a schedule that moves five real fields per stage
                # (B32 = 32 S + 16 P, S = 8 N (N/2+1), P = 8 N^2 bytes; twice that in FP64);
                # this design moves fewer bytes, so this fraction exceeds 1
                "step_model": {"bytes_per_member_step": model_bytes,
                               "achieved": value * model_bytes / 1e9,
                               "frac": value * model_bytes / 1e9 / peak}}

    # e2e: host state in and out around every step
    state_bytes = M * ens.compact_size * cb
    view = np.float32 if precision == 4 else np.float64
    host_in = torch.from_numpy(ens.get_state_compact().view(view)).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    e2e_steps = max(3, steps // 2)
    for _ in range(2):
        ens.step_host_ptr(host_in.data_ptr(), host_out.data_ptr(), DT, 1)
    barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(e2e_steps):
        ens.step_host_ptr(host_in.data_ptr(), host_out.data_ptr(), DT, 1)
    t1.record(stream)
    ens.synchronize()
    barrier()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1))
    e2e = {"value": world * M * e2e_steps / (e2e_ms / 1e3), "unit": "member-steps/s",
           "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
           "steps": e2e_steps}
    return {"value": value, "ms_per_step": ms / steps, "status": status, "roofline": roofline,
            "e2e": e2e, "members": M, "steps": steps, "dtype": "f32" if precision == 4 else "f64",
            "gpu_launches": launches(ens, steps)}


def config1_experiment(hz) -> dict:
    """Config 1 at its own size: 256 members at 128^2, nu = dt = 5e-4, 2000 steps, from the
    same random fields and the same Philox noise in FP32 (complex64 spectra) and FP64.  Every
    250 steps, per member: the relative L2 error of the FP32 vorticity spectrum against the FP64
    one and the FP32 enstrophy drift |Z32 / Z64 - 1| (Z = A/2 sum |w_k|^2 over the whole
    spectrum; the compact half-spectrum's kx > 0 columns count twice).  The FP64 path itself
    equals the reference CPU solver to 1e-12 over these 2000 steps (tests/test_step_gpu.py)."""
    try:
        n, M, steps, every, dt, nu = 128, 256, 2000, 250, 5e-4, 5e-4
        ens = {}
        for prec in (4, 8):
            cfg = hz.Config(n=n, members=M, precision=prec, nu=nu, alpha=0.0, forcing_kmax=0,
                            noise_sigma=SIGMA, noise_kmax=4, seed=SEED)
            e = hz.Ensemble(cfg)
            init = np.array([hz.full_to_compact(hz.grf_spectrum(n, SEED, m), n)[0]
                             for m in range(M)])
            e.set_state_compact(init.astype(np.complex64 if prec == 4 else np.complex128))
            e.set_forcing(hz.kolmogorov_forcing(n)[None])
            e.set_time(0.0, 0)
            ens[prec] = e
        K = (n - 1) // 3
        w = np.full(ens[8].compact_size, 2.0)
        w[:2 * K + 1] = 1.0   # the kx = 0 column holds both signs of ky
        series, seconds = [], {4: 0.0, 8: 0.0}
        for done in range(every, steps + 1, every):
            for prec in (4, 8):
                t0 = time.perf_counter()
                ens[prec].step(dt, every)
                ens[prec].synchronize()
                seconds[prec] += time.perf_counter() - t0
            a = ens[4].get_state_compact().astype(np.complex128)
            b = ens[8].get_state_compact()
            za, zb = (w * np.abs(a) ** 2).sum(axis=1), (w * np.abs(b) ** 2).sum(axis=1)
            err = np.sqrt((w * np.abs(a - b) ** 2).sum(axis=1) / zb)
            drift = np.abs(za / zb - 1)
            series.append({"step": done, "l2_max": float(err.max()),
                           "l2_median": float(np.median(err)),
                           "l2_p90": float(np.percentile(err, 90)),
                           "enstrophy_drift_max": float(drift.max()),
                           "enstrophy_drift_median": float(np.median(drift))})
        status = {"f32": ens[4].status(), "f64": ens[8].status()}
        for e in ens.values():
            e.close()
        return {"workload": f"{M} members at {n}^2, nu {nu}, dt {dt}, {steps} steps, Kolmogorov "
                            f"forcing + sigma {SIGMA} Philox noise, seeded random fields; FP32 "
                            "against FP64 from identical inputs",
                "final": series[-1], "series": series, "status": status,
                "wall_seconds": {"f32": seconds[4], "f64": seconds[8]}}
    except Exception as exc:   # report, never lose the main line
        return {"error": f"{type(exc).__name__}: {exc}"}


def mixed_experiment() -> dict:
    try:
        from hzl_stochasticflowinference_b200 import batch
        t0 = time.perf_counter()
        res = batch.run()
        res["seconds"] = time.perf_counter() - t0
        peak, kind = peaks()
        res["tuned"]["frac_of_hbm"] = res["tuned"]["algorithmic_gbs"] / peak
        res["peak_kind"] = kind
        return res
    except Exception as exc:   # report, never lose the main line
        return {"error": f"{type(exc).__name__}: {exc}"}


LIKELIHOOD_CASES = [
    # name, n, dt, steps, every, noise, particles, replicates, reference sample (particles, replicates)
    ("calibration objective", 16, 0.01, 150, 10, 0.02, 32, 3, (32, 3)),
    ("batched replicates", 64, 0.005, 150, 10, 0.02, 256, 8, (32, 1)),
]


def likelihood_experiment(cpu: bool) -> dict:
    """averaged_particle_log_likelihood (src/filter.cpp:150-165) on a synthetic stochastic
    dataset made by the device truth run (synthetic_observations, the reference's defaults:
    truth nu 0.03, alpha 0.1, sigma 0.2, tau 0.5, shell 2..3, 8 sites every 10 steps): every
    replicate's particles advance as one ensemble.  Seconds per likelihood evaluation (wall
    clock, host OU forcing and resampling included) against the reference library's own
    function on the host (one thread per call, as it runs), timed on a bounded sample of
    particles x replicates and scaled to the workload (its cost is linear in both)."""
    try:
        import hzl_stochasticflowinference_b200 as hz
        truth = hz.Parameters(0.03, 0.1, 0.2, 0.5, 2, 3)
        q = np.log([0.03, 0.1, 0.2, 0.5])
        out = []
        for name, n, dt, steps, every, noise, P, R, (rp, rr) in LIKELIHOOD_CASES:
            ds = hz.synthetic_observations(n, truth, dt, steps, every, noise, 314159)
            hz.averaged_particle_log_likelihood(ds, q, P, R, 123)   # set-up, first-touch
            reps = 3
            t0 = time.perf_counter()
            for _ in range(reps):
                ll = hz.averaged_particle_log_likelihood(ds, q, P, R, 123)
            sec = (time.perf_counter() - t0) / reps
            row = {"workload": f"{name}: {n}^2, {steps} steps of dt {dt}, {len(ds['steps'])} "
                               f"observations, {P} particles x {R} replicates",
                   "seconds": sec, "member_steps_per_s": P * R * steps / sec,
                   "log_likelihood": ll}
            if cpu:
                try:
                    from oracle.oracle import Reference
                    ref = Reference()
                    t0 = time.perf_counter()
                    ref_ll = ref.particle_log_likelihood(ds, q, rp, 123, replicates=rr)
                    rs = (time.perf_counter() - t0) * (P * R) / (rp * rr)
                    row["reference_cpu"] = {
                        "seconds": rs, "member_steps_per_s": P * R * steps / rs,
                        "sample": f"{rp} particles x {rr} replicates, scaled by {P * R // (rp * rr)}",
                        "cores": 1}
                    row["speedup"] = rs / sec
                    if (rp, rr) == (P, R):
                        row["reference_log_likelihood"] = ref_ll
                except Exception as exc:
                    row["reference_cpu"] = {"sample": f"unavailable: {exc}"}
            out.append(row)
        return {"cases": out}
    except Exception as exc:   # report, never lose the main line
        return {"error": f"{type(exc).__name__}: {exc}"}


def tangent_experiment(cpu: bool, n: int = 128, count: int = 1024, sample: int = 16) -> dict:
    """Batched Solver::linearized_drift / adjoint_drift (src/solver.cpp:264-324), FP64, `count`
    (state, field) pairs of n^2 spectra per call from host memory (wall clock, transfers
    included), against the reference library's own functions on the host (one thread, one pair
    per call as its adjoint loop calls them), timed on `sample` pairs and scaled to `count`."""
    try:
        import hzl_stochasticflowinference_b200 as hz
        rng = np.random.default_rng(SEED)
        k = np.fft.fftfreq(n, 1 / n).astype(int)
        mask = (3 * np.abs(k)[None, :] < n) & (3 * np.abs(k)[:, None] < n)
        mask[0, 0] = False

        def fields(c):
            return np.fft.fft2(rng.normal(size=(c, n, n)), axes=(1, 2)) / n ** 2 * mask

        w, d = fields(count), fields(count)
        p = hz.Parameters(0.02, 0.1, 0.2, 0.5, 2, 3)
        out = {"workload": f"{count} pairs at {n}^2 per call, FP64, host arrays"}
        for name, fn in (("linearized_drift", hz.linearized_drift), ("adjoint_drift", hz.adjoint_drift)):
            fn(n, p, w[:8], d[:8])
            t0 = time.perf_counter()
            fn(n, p, w, d)
            sec = time.perf_counter() - t0
            row = {"seconds": sec, "pairs_per_s": count / sec}
            if cpu:
                try:
                    from oracle.oracle import Reference, params6
                    s = Reference().solver(n, params6(0.02, 0.1, 0.2, 0.5, 2, 3), 1)
                    t0 = time.perf_counter()
                    for i in range(sample):
                        getattr(s, name)(w[i], d[i])
                    rs = (time.perf_counter() - t0) / sample
                    row["reference_cpu"] = {"pairs_per_s": 1 / rs, "cores": 1,
                                            "sample": f"{sample} pairs, one call each"}
                    row["speedup"] = (count / sec) * rs
                except Exception as exc:
                    row["reference_cpu"] = {"sample": f"unavailable: {exc}"}
            out[name] = row
        out["likelihood_adjoint"] = adjoint_gradient_sample(cpu)
        return out
    except Exception as exc:   # report, never lose the main line
        return {"error": f"{type(exc).__name__}: {exc}"}


def adjoint_gradient_sample(cpu: bool, vectors: int = 64, sample: int = 2) -> dict:
    """likelihood_adjoint (src/adjoint.cpp:43-161) for `vectors` (log nu, log alpha) points in
    one call, on a deterministic dataset from the device truth run with the reference's
    observation defaults (16^2, 150 steps of dt 0.01, 8 sites every 10 steps), checkpoint
    stride 20; against the reference library's one call per point on one host thread."""
    import hzl_stochasticflowinference_b200 as hz
    ds = hz.synthetic_observations(16, hz.Parameters(0.03, 0.1, 0.0, 0.5, 2, 3), 0.01, 150, 10,
                                   0.02, 314159)
    rng = np.random.default_rng(SEED)
    q = np.stack([rng.uniform(np.log(0.01), np.log(0.08), vectors),
                  rng.uniform(np.log(0.05), np.log(0.3), vectors)], axis=1)
    hz.likelihood_adjoint(ds, q[:2], 20)
    t0 = time.perf_counter()
    got = hz.likelihood_adjoint(ds, q, 20)
    sec = time.perf_counter() - t0
    row = {"workload": f"{vectors} parameter vectors per call, 16^2, 150 steps, stride 20",
           "seconds": sec, "gradients_per_s": vectors / sec,
           "replayed_steps": int(got[0]["replayed_steps"])}
    if cpu:
        try:
            from oracle.oracle import Reference
            ref = Reference()
            t0 = time.perf_counter()
            for i in range(sample):
                r = ref.likelihood_adjoint(ds, q[i], 20)
            rs = (time.perf_counter() - t0) / sample
            row["reference_cpu"] = {"gradients_per_s": 1 / rs, "cores": 1,
                                    "sample": f"{sample} points, one call each"}
            row["speedup"] = (vectors / sec) * rs
            row["max_rel_gradient_difference_sampled"] = float(np.max(
                np.abs(got[sample - 1]["gradient"] - r["gradient"]) / np.abs(r["gradient"])))
        except Exception as exc:
            row["reference_cpu"] = {"sample": f"unavailable: {exc}"}
    return row


def learned_experiment() -> dict:
    """The learned-forecast EnKF twin experiment (hzl_stochasticflowinference_b200.learned) at
    its full size; wall-clock per cycle (forecast + analysis + fallback) with the GPU
    synchronised, the first cycle of each filter excluded as set-up."""
    try:
        from hzl_stochasticflowinference_b200 import learned as L
        tc = L.TwinConfig()
        t0 = time.perf_counter()
        res = L.run(tc)
        keep = ("mean_rmse", "final_rmse", "seconds_per_cycle", "fallback_cycles", "speedup",
                "rmse_ratio")
        out = {"workload": f"{tc.n}^2 FP32, EnKF {tc.members} members, {len(L.observation_grid(tc)[0])} "
                           f"point observations (sigma {tc.obs_sd}) every {tc.window} steps of dt "
                           f"{tc.dt}, {tc.cycles} cycles; POD r={tc.rank} from {tc.snapshots} "
                           f"snapshots; MLP {tc.rank + 8}-{tc.hidden}-{tc.hidden}-{tc.rank} BF16 "
                           f"trained on {res['transitions']} transitions; NIS fallback limit "
                           f"{tc.nis_limit}",
               "seconds": time.perf_counter() - t0,
               "pod": {"captured": res["pod"]["captured"], "residual": res["pod"]["residual"],
                       "seconds": res["pod_seconds"]},
               "network": {k: res["training"][k] for k in ("val_mse_network",
                                                           "val_mse_persistence", "val_skill",
                                                           "train_seconds", "train_steps")},
               "data_seconds": res["data_seconds"]}
        for mode in ("spectral", "learned", "hybrid", "complement", "persistence",
                     "hybrid_persistence", "complement_persistence"):
            out[mode] = {k: res[mode][k] for k in keep if k in res[mode]}
        # the variant whose POD coefficients move by the network alone (the one-member
        # spectral step of the mean supplies only the motion outside the POD space), with the
        # same pipeline's network-off ablation beside it
        out["headline"] = {"mode": "complement", "rmse_ratio": res["rmse_ratio"],
                           "speedup": res["speedup"],
                           "network_off_rmse_ratio": res["complement_persistence"]["rmse_ratio"]}
        return out
    except Exception as exc:   # report, never lose the main line
        return {"error": f"{type(exc).__name__}: {exc}"}


def run_case(case: str, steps: int, warmup: int) -> None:
    """Isolated workloads for micro-benchmarks and small profiler captures."""
    import ctypes as C
    import torch
    import hzl_stochasticflowinference_b200 as hz
    from hzl_stochasticflowinference_b200 import learned as L
    steps, warmup = max(1, min(steps, 10)), max(1, min(warmup, 3))
    ev = lambda: torch.cuda.Event(enable_timing=True)   # noqa: E731
    out = {"case": case}
    if case == "likelihood":
        print(json.dumps({"case": case, **likelihood_experiment(True)}), flush=True)
        return
    if case == "tangent":
        print(json.dumps({"case": case, **tangent_experiment(True)}), flush=True)
        return
    if case == "gemm":
        lib = hz.library()
        fn = lib.hzlb_gemm
        fn.restype = C.c_int
        fn.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_longlong,
                                       C.c_int, C.c_void_p, C.c_longlong, C.c_float, C.c_float,
                                       C.c_void_p]
        n = 4096
        for name, code, dt in (("tf32", 4, torch.float32), ("bf16", 2, torch.bfloat16)):
            a = torch.randn(n, n, device="cuda").to(dt)
            b = torch.randn(n, n, device="cuda").to(dt)
            c = torch.zeros(n, n, device="cuda")
            s = torch.cuda.current_stream().cuda_stream
            run = lambda: fn(n, n, n, code, a.data_ptr(), n, 1, b.data_ptr(), n, 1,  # noqa: E731
                             c.data_ptr(), n, 1.0, 0.0, s)
            for _ in range(warmup):
                assert run() == 0
            t0, t1 = ev(), ev()
            t0.record()
            for _ in range(steps):
                run()
            t1.record()
            torch.cuda.synchronize()
            ms = t0.elapsed_time(t1) / steps
            out[name] = {"ms": ms, "tflops": 2 * n ** 3 / ms / 1e9, "shape": [n, n, n]}
    else:
        tc = L.TwinConfig()
        cfg = tc.config(tc.members, 0)
        e = hz.Ensemble(cfg)
        e.set_forcing(hz.kolmogorov_forcing(tc.n, tc.forcing_amplitude, tc.forcing_wavenumber))
        init = np.zeros((tc.members, e.compact_size), np.complex64)
        g = hz.full_to_compact(hz.grf_spectrum(tc.n, SEED, 0), tc.n)[0]
        for m in range(tc.members):
            init[m] = g + L.perturbation(tc, m)
        e.set_state_compact(init)
        e.synchronize()
        xs, ys = L.observation_grid(tc)
        vals, sd = np.zeros(len(xs)), np.full(len(xs), tc.obs_sd)
        if case == "enkf":
            work = lambda i: e.enkf_analysis_nis(xs, ys, vals, sd, None, seed=1, cycle=i)  # noqa: E731
        else:
            # the window's cost does not depend on the basis: one fitted to seeded random
            # snapshots keeps the case's set-up to a few launches (profiler captures included)
            g = torch.Generator(device="cuda").manual_seed(SEED)
            snaps = torch.randn((4 * tc.rank, 2 * e.compact_size), device="cuda", generator=g)
            pod = hz.Pod(tc.n, snaps, tc.rank, seed=1)
            del snaps
            net = hz.Mlp(tc.rank, 8, tc.hidden, tc.members, seed=1)
            work = lambda i: e.learned_forecast(pod, net, tc.dt, tc.window)  # noqa: E731
        for i in range(warmup):
            work(i)
        e.synchronize()
        t = time.perf_counter()
        for i in range(steps):
            work(warmup + i)
        e.synchronize()
        out["ms"] = (time.perf_counter() - t) * 1e3 / steps
        out["members"], out["observations"] = tc.members, len(xs)
        e.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--members", type=int, default=MEMBERS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--step-schedule", choices=["single", "parts", "offset_parts"],
                    help="hzlb_set_step_schedule for the main and FP64 legs (default: the "
                         "library's, two member parts from 256 members)")
    ap.add_argument("--case", choices=["gemm", "enkf", "learned", "likelihood", "tangent"])
    args = ap.parse_args()
    if args.case:
        run_case(args.case, args.steps, args.warmup)
        return
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import hzl_stochasticflowinference_b200 as hz

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    M = args.members

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    def max_over_ranks(x: float) -> float:
        if not pg:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    # ---- the headline: FP32 at 256^2 --------------------------------------------------
    ens = build_ensemble(hz, 4, M, rank * M, local)
    if args.step_schedule:
        ens.set_step_schedule(args.step_schedule)
    clocks = ClockSampler(local)
    main_leg = measure(hz, torch, ens, 4, args.steps, args.warmup, world, barrier, max_over_ranks,
                       clocks)
    ens.close()
    # ---- the same workload in FP64 (the reference's precision), same members and steps ----
    ens = build_ensemble(hz, 8, M, rank * M, local)
    if args.step_schedule:
        ens.set_step_schedule(args.step_schedule)
    fp64 = measure(hz, torch, ens, 8, args.steps, args.warmup, world, barrier, max_over_ranks)
    ens.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, cores, sample = cpu_reference_sample(N)
            cpu = {"value": v, "unit": "member-steps/s", "cores": cores, "kind": "reference",
                   "sample": sample}
        except Exception as exc:   # the reference library is test infrastructure; report why
            cpu = {"value": None, "unit": "member-steps/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {exc}"}
    if cpu and cpu.get("value"):
        fp64["vs_cpu_reference"] = fp64["value"] / cpu["value"]
        fp64["e2e"]["vs_cpu_reference"] = fp64["e2e"]["value"] / cpu["value"]

    learned = gpu_ref = filters = mixed = likelihood = tangent = config1 = None
    if rank == 0 and world == 1:
        if not args.no_cpu_baseline:
            gpu_ref = reference_gpu_sample(N)
        config1 = config1_experiment(hz)
        if not args.no_learned:
            learned = learned_experiment()
            filters = filter_experiment(not args.no_cpu_baseline)
            mixed = mixed_experiment()
            likelihood = likelihood_experiment(not args.no_cpu_baseline)
            tangent = tangent_experiment(not args.no_cpu_baseline)

    if rank == 0:
        out = {
            "metric": METRIC, "value": main_leg["value"], "unit": "member-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": main_leg["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": arm_config(M, world),
            "roofline": main_leg["roofline"],
            "e2e": main_leg["e2e"],
            "gpu_launches": main_leg["gpu_launches"],
            "clocks": clocks.summary(),
            "status": main_leg["status"],
            "cpu_baseline": cpu,
            # the same workload in FP64, the reference's precision: like-for-like with the
            # reference arm and with gpu_reference
            "fp64": fp64,
            "gpu_reference": gpu_ref,
            "config1": config1,
            "learned": learned,
            "filters": filters,
            "mixed": mixed,
            "likelihood": likelihood,
            "tangent": tangent,
        }
        print(json.dumps(out), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
