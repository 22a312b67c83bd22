"""TEST INFRASTRUCTURE ONLY: ctypes bindings to the two CPU checkers.

* ``Oracle`` wraps ``oracle/liboracle.so``, the C restatement of the reference algorithm
  (``hzl_oracle.c``; every function there cites the reference file:line it follows).
* ``Reference`` wraps ``oracle/_ref/libhzlref.so``, the reference's own CPU library compiled
  from its sources by ``oracle/Makefile`` plus the C wrapper ``ref_capi.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import this module.
Complex fields are numpy complex128 arrays of shape (n, n) indexed [y, x], the reference
layout (include/hzl/fft.hpp:7-8).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libhzlref.so"

_dp = C.POINTER(C.c_double)
_u64 = C.c_uint64
_u32p = C.POINTER(C.c_uint32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def params6(nu, alpha, sigma, tau, kmin, kmax) -> np.ndarray:
    return np.array([nu, alpha, sigma, tau, kmin, kmax], dtype=np.float64)


class OracleError(RuntimeError):
    pass


class Oracle:
    """The C restatement (hzl_oracle.c)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built; run `make -C oracle`")
        lib = C.CDLL(str(path))
        self.lib = lib
        lib.ho_last_error.restype = C.c_char_p
        lib.ho_stream_seed.restype = _u64
        lib.ho_stream_seed.argtypes = [_u64, _u64]
        lib.ho_mode_code.restype = C.c_uint32
        lib.ho_mode_code.argtypes = [C.c_int, C.c_int]
        lib.ho_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        lib.ho_philox_normal_pair.argtypes = [_u64, C.c_uint32, _u64, C.c_uint32, _dp, _dp]
        lib.ho_fft.argtypes = [C.c_int, _dp, C.c_int]
        lib.ho_solver_create.argtypes = [C.c_int, _dp, _u64, C.POINTER(C.c_void_p)]
        lib.ho_solver_destroy.argtypes = [C.c_void_p]
        lib.ho_solver_initialize.argtypes = [C.c_void_p, C.c_char_p]
        lib.ho_solver_initialize_physical.argtypes = [C.c_void_p, _dp]
        lib.ho_solver_set_state.argtypes = [C.c_void_p, _dp, _dp]
        lib.ho_solver_get_state.argtypes = [C.c_void_p, _dp, _dp]
        lib.ho_solver_midpoint_forcing.argtypes = [C.c_void_p, _dp]
        lib.ho_solver_step.argtypes = [C.c_void_p, C.c_double]
        lib.ho_solver_step_forced.argtypes = [C.c_void_p, C.c_double, _dp]
        lib.ho_solver_diagnostics.argtypes = [C.c_void_p, _dp]
        lib.ho_solver_physical_vorticity.argtypes = [C.c_void_p, _dp]
        lib.ho_solver_update_latent_state.argtypes = [C.c_void_p, _dp, _dp]
        lib.ho_solver_time.restype = C.c_double
        lib.ho_solver_time.argtypes = [C.c_void_p]
        lib.ho_solver_reseed_future.argtypes = [C.c_void_p, _u64]
        lib.ho_grf_spectrum.argtypes = [C.c_int, _u64, C.c_uint32, _dp]
        lib.ho_kolmogorov_forcing.argtypes = [C.c_int, C.c_double, C.c_int, _dp]
        lib.ho_add_noise.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_int, _u64,
                                     C.c_uint32, _u64]
        lib.ho_synthetic_step.argtypes = [C.c_void_p, C.c_double, _dp, C.c_double, C.c_int, _u64,
                                          C.c_uint32, _u64]
        lib.ho_pf_weights.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp]
        lib.ho_systematic_resample.argtypes = [C.c_int, _dp, C.c_double, _u32p]
        lib.ho_resampling_uniform.restype = C.c_double
        lib.ho_resampling_uniform.argtypes = [_u64]
        lib.ho_enkf_scalar_update.argtypes = [C.c_int, C.POINTER(C.c_void_p), _dp, C.c_double,
                                              C.c_double, _dp]
        lib.ho_fit_pod.argtypes = [C.c_int, C.c_int64, _dp, C.c_int, C.c_double,
                                   C.POINTER(C.c_int), _dp, _dp, _dp, _dp]

    def check(self, rc: int):
        if rc != 0:
            raise OracleError(self.lib.ho_last_error().decode())

    # -- random numbers --------------------------------------------------------------
    def stream_seed(self, base: int, index: int) -> int:
        return int(self.lib.ho_stream_seed(base, index))

    def philox(self, ctr, key) -> np.ndarray:
        c = np.ascontiguousarray(ctr, dtype=np.uint32)
        k = np.ascontiguousarray(key, dtype=np.uint32)
        out = np.zeros(4, dtype=np.uint32)
        self.lib.ho_philox4x32_10(c.ctypes.data_as(_u32p), k.ctypes.data_as(_u32p),
                                  out.ctypes.data_as(_u32p))
        return out

    # -- transform -------------------------------------------------------------------
    def fft(self, field: np.ndarray, inverse: bool) -> np.ndarray:
        a = np.ascontiguousarray(field, dtype=np.complex128).copy()
        self.check(self.lib.ho_fft(a.shape[0], _ptr(a), int(inverse)))
        return a

    # -- synthetic workload ----------------------------------------------------------
    def grf(self, n: int, seed: int, member: int) -> np.ndarray:
        a = np.zeros((n, n), np.complex128)
        self.check(self.lib.ho_grf_spectrum(n, seed, member, _ptr(a)))
        return a

    def kolmogorov(self, n: int, amplitude: float = 0.1, wavenumber: int = 4) -> np.ndarray:
        a = np.zeros((n, n), np.complex128)
        self.check(self.lib.ho_kolmogorov_forcing(n, amplitude, wavenumber, _ptr(a)))
        return a

    def add_noise(self, omega: np.ndarray, sigma, dt, kmax, seed, member, step) -> np.ndarray:
        a = np.ascontiguousarray(omega, dtype=np.complex128).copy()
        self.check(self.lib.ho_add_noise(a.shape[0], _ptr(a), sigma, dt, kmax, seed, member, step))
        return a

    # -- filters ---------------------------------------------------------------------
    def pf_weights(self, logs: np.ndarray):
        logs = np.ascontiguousarray(logs, dtype=np.float64)
        w = np.zeros_like(logs)
        inc, ess, mw = C.c_double(), C.c_double(), C.c_double()
        self.check(self.lib.ho_pf_weights(len(logs), _ptr(logs), _ptr(w), C.byref(inc),
                                          C.byref(ess), C.byref(mw)))
        return w, inc.value, ess.value, mw.value

    def systematic_resample(self, weights: np.ndarray, u: float) -> np.ndarray:
        weights = np.ascontiguousarray(weights, dtype=np.float64)
        out = np.zeros(len(weights), np.uint32)
        self.check(self.lib.ho_systematic_resample(len(weights), _ptr(weights), u,
                                                   out.ctypes.data_as(_u32p)))
        return out

    def fit_pod(self, snapshots: np.ndarray, max_rank: int, fraction: float = 0.9999):
        s = np.ascontiguousarray(snapshots.reshape(len(snapshots), -1), dtype=np.complex128)
        m, dim = s.shape
        mean = np.zeros(dim, np.complex128)
        modes = np.zeros((max_rank, dim), np.complex128)
        sv = np.zeros(max_rank)
        rank, cap = C.c_int(), C.c_double()
        self.check(self.lib.ho_fit_pod(m, dim, _ptr(s), max_rank, fraction, C.byref(rank),
                                       _ptr(mean), _ptr(modes), _ptr(sv), C.byref(cap)))
        r = rank.value
        return mean, modes[:r].copy(), sv[:r].copy(), cap.value

    def solver(self, n: int, p6, seed: int) -> "OracleSolver":
        return OracleSolver(self, n, p6, seed)


class OracleSolver:
    def __init__(self, o: Oracle, n: int, p6, seed: int):
        self.o, self.n = o, n
        self.h = C.c_void_p()
        p = np.ascontiguousarray(p6, dtype=np.float64)
        o.check(o.lib.ho_solver_create(n, _ptr(p), seed, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.o.lib.ho_solver_destroy(self.h)
            self.h = None

    def initialize(self, name: str):
        self.o.check(self.o.lib.ho_solver_initialize(self.h, name.encode()))

    def initialize_physical(self, field: np.ndarray):
        a = np.ascontiguousarray(field, dtype=np.complex128)
        self.o.check(self.o.lib.ho_solver_initialize_physical(self.h, _ptr(a)))

    def set_state(self, omega=None, forcing=None):
        w = None if omega is None else np.ascontiguousarray(omega, dtype=np.complex128)
        f = None if forcing is None else np.ascontiguousarray(forcing, dtype=np.complex128)
        self.o.check(self.o.lib.ho_solver_set_state(self.h, None if w is None else _ptr(w),
                                                    None if f is None else _ptr(f)))

    def state(self):
        w = np.zeros((self.n, self.n), np.complex128)
        f = np.zeros_like(w)
        self.o.check(self.o.lib.ho_solver_get_state(self.h, _ptr(w), _ptr(f)))
        return w, f

    def step(self, dt: float, steps: int = 1):
        for _ in range(steps):
            self.o.check(self.o.lib.ho_solver_step(self.h, dt))

    def step_forced(self, dt: float, forcing=None):
        f = None if forcing is None else np.ascontiguousarray(forcing, dtype=np.complex128)
        self.o.check(self.o.lib.ho_solver_step_forced(self.h, dt, None if f is None else _ptr(f)))

    def synthetic_step(self, dt, forcing, sigma, kmax, seed, member, step):
        f = np.ascontiguousarray(forcing, dtype=np.complex128)
        self.o.check(self.o.lib.ho_synthetic_step(self.h, dt, _ptr(f), sigma, kmax, seed, member,
                                                  step))

    def diagnostics(self) -> np.ndarray:
        d = np.zeros(6)
        self.o.check(self.o.lib.ho_solver_diagnostics(self.h, _ptr(d)))
        return d

    def physical_vorticity(self) -> np.ndarray:
        a = np.zeros((self.n, self.n), np.complex128)
        self.o.check(self.o.lib.ho_solver_physical_vorticity(self.h, _ptr(a)))
        return a

    def midpoint_forcing(self) -> np.ndarray:
        a = np.zeros((self.n, self.n), np.complex128)
        self.o.check(self.o.lib.ho_solver_midpoint_forcing(self.h, _ptr(a)))
        return a

    def update_latent_state(self, omega, forcing):
        w = np.ascontiguousarray(omega, dtype=np.complex128)
        f = np.ascontiguousarray(forcing, dtype=np.complex128)
        self.o.check(self.o.lib.ho_solver_update_latent_state(self.h, _ptr(w), _ptr(f)))

    def reseed_future(self, seed: int):
        self.o.lib.ho_solver_reseed_future(self.h, seed)


class Reference:
    """The reference's own CPU library (oracle/_ref/libhzlref.so)."""

    def __init__(self, path: Path = REF_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built; run `make -C oracle` where the "
                                    "reference sources are present")
        lib = C.CDLL(str(path))
        self.lib = lib
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_stream_seed.restype = _u64
        lib.ref_stream_seed.argtypes = [_u64, _u64]
        lib.ref_fft.argtypes = [C.c_int, _dp, C.c_int]
        lib.ref_solver_create.argtypes = [C.c_int, _dp, _u64, C.POINTER(C.c_void_p)]
        lib.ref_solver_destroy.argtypes = [C.c_void_p]
        for name in ("initialize",):
            getattr(lib, f"ref_solver_{name}").argtypes = [C.c_void_p, C.c_char_p]
        lib.ref_solver_initialize_physical.argtypes = [C.c_void_p, _dp]
        lib.ref_solver_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
        for name in ("coefficients", "forcing", "midpoint_forcing", "diagnostics",
                     "physical_vorticity"):
            getattr(lib, f"ref_solver_{name}").argtypes = [C.c_void_p, _dp]
        lib.ref_solver_update_latent_state.argtypes = [C.c_void_p, _dp, _dp]
        lib.ref_solver_drift.argtypes = [C.c_void_p, _dp, _dp]
        lib.ref_solver_reseed_future.argtypes = [C.c_void_p, _u64]
        lib.ref_shell_forcing_create.argtypes = [C.c_int, _dp, _u64, C.POINTER(C.c_void_p)]
        lib.ref_shell_forcing_destroy.argtypes = [C.c_void_p]
        lib.ref_shell_forcing_midpoint_step.argtypes = [C.c_void_p, C.c_double, _dp]
        lib.ref_shell_forcing_coefficients.argtypes = [C.c_void_p, _dp]
        lib.ref_ensemble.argtypes = [C.c_int, _dp, C.c_double, _u64, _u64, _u64, _u64, _dp]
        lib.ref_synthetic_ensemble.argtypes = [C.c_int, C.c_double, C.c_double, _u64, _u64, _u64,
                                               _u64, C.c_double, C.c_int, _dp]
        u64p = C.POINTER(_u64)
        lib.ref_synthetic_observations.argtypes = [C.c_int, C.c_double, _u64, _u64, _dp, C.c_double,
                                                   _u64, _u64, u64p, u64p, _u32p, _u32p, _dp, _dp]
        lib.ref_bootstrap_filter.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _u64,
                                             u64p, _u32p, _u32p, _dp, _dp, _dp, _u64, _u64, C.c_int,
                                             _dp, u64p, _u64, u64p, _dp, _dp]
        lib.ref_solver_save.argtypes = [C.c_void_p, C.c_char_p]
        lib.ref_solver_linearized_drift.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.ref_solver_adjoint_drift.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.ref_solver_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        lib.ref_solver_size.argtypes = [C.c_void_p]
        lib.ref_likelihood_adjoint.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                               _u64, u64p, _u32p, _u32p, _dp, _dp, _dp, _u64, _dp,
                                               _dp, u64p]
        lib.ref_dataset_save.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _u64,
                                         u64p, _u32p, _u32p, _dp, _dp, C.c_char_p]
        ip = C.POINTER(C.c_int)
        lib.ref_dataset_load.argtypes = [C.c_char_p, _u64, ip, _dp, ip, ip, ip, u64p, u64p,
                                         _u32p, _u32p, _dp, _dp]
        lib.ref_particle_log_likelihood.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                                    _u64, u64p, _u32p, _u32p, _dp, _dp, _dp, _u64,
                                                    _u64, _u64, C.c_int, _dp]
        lib.ref_enkf.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _u64, u64p, _u32p,
                                 _u32p, _dp, _dp, _dp, _u64, _u64, C.c_double, C.c_double, _u64,
                                 _u64, _u64, u64p, _dp, _dp]
        lib.ref_fit_pod.argtypes = [_u64, _u64, _dp, _u64, C.c_double, u64p, _dp, _dp, _dp, _dp]
        lib.ref_galerkin.argtypes = [C.c_int, _dp, _u64, _dp, _dp, _u64, _dp, _dp, _dp, C.c_double,
                                     _u64]

    def check(self, rc: int):
        if rc != 0:
            raise OracleError(self.lib.ref_last_error().decode())

    def stream_seed(self, base: int, index: int) -> int:
        return int(self.lib.ref_stream_seed(base, index))

    def fft(self, field: np.ndarray, inverse: bool) -> np.ndarray:
        a = np.ascontiguousarray(field, dtype=np.complex128).copy()
        self.check(self.lib.ref_fft(a.shape[0], _ptr(a), int(inverse)))
        return a

    def solver(self, n: int, p6, seed: int) -> "ReferenceSolver":
        return ReferenceSolver(self, n, p6, seed)

    def synthetic_ensemble(self, n: int, nu: float, dt: float, steps: int, count: int,
                           workers: int, seed: int, sigma: float = 0.05, noise_kmax: int = 4,
                           keep: bool = True):
        """The benchmark's seeded-synthetic workload through the reference's Solver API on
        `workers` threads (ref_synthetic_ensemble); final spectra (count, n, n) or None."""
        out = np.zeros((count, n, n), np.complex128) if keep else None
        self.check(self.lib.ref_synthetic_ensemble(n, nu, dt, steps, count, workers, seed, sigma,
                                                   noise_kmax, _ptr(out) if keep else None))
        return out

    def solver_load(self, path) -> "ReferenceSolver":
        """Solver::load (src/solver.cpp:453-491)."""
        h = C.c_void_p()
        self.check(self.lib.ref_solver_load(str(path).encode(), C.byref(h)))
        s = ReferenceSolver.__new__(ReferenceSolver)
        s.r, s.h = self, h
        s.n = int(self.lib.ref_solver_size(h))
        return s

    def shell_forcing(self, n: int, p6, seed: int) -> "ReferenceShellForcing":
        return ReferenceShellForcing(self, n, p6, seed)

    def ensemble(self, n, p6, dt, steps, count, workers, seed) -> np.ndarray:
        p = np.ascontiguousarray(p6, dtype=np.float64)
        out = np.zeros((count, 6))
        self.check(self.lib.ref_ensemble(n, _ptr(p), dt, steps, count, workers, seed, _ptr(out)))
        return out

    def synthetic_observations(self, n, dt, steps, every, p6, noise, seed):
        cap = (steps // every) * 8 + 8 if every else 8
        count = _u64()
        st = np.zeros(cap, np.uint64)
        xs = np.zeros(cap, np.uint32)
        ys = np.zeros(cap, np.uint32)
        vals = np.zeros(cap)
        sds = np.zeros(cap)
        p = np.ascontiguousarray(p6, dtype=np.float64)
        self.check(self.lib.ref_synthetic_observations(
            n, dt, steps, every, _ptr(p), noise, seed, cap, C.byref(count),
            st.ctypes.data_as(C.POINTER(_u64)), xs.ctypes.data_as(_u32p),
            ys.ctypes.data_as(_u32p), _ptr(vals), _ptr(sds)))
        k = count.value
        return dict(n=n, dt=dt, stochastic=int(p6[2] > 0), forcing_min=int(p6[4]),
                    forcing_max=int(p6[5]), steps=st[:k].copy(), x=xs[:k].copy(), y=ys[:k].copy(),
                    value=vals[:k].copy(), sd=sds[:k].copy())

    def _ds_args(self, ds):
        st = np.ascontiguousarray(ds["steps"], dtype=np.uint64)
        xs = np.ascontiguousarray(ds["x"], dtype=np.uint32)
        ys = np.ascontiguousarray(ds["y"], dtype=np.uint32)
        vals = np.ascontiguousarray(ds["value"], dtype=np.float64)
        sds = np.ascontiguousarray(ds["sd"], dtype=np.float64)
        keep = (st, xs, ys, vals, sds)
        args = [ds["n"], ds["dt"], ds["stochastic"], ds["forcing_min"], ds["forcing_max"], len(st),
                st.ctypes.data_as(C.POINTER(_u64)), xs.ctypes.data_as(_u32p),
                ys.ctypes.data_as(_u32p), _ptr(vals), _ptr(sds)]
        return args, keep

    def bootstrap_filter(self, ds, p6, particles, seed, retain=True):
        args, keep = self._ds_args(ds)
        groups_cap = len(np.unique(ds["steps"])) + 1
        n = ds["n"]
        ll = C.c_double()
        ev, groups = _u64(), _u64()
        rec = np.zeros((groups_cap, 4))
        means = np.zeros((groups_cap, n, n), np.complex128)
        p = np.ascontiguousarray(p6, dtype=np.float64)
        self.check(self.lib.ref_bootstrap_filter(*args, _ptr(p), particles, seed, int(retain),
                                                 C.byref(ll), C.byref(ev), groups_cap,
                                                 C.byref(groups), _ptr(rec), _ptr(means)))
        g = groups.value
        return dict(log_likelihood=ll.value, resampling_events=ev.value, records=rec[:g].copy(),
                    means=means[:g].copy())

    def likelihood_adjoint(self, ds, q, stride=20):
        """likelihood_adjoint (src/adjoint.cpp:43-161)."""
        args, keep = self._ds_args(ds)
        qa = np.ascontiguousarray(q, dtype=np.float64)
        value = C.c_double()
        grad = np.zeros(2)
        counters = np.zeros(3, np.uint64)
        self.check(self.lib.ref_likelihood_adjoint(*args, _ptr(qa), stride, C.byref(value),
                                                   _ptr(grad),
                                                   counters.ctypes.data_as(C.POINTER(_u64))))
        return dict(value=value.value, gradient=grad, checkpoint_fields=int(counters[0]),
                    peak_block_fields=int(counters[1]), replayed_steps=int(counters[2]))

    def dataset_save(self, ds, path):
        """Dataset::save (src/inference.cpp:214-226)."""
        args, keep = self._ds_args(ds)
        self.check(self.lib.ref_dataset_save(*args, str(path).encode()))

    def dataset_load(self, path, capacity=100000):
        """Dataset::load (src/inference.cpp:227-257)."""
        n, stochastic, fmin, fmax = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        dt, count = C.c_double(), _u64()
        st = np.zeros(capacity, np.uint64)
        xs = np.zeros(capacity, np.uint32)
        ys = np.zeros(capacity, np.uint32)
        vals = np.zeros(capacity)
        sds = np.zeros(capacity)
        self.check(self.lib.ref_dataset_load(
            str(path).encode(), capacity, C.byref(n), C.byref(dt), C.byref(stochastic),
            C.byref(fmin), C.byref(fmax), C.byref(count), st.ctypes.data_as(C.POINTER(_u64)),
            xs.ctypes.data_as(_u32p), ys.ctypes.data_as(_u32p), _ptr(vals), _ptr(sds)))
        k = count.value
        return dict(n=n.value, dt=dt.value, stochastic=stochastic.value, forcing_min=fmin.value,
                    forcing_max=fmax.value, steps=st[:k].copy(), x=xs[:k].copy(),
                    y=ys[:k].copy(), value=vals[:k].copy(), sd=sds[:k].copy())

    def particle_log_likelihood(self, ds, q, particles, seed, replicates=None):
        """particle_log_likelihood, or averaged_particle_log_likelihood when replicates is
        given (filter.cpp:141-165)."""
        args, keep = self._ds_args(ds)
        qa = np.ascontiguousarray(q, dtype=np.float64)
        out = C.c_double()
        self.check(self.lib.ref_particle_log_likelihood(
            *args, _ptr(qa), particles, replicates or 0, seed, int(replicates is not None),
            C.byref(out)))
        return out.value

    def enkf(self, ds, p6, members, seed, inflation=1.0, localization=0.0, forecast_steps=0,
             forecast_every=1):
        args, keep = self._ds_args(ds)
        cap = len(np.unique(ds["steps"])) + forecast_steps + 1
        n = ds["n"]
        records = _u64()
        rec = np.zeros((cap, 4))
        means = np.zeros((cap, n, n), np.complex128)
        p = np.ascontiguousarray(p6, dtype=np.float64)
        self.check(self.lib.ref_enkf(*args, _ptr(p), members, seed, inflation, localization,
                                     forecast_steps, forecast_every, cap, C.byref(records),
                                     _ptr(rec), _ptr(means)))
        r = records.value
        return dict(records=rec[:r].copy(), means=means[:r].copy())

    def galerkin(self, n: int, p6, mean, modes, a, dt: float, steps: int):
        """hzl::GalerkinModel: (rhs at a, state after `steps` RK4 steps of dt from a)."""
        p = np.ascontiguousarray(p6, dtype=np.float64)
        m = np.ascontiguousarray(mean, dtype=np.complex128).reshape(-1)
        u = np.ascontiguousarray(modes, dtype=np.complex128).reshape(len(modes), -1)
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, len(u))
        rhs, stepped = np.zeros_like(a), np.zeros_like(a)
        self.check(self.lib.ref_galerkin(n, _ptr(p), len(u), _ptr(m.view(np.float64)),
                                         _ptr(u.view(np.float64)), len(a), _ptr(a), _ptr(rhs),
                                         _ptr(stepped), dt, steps))
        return rhs, stepped

    def fit_pod(self, snapshots: np.ndarray, max_rank: int, fraction: float = 0.9999):
        s = np.ascontiguousarray(snapshots.reshape(len(snapshots), -1), dtype=np.complex128)
        m, dim = s.shape
        mean = np.zeros(dim, np.complex128)
        modes = np.zeros((max_rank, dim), np.complex128)
        sv = np.zeros(max_rank)
        rank = _u64()
        cap = C.c_double()
        self.check(self.lib.ref_fit_pod(m, dim, _ptr(s), max_rank, fraction, C.byref(rank),
                                        _ptr(mean), _ptr(modes), _ptr(sv), C.byref(cap)))
        r = rank.value
        return mean, modes[:r].copy(), sv[:r].copy(), cap.value


class ReferenceSolver:
    def __init__(self, r: Reference, n: int, p6, seed: int):
        self.r, self.n = r, n
        self.h = C.c_void_p()
        p = np.ascontiguousarray(p6, dtype=np.float64)
        r.check(r.lib.ref_solver_create(n, _ptr(p), seed, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.r.lib.ref_solver_destroy(self.h)
            self.h = None

    def _get(self, name):
        a = np.zeros((self.n, self.n), np.complex128)
        self.r.check(getattr(self.r.lib, f"ref_solver_{name}")(self.h, _ptr(a)))
        return a

    def initialize(self, name: str):
        self.r.check(self.r.lib.ref_solver_initialize(self.h, name.encode()))

    def linearized_drift(self, state, direction):
        """Solver::linearized_drift (src/solver.cpp:264-292)."""
        a = np.ascontiguousarray(state, dtype=np.complex128)
        b = np.ascontiguousarray(direction, dtype=np.complex128)
        out = np.zeros((self.n, self.n), np.complex128)
        self.r.check(self.r.lib.ref_solver_linearized_drift(self.h, _ptr(a), _ptr(b), _ptr(out)))
        return out

    def adjoint_drift(self, state, cotangent):
        """Solver::adjoint_drift (src/solver.cpp:293-324)."""
        a = np.ascontiguousarray(state, dtype=np.complex128)
        b = np.ascontiguousarray(cotangent, dtype=np.complex128)
        out = np.zeros((self.n, self.n), np.complex128)
        self.r.check(self.r.lib.ref_solver_adjoint_drift(self.h, _ptr(a), _ptr(b), _ptr(out)))
        return out

    def save(self, path):
        """Solver::save (src/solver.cpp:434-452)."""
        self.r.check(self.r.lib.ref_solver_save(self.h, str(path).encode()))

    def initialize_physical(self, field: np.ndarray):
        a = np.ascontiguousarray(field, dtype=np.complex128)
        self.r.check(self.r.lib.ref_solver_initialize_physical(self.h, _ptr(a)))

    def step(self, dt: float, steps: int = 1):
        self.r.check(self.r.lib.ref_solver_step(self.h, dt, steps))

    def coefficients(self):
        return self._get("coefficients")

    def forcing(self):
        return self._get("forcing")

    def midpoint_forcing(self):
        return self._get("midpoint_forcing")

    def physical_vorticity(self):
        return self._get("physical_vorticity")

    def diagnostics(self) -> np.ndarray:
        d = np.zeros(6)
        self.r.check(self.r.lib.ref_solver_diagnostics(self.h, _ptr(d)))
        return d

    def update_latent_state(self, omega, forcing):
        w = np.ascontiguousarray(omega, dtype=np.complex128)
        f = np.ascontiguousarray(forcing, dtype=np.complex128)
        self.r.check(self.r.lib.ref_solver_update_latent_state(self.h, _ptr(w), _ptr(f)))

    def drift(self, state):
        s = np.ascontiguousarray(state, dtype=np.complex128)
        out = np.zeros_like(s)
        self.r.check(self.r.lib.ref_solver_drift(self.h, _ptr(s), _ptr(out)))
        return out


class ReferenceShellForcing:
    def __init__(self, r: Reference, n: int, p6, seed: int):
        self.r, self.n = r, n
        self.h = C.c_void_p()
        p = np.ascontiguousarray(p6, dtype=np.float64)
        r.check(r.lib.ref_shell_forcing_create(n, _ptr(p), seed, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.r.lib.ref_shell_forcing_destroy(self.h)
            self.h = None

    def midpoint_step(self, dt: float) -> np.ndarray:
        a = np.zeros((self.n, self.n), np.complex128)
        self.r.check(self.r.lib.ref_shell_forcing_midpoint_step(self.h, dt, _ptr(a)))
        return a

    def coefficients(self) -> np.ndarray:
        a = np.zeros((self.n, self.n), np.complex128)
        self.r.check(self.r.lib.ref_shell_forcing_coefficients(self.h, _ptr(a)))
        return a


def reference_available() -> bool:
    return REF_SO.exists()


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_cores() -> int:
    return len(os.sched_getaffinity(0))
