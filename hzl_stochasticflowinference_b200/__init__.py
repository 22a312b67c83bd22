"""B200 ensemble forecast/analysis path for pvasbob/HZL-stochasticFlowInference.

Python mirror of the reference's interface for this path, over the C ABI of
``include/hzlb.h`` (``libhzlb.so``, built in-tree by ``build.py``).  There is no CPU
fallback: importing this package without the built library, or creating an ensemble without
a CUDA device, raises.

Reference correspondences (paths relative to the reference repository):

* :class:`Ensemble` -- M resident ``hzl::CudaSolver`` instances advanced together
  (include/hzl/cuda_solver.hpp:7-22, src/cuda_solver.cu); state I/O in the reference's
  full-complex layout (include/hzl/fft.hpp:7-9).
* :meth:`Ensemble.diagnostics` -- ``Solver::diagnostics`` per member (src/solver.cpp:381-397).
* :meth:`Ensemble.observe` -- ``Solver::physical_vorticity`` sampled at sensors
  (src/solver.cpp:398-402).
* :meth:`Ensemble.pf_assimilate` (with :meth:`Ensemble.pf_reset`), :meth:`Ensemble.pf_loglik`,
  :meth:`Ensemble.pf_weights`, :meth:`Ensemble.resample`, :meth:`Ensemble.gather` -- the
  weight and resample steps of ``bootstrap_filter`` (src/filter.cpp:65-120), in FP64 on the
  device.
* :meth:`Ensemble.inflate`, :meth:`Ensemble.enkf_analysis` -- the analysis of
  ``ensemble_kalman_filter`` (src/filter.cpp:237-321) in batched form.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libhzlb.so"

HZLB_OK, HZLB_EINVAL, HZLB_ERUNTIME, HZLB_ECUDA, HZLB_ETIMEOUT = 0, -1, -2, -3, -4
STATUS_CFL, STATUS_NONFINITE, STATUS_TIMEOUT = 1, 2, 4

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_fp = C.POINTER(C.c_float)


class hzlb_config(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("members", C.c_int), ("precision", C.c_int),
        ("nu", C.c_double), ("alpha", C.c_double),
        ("forcing_kmax", C.c_int), ("forcing_per_member", C.c_int),
        ("noise_sigma", C.c_double), ("noise_kmax", C.c_int),
        ("seed", C.c_uint64), ("member_base", C.c_uint32), ("device", C.c_int),
    ]


class hzlb_parameters(C.Structure):
    _fields_ = [("viscosity", C.c_double), ("friction", C.c_double),
                ("forcing_sigma", C.c_double), ("forcing_tau", C.c_double),
                ("forcing_min", C.c_int), ("forcing_max", C.c_int)]


class hzlb_pf_record(C.Structure):
    _fields_ = [("increment", C.c_double), ("ess", C.c_double), ("max_weight", C.c_double),
                ("resampled", C.c_int32), ("collapsed", C.c_int32)]


class hzlb_observation(C.Structure):
    _fields_ = [("step", C.c_uint64), ("x", C.c_uint32), ("y", C.c_uint32),
                ("value", C.c_double), ("standard_deviation", C.c_double)]


class hzlb_dataset(C.Structure):
    _fields_ = [("n", C.c_int), ("dt", C.c_double), ("stochastic", C.c_int),
                ("forcing_min", C.c_int), ("forcing_max", C.c_int), ("count", C.c_size_t),
                ("observations", C.POINTER(hzlb_observation))]


class hzlb_filter_record(C.Structure):
    _fields_ = [("step", C.c_uint64), ("log_likelihood_increment", C.c_double),
                ("effective_particles", C.c_double), ("maximum_weight", C.c_double)]


class hzlb_enkf_options(C.Structure):
    _fields_ = [("inflation", C.c_double), ("localization_radius", C.c_double),
                ("forecast_steps", C.c_uint64), ("forecast_every", C.c_uint64)]


class hzlb_enkf_record(C.Structure):
    _fields_ = [("step", C.c_uint64), ("forecast_sensor_rmse", C.c_double),
                ("posterior_spread", C.c_double), ("is_forecast", C.c_int)]


class hzlb_adjoint_evaluation(C.Structure):
    _fields_ = [("value", C.c_double), ("gradient", C.c_double * 2),
                ("checkpoint_fields", C.c_uint64), ("peak_block_fields", C.c_uint64),
                ("replayed_steps", C.c_uint64)]


class HzlbError(RuntimeError):
    """A failure reported through the C ABI (std::runtime_error in the reference)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class HzlbInvalidArgument(HzlbError, ValueError):
    """HZLB_EINVAL (std::invalid_argument in the reference)."""


_lib = None


def library() -> C.CDLL:
    """Loads libhzlb.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run `python {PKG / 'build.py'}` "
                          "(nvcc, sm_100a) before using the B200 path")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "hzlb_last_error": (C.c_char_p, []),
        "hzlb_version": (C.c_char_p, []),
        "hzlb_ensemble_create": (C.c_int, [C.POINTER(hzlb_config), C.POINTER(vp)]),
        "hzlb_ensemble_destroy": (None, [vp]),
        "hzlb_set_state": (C.c_int, [vp, _dp, C.c_int, C.c_int]),
        "hzlb_get_state": (C.c_int, [vp, _dp, C.c_int, C.c_int]),
        "hzlb_set_state_compact": (C.c_int, [vp, vp, C.c_int, C.c_int]),
        "hzlb_get_state_compact": (C.c_int, [vp, vp, C.c_int, C.c_int]),
        "hzlb_compact_size": (C.c_size_t, [vp]),
        "hzlb_set_forcing": (C.c_int, [vp, _dp, C.c_int, C.c_int]),
        "hzlb_step": (C.c_int, [vp, C.c_double, C.c_uint64]),
        "hzlb_step_checked": (C.c_int, [vp, C.c_double]),
        "hzlb_test_inject_wait_timeout": (C.c_int, [vp]),
        "hzlb_step_host": (C.c_int, [vp, vp, vp, C.c_double, C.c_uint64, C.c_int]),
        "hzlb_status": (C.c_int, [vp, _u32p]),
        "hzlb_synchronize": (C.c_int, [vp]),
        "hzlb_stream": (C.c_void_p, [vp]),
        "hzlb_step_profiled": (C.c_int, [vp, C.c_double, C.c_uint64, _dp, _dp]),
        "hzlb_time": (C.c_int, [vp, _dp, C.POINTER(C.c_uint64)]),
        "hzlb_set_time": (C.c_int, [vp, C.c_double, C.c_uint64]),
        "hzlb_diagnostics": (C.c_int, [vp, _dp]),
        "hzlb_physical": (C.c_int, [vp, _dp]),
        "hzlb_observe": (C.c_int, [vp, _u32p, _u32p, C.c_size_t, _dp]),
        "hzlb_pf_loglik": (C.c_int, [vp, _u32p, _u32p, _dp, _dp, C.c_size_t, _dp]),
        "hzlb_pf_weights": (C.c_int, [vp, _dp, C.c_size_t, _dp, _dp, _dp, _dp]),
        "hzlb_pf_reset": (C.c_int, [vp, C.c_int]),
        "hzlb_pf_assimilate": (C.c_int, [vp, _u32p, _u32p, _dp, _dp, C.c_size_t, _dp,
                                         C.POINTER(C.c_uint8), C.POINTER(hzlb_pf_record), _u32p,
                                         _dp]),
        "hzlb_pf_get_weights": (C.c_int, [vp, _dp]),
        "hzlb_enkf_weights": (C.c_int, [vp, vp, _dp, _dp, vp, C.c_int, C.c_size_t, vp, _dp]),
        "hzlb_dgemm": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_longlong,
                                 C.c_longlong, vp, C.c_longlong, C.c_longlong, C.c_double, vp,
                                 C.c_longlong, vp]),
        "hzlb_systematic_resample": (C.c_int, [vp, _dp, C.c_size_t, C.c_double, _u32p]),
        "hzlb_gather_members": (C.c_int, [vp, _u32p]),
        "hzlb_inflate": (C.c_int, [vp, C.c_double]),
        "hzlb_enkf_analysis": (C.c_int, [vp, _u32p, _u32p, _dp, _dp, C.c_size_t, _dp]),
        "hzlb_enkf_analysis_nis": (C.c_int, [vp, _u32p, _u32p, _dp, _dp, C.c_size_t, _dp,
                                             C.c_uint64, C.c_uint64, C.c_double, _dp,
                                             C.POINTER(C.c_int)]),
        "hzlb_state_device": (C.c_int, [vp, C.POINTER(vp)]),
        "hzlb_ensemble_mean": (C.c_int, [vp, _dp]),
        "hzlb_galerkin_create": (C.c_int, [C.c_int, C.POINTER(hzlb_parameters), _dp, _dp,
                                           C.c_size_t, C.c_int, C.POINTER(vp)]),
        "hzlb_galerkin_destroy": (None, [vp]),
        "hzlb_galerkin_coefficients": (C.c_int, [vp, _dp, _dp, _dp]),
        "hzlb_galerkin_rhs": (C.c_int, [vp, _dp, C.c_size_t, _dp]),
        "hzlb_galerkin_step": (C.c_int, [vp, _dp, C.c_size_t, C.c_double, C.c_uint64]),
        "hzlb_enable_ou": (C.c_int, [vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
        "hzlb_get_forcing_compact": (C.c_int, [vp, _dp, C.c_int, C.c_int]),
        "hzlb_weighted_mean": (C.c_int, [vp, _dp, _dp]),
        "hzlb_grf_spectrum": (C.c_int, [C.c_int, C.c_uint64, C.c_uint32, _dp]),
        "hzlb_run_ensemble": (C.c_int, [C.c_int, C.POINTER(hzlb_parameters), C.c_double,
                                        C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_int,
                                        _dp]),
        "hzlb_bootstrap_filter": (C.c_int, [C.POINTER(hzlb_dataset), C.POINTER(hzlb_parameters),
                                            C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                            _dp, C.POINTER(C.c_uint64),
                                            C.POINTER(hzlb_filter_record), C.c_size_t,
                                            C.POINTER(C.c_size_t), _dp]),
        "hzlb_synthetic_observations": (C.c_int, [C.c_int, C.POINTER(hzlb_parameters),
                                                  C.c_double, C.c_uint64, C.c_uint64,
                                                  C.c_double, C.c_uint64, C.c_int, C.c_int,
                                                  C.POINTER(hzlb_dataset),
                                                  C.POINTER(hzlb_observation), C.c_size_t,
                                                  C.POINTER(C.c_size_t), _dp]),
        "hzlb_likelihood_adjoint": (C.c_int, [C.POINTER(hzlb_dataset), _dp, C.c_uint64,
                                              C.c_uint64, C.c_int,
                                              C.POINTER(hzlb_adjoint_evaluation)]),
        "hzlb_linearized_drift": (C.c_int, [C.c_int, C.POINTER(hzlb_parameters), _dp, _dp,
                                            C.c_uint64, C.c_int, _dp]),
        "hzlb_adjoint_drift": (C.c_int, [C.c_int, C.POINTER(hzlb_parameters), _dp, _dp,
                                         C.c_uint64, C.c_int, _dp]),
        "hzlb_solvers_create": (C.c_int, [C.c_int, C.POINTER(hzlb_parameters),
                                          C.POINTER(C.c_uint64), C.c_uint64, C.c_char_p, C.c_int,
                                          C.c_int, C.POINTER(vp)]),
        "hzlb_solvers_load": (C.c_int, [C.POINTER(C.c_char_p), C.c_uint64, C.c_int, C.c_int,
                                        C.POINTER(vp)]),
        "hzlb_solvers_destroy": (None, [vp]),
        "hzlb_solvers_step": (C.c_int, [vp, C.c_double, C.c_uint64]),
        "hzlb_solvers_diagnostics": (C.c_int, [vp, _dp]),
        "hzlb_solvers_coefficients": (C.c_int, [vp, _dp, _dp]),
        "hzlb_solvers_save": (C.c_int, [vp, C.c_uint64, C.c_char_p]),
        "hzlb_solvers_shape": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_uint64)]),
        "hzlb_dataset_save": (C.c_int, [C.POINTER(hzlb_dataset), C.c_char_p]),
        "hzlb_dataset_validate": (C.c_int, [C.POINTER(hzlb_dataset)]),
        "hzlb_dataset_load": (C.c_int, [C.c_char_p, C.POINTER(hzlb_dataset),
                                        C.POINTER(hzlb_observation), C.c_size_t,
                                        C.POINTER(C.c_size_t)]),
        "hzlb_particle_log_likelihood": (C.c_int, [C.POINTER(hzlb_dataset), _dp, C.c_uint64,
                                                   C.c_uint64, C.c_uint64, C.c_int, C.c_int,
                                                   C.c_int, _dp]),
        "hzlb_ensemble_kalman_filter": (C.c_int, [C.POINTER(hzlb_dataset),
                                                  C.POINTER(hzlb_parameters), C.c_uint64,
                                                  C.c_uint64, C.POINTER(hzlb_enkf_options),
                                                  C.c_int, C.c_int, C.POINTER(hzlb_enkf_record),
                                                  C.c_size_t, C.POINTER(C.c_size_t), _dp]),
        "hzlb_kolmogorov_forcing": (C.c_int, [C.c_int, C.c_double, C.c_int, _dp]),
        "hzlb_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                      C.POINTER(vp)]),
        "hzlb_mlp_destroy": (None, [vp]),
        "hzlb_mlp_param_count": (C.c_size_t, [vp]),
        "hzlb_mlp_set_params": (C.c_int, [vp, _fp]),
        "hzlb_mlp_get_params": (C.c_int, [vp, _fp, _fp]),
        "hzlb_mlp_set_scales": (C.c_int, [vp, _fp, _fp]),
        "hzlb_mlp_forward": (C.c_int, [vp, vp, C.c_int, vp, vp]),
        "hzlb_mlp_train_step": (C.c_int, [vp, vp, vp, C.c_int, C.c_float, _dp]),
        "hzlb_mlp_shape": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "hzlb_fit_pod": (C.c_int, [C.c_size_t, C.c_size_t, _dp, C.c_size_t, C.c_double, C.c_int,
                                   C.POINTER(C.c_size_t), _dp, _dp, _dp, _dp]),
        "hzlb_pod_fit": (C.c_int, [C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                   C.c_int, C.POINTER(vp)]),
        "hzlb_pod_destroy": (None, [vp]),
        "hzlb_pod_info": (C.c_int, [vp, C.POINTER(C.c_int), _dp, _dp, _dp]),
        "hzlb_pod_modes": (C.c_int, [vp, _fp, _fp]),
        "hzlb_pod_project": (C.c_int, [vp, vp, C.c_int, vp, C.c_longlong, vp]),
        "hzlb_noise_amplitudes": (C.c_int, [C.POINTER(hzlb_config), C.c_double, C.c_uint64,
                                            C.c_uint64, C.c_int, vp, C.c_longlong, vp]),
        "hzlb_set_step_schedule": (C.c_int, [vp, C.c_int]),
        "hzlb_mixed_row_threads": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "hzlb_mixed_set_row_threads": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "hzlb_step_schedule": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "hzlb_learned_forecast": (C.c_int, [vp, vp, vp, C.c_double, C.c_uint64, vp, C.c_int]),
        "hzlb_ensemble_mean_device": (C.c_int, [vp, vp]),
        "hzlb_mixed_create": (C.c_int, [C.POINTER(hzlb_config), C.c_int, C.POINTER(vp)]),
        "hzlb_mixed_destroy": (None, [vp]),
        "hzlb_mixed_group": (vp, [vp, C.c_int]),
        "hzlb_mixed_step": (C.c_int, [vp, _dp, C.c_uint64]),
        "hzlb_mixed_set_mode": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "hzlb_mixed_mode": (C.c_int, [vp, C.POINTER(C.c_int), _dp]),
        "hzlb_mixed_tune": (C.c_int, [vp, _dp, C.c_int, _dp]),
        "hzlb_mixed_schedule": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int)]),
        "hzlb_mixed_set_schedule": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int),
                                              C.POINTER(C.c_int)]),
        "hzlb_add_window_noise": (C.c_int, [C.POINTER(hzlb_config), C.c_double, C.c_uint64,
                                            C.c_uint64, C.c_int, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc: int):
    if rc != HZLB_OK:
        msg = library().hzlb_last_error().decode()
        if rc == HZLB_EINVAL:
            raise HzlbInvalidArgument(rc, msg)
        raise HzlbError(rc, msg)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _pu(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def retained_k(n: int) -> int:
    """Largest retained |k| under the strict 2/3 rule 3|k| < n (src/solver.cpp:133-134)."""
    return (n - 1) // 3


@dataclass
class Config:
    n: int
    members: int
    precision: int = 4            # 4: FP32 spectra, 8: FP64 spectra
    nu: float = 1e-3
    alpha: float = 0.0
    forcing_kmax: int = -1        # forcing columns kx <= forcing_kmax; -1: none
    forcing_per_member: bool = False
    noise_sigma: float = 0.0
    noise_kmax: int = 4
    seed: int = 42
    member_base: int = 0
    device: int = 0

    def to_c(self) -> hzlb_config:
        return hzlb_config(self.n, self.members, self.precision, self.nu, self.alpha,
                           self.forcing_kmax, int(self.forcing_per_member), self.noise_sigma,
                           self.noise_kmax, self.seed, self.member_base, self.device)


class Ensemble:
    """M members of the periodic 2-D vorticity model advanced together on one B200."""

    def __init__(self, config: Config):
        self.config = config
        self.n, self.members = config.n, config.members
        self._lib = library()
        self._h = C.c_void_p()
        cfg = config.to_c()
        _check(self._lib.hzlb_ensemble_create(C.byref(cfg), C.byref(self._h)))
        self.compact_size = int(self._lib.hzlb_compact_size(self._h))

    @classmethod
    def borrow(cls, handle: int, config: Config, owner) -> "Ensemble":
        """Wraps a handle owned by another object (a mixed batch); never destroys it."""
        e = cls.__new__(cls)
        e.config = config
        e.n, e.members = config.n, config.members
        e._lib = library()
        e._h = C.c_void_p(handle)
        e._borrowed = owner
        e.compact_size = int(e._lib.hzlb_compact_size(e._h))
        return e

    def close(self):
        if getattr(self, "_borrowed", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            self._lib.hzlb_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ------------------------------------------------------------------------
    def set_state(self, spectra: np.ndarray, first: int = 0):
        """spectra: (count, n, n) complex128 in the reference layout [y, x]."""
        s = _c128(spectra).reshape(-1, self.n, self.n)
        _check(self._lib.hzlb_set_state(self._h, s.view(np.float64).ctypes.data_as(_dp), first,
                                        len(s)))

    def get_state(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.members - first if count is None else count
        out = np.zeros((count, self.n, self.n), np.complex128)
        _check(self._lib.hzlb_get_state(self._h, out.view(np.float64).ctypes.data_as(_dp), first,
                                        count))
        return out

    @property
    def compact_dtype(self):
        return np.complex64 if self.config.precision == 4 else np.complex128

    def set_state_compact(self, compact: np.ndarray, first: int = 0):
        a = np.ascontiguousarray(compact, dtype=self.compact_dtype).reshape(-1, self.compact_size)
        _check(self._lib.hzlb_set_state_compact(self._h, a.ctypes.data_as(C.c_void_p), first,
                                                len(a)))
        self._keep = a   # the copy is asynchronous; keep the source alive until the next call

    def get_state_compact(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.members - first if count is None else count
        out = np.zeros((count, self.compact_size), self.compact_dtype)
        _check(self._lib.hzlb_get_state_compact(self._h, out.ctypes.data_as(C.c_void_p), first,
                                                count))
        return out

    def set_state_compact_ptr(self, ptr: int, first: int, count: int):
        """Bulk upload from a raw (device or pinned host) pointer in the compact layout."""
        _check(self._lib.hzlb_set_state_compact(self._h, C.c_void_p(ptr), first, count))

    def get_state_compact_ptr(self, ptr: int, first: int, count: int):
        _check(self._lib.hzlb_get_state_compact(self._h, C.c_void_p(ptr), first, count))

    def step_host_ptr(self, in_ptr: int, out_ptr: int, dt: float, nsteps: int = 1,
                      chunk_members: int = 0):
        """nsteps steps of a host-resident ensemble state (compact layout, all members) read
        from in_ptr and written to out_ptr, copies overlapping the stepping in member chunks
        (hzlb_step_host); pinned host buffers give the overlap."""
        _check(self._lib.hzlb_step_host(self._h, C.c_void_p(in_ptr), C.c_void_p(out_ptr), dt,
                                        nsteps, chunk_members))

    def set_forcing(self, spectra: np.ndarray, first: int = 0):
        s = _c128(spectra).reshape(-1, self.n, self.n)
        _check(self._lib.hzlb_set_forcing(self._h, s.view(np.float64).ctypes.data_as(_dp), first,
                                          len(s)))

    # -- stepping ---------------------------------------------------------------------
    def step(self, dt: float, steps: int = 1):
        _check(self._lib.hzlb_step(self._h, dt, steps))

    def inject_wait_timeout(self):
        """Test hook (hzlb_test_inject_wait_timeout): the next step's row pass leaves one
        block's first tile copy unissued, its bounded wait runs out and the step reports
        STATUS_TIMEOUT."""
        _check(self._lib.hzlb_test_inject_wait_timeout(self._h))

    STEP_SCHEDULES = ("single", "parts", "offset_parts")

    def set_step_schedule(self, schedule) -> None:
        """How step graphs run the members (hzlb_set_step_schedule): "single" (one pass per
        RK stage), "parts" (two member parts on two streams), "offset_parts" (the second part
        one row pass behind); a name or its index."""
        code = self.STEP_SCHEDULES.index(schedule) if isinstance(schedule, str) else int(schedule)
        _check(self._lib.hzlb_set_step_schedule(self._h, code))

    def step_schedule(self) -> str:
        v = C.c_int()
        _check(self._lib.hzlb_step_schedule(self._h, C.byref(v)))
        return self.STEP_SCHEDULES[v.value]

    def step_checked(self, dt: float):
        """One step that is undone when its stage-1 CFL check fails (hzlb_step_checked);
        raises HzlbError (HZLB_ERUNTIME) in that case."""
        _check(self._lib.hzlb_step_checked(self._h, dt))
    def step_profiled(self, dt: float, steps: int):
        """Steps with per-launch CUDA events; returns mean (row_ms, column_ms) per launch."""
        r, c = C.c_double(), C.c_double()
        _check(self._lib.hzlb_step_profiled(self._h, dt, steps, C.byref(r), C.byref(c)))
        return r.value, c.value

    @property
    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self._lib.hzlb_stream(self._h) or 0)

    def status(self) -> int:
        s = C.c_uint32()
        _check(self._lib.hzlb_status(self._h, C.byref(s)))
        return s.value

    def synchronize(self):
        _check(self._lib.hzlb_synchronize(self._h))

    def time(self):
        t, s = C.c_double(), C.c_uint64()
        _check(self._lib.hzlb_time(self._h, C.byref(t), C.byref(s)))
        return t.value, s.value

    def set_time(self, time: float, step_index: int):
        _check(self._lib.hzlb_set_time(self._h, time, step_index))

    # -- diagnostics / observation --------------------------------------------------
    def diagnostics(self) -> np.ndarray:
        """(members, 6): time, energy, enstrophy, dissipation, injection, cfl_rate."""
        out = np.zeros((self.members, 6))
        _check(self._lib.hzlb_diagnostics(self._h, _p(out)))
        return out

    def physical(self) -> np.ndarray:
        out = np.zeros((self.members, self.n, self.n))
        _check(self._lib.hzlb_physical(self._h, _p(out)))
        return out

    def observe(self, x, y) -> np.ndarray:
        x, y = _u32(x), _u32(y)
        out = np.zeros((self.members, len(x)))
        _check(self._lib.hzlb_observe(self._h, _pu(x), _pu(y), len(x), _p(out)))
        return out

    # -- particle filter -------------------------------------------------------------
    def pf_loglik(self, x, y, values, sd, log_weights) -> np.ndarray:
        x, y, v, s = _u32(x), _u32(y), _f64(values), _f64(sd)
        lw = _f64(log_weights).copy()
        _check(self._lib.hzlb_pf_loglik(self._h, _pu(x), _pu(y), _p(v), _p(s), len(x), _p(lw)))
        return lw

    def pf_weights(self, log_weights):
        """(weights, increment, ess, max_weight) of host log-weights (filter.cpp:76-92),
        computed on this ensemble's device."""
        lw = _f64(log_weights)
        w = np.zeros_like(lw)
        inc, ess, mw = C.c_double(), C.c_double(), C.c_double()
        _check(self._lib.hzlb_pf_weights(self._h, _p(lw), len(lw), _p(w), C.byref(inc),
                                         C.byref(ess), C.byref(mw)))
        return w, inc.value, ess.value, mw.value

    def pf_reset(self, particles: int | None = None):
        """members / particles independent filters, device weights reset to 1/particles."""
        particles = self.members if particles is None else int(particles)
        _check(self._lib.hzlb_pf_reset(self._h, particles))
        self._pf_particles = particles

    def pf_assimilate(self, x, y, values, sd, u=None, active=None, weighted_mean: bool = False):
        """One observation time of every segment's bootstrap filter on the device
        (hzlb_pf_assimilate).  u: per-segment uniforms (negative: no resampling) or None.
        Returns dict(increment, ess, max_weight, resampled, collapsed: per-segment arrays,
        ancestors: members, mean: (segments, compact) complex128 when weighted_mean)."""
        x, y, v, s = _u32(x), _u32(y), _f64(values), _f64(sd)
        segments = self.members // self._particles() if u is None and active is None else None
        if u is not None:
            uu = _f64(np.atleast_1d(u))
            segments = len(uu)
        if active is not None:
            act = np.ascontiguousarray(np.asarray(active, np.uint8))
            segments = len(act)
        recs = (hzlb_pf_record * segments)()
        anc = np.zeros(self.members, np.uint32)
        mean = np.zeros((segments, self.compact_size), np.complex128) if weighted_mean else None
        _check(self._lib.hzlb_pf_assimilate(
            self._h, _pu(x), _pu(y), _p(v), _p(s), len(x), None if u is None else _p(uu),
            None if active is None else act.ctypes.data_as(C.POINTER(C.c_uint8)), recs, _pu(anc),
            None if mean is None else mean.view(np.float64).ctypes.data_as(_dp)))
        out = {k: np.array([getattr(r, k) for r in recs])
               for k in ("increment", "ess", "max_weight", "resampled", "collapsed")}
        out["ancestors"] = anc
        if mean is not None:
            out["mean"] = mean
        return out

    def _particles(self) -> int:
        return getattr(self, "_pf_particles", self.members)

    def pf_get_weights(self) -> np.ndarray:
        out = np.zeros(self.members)
        _check(self._lib.hzlb_pf_get_weights(self._h, _p(out)))
        return out

    def resample(self, weights, u: float) -> np.ndarray:
        w = _f64(weights)
        out = np.zeros(len(w), np.uint32)
        _check(self._lib.hzlb_systematic_resample(self._h, _p(w), len(w), u, _pu(out)))
        return out

    def gather(self, ancestors):
        a = _u32(ancestors)
        _check(self._lib.hzlb_gather_members(self._h, _pu(a)))

    # -- EnKF -------------------------------------------------------------------------
    def inflate(self, inflation: float):
        _check(self._lib.hzlb_inflate(self._h, inflation))

    def enkf_analysis(self, x, y, values, sd, perturbations):
        x, y, v, s = _u32(x), _u32(y), _f64(values), _f64(sd)
        e = _f64(perturbations).reshape(self.members, len(x))
        _check(self._lib.hzlb_enkf_analysis(self._h, _pu(x), _pu(y), _p(v), _p(s), len(x),
                                            _p(e)))

    def enkf_analysis_nis(self, x, y, values, sd, perturbations=None, seed: int = 0,
                          cycle: int = 0, nis_limit: float = 0.0):
        """Analysis with the normalised innovation statistic; returns (nis, applied).
        perturbations None: drawn on the device from Philox (seed, member, cycle)."""
        x, y, v, s = _u32(x), _u32(y), _f64(values), _f64(sd)
        e = None if perturbations is None else _f64(perturbations).reshape(self.members, len(x))
        nis, applied = C.c_double(), C.c_int()
        _check(self._lib.hzlb_enkf_analysis_nis(self._h, _pu(x), _pu(y), _p(v), _p(s), len(x),
                                                None if e is None else _p(e), seed, cycle,
                                                nis_limit, C.byref(nis), C.byref(applied)))
        return nis.value, bool(applied.value)

    def enkf_weights(self, hx, values, sd, eps):
        """Ensemble-space EnKF weights of gathered predicted observations (hzlb_enkf_weights):
        hx, eps CUDA float64 tensors (members, p); returns (W as a CUDA float64 tensor
        (members, members), innovation statistic)."""
        import torch
        hx = hx.contiguous().to(torch.float64)
        eps = eps.contiguous().to(torch.float64)
        members, p = hx.shape
        w = torch.empty((members, members), dtype=torch.float64, device=hx.device)
        v, s = _f64(values), _f64(sd)
        nis = C.c_double()
        torch.cuda.current_stream(hx.device).synchronize()   # hx and eps are written
        _check(self._lib.hzlb_enkf_weights(self._h, C.c_void_p(hx.data_ptr()), _p(v), _p(s),
                                           C.c_void_p(eps.data_ptr()), members, p,
                                           C.c_void_p(w.data_ptr()), C.byref(nis)))
        return w, nis.value

    def learned_forecast(self, pod: "Pod", mlp: "Mlp", dt: float, steps: int,
                         mean_increment=None, centre: bool = True) -> None:
        """One window of the learned reduced forecast (hzlb_learned_forecast);
        mean_increment: optional CUDA float32 tensor (compact field) added to every member;
        centre: the network then moves the members only about their mean (the increment is the
        mean's change), else its changes are kept whole (the increment carries the rest)."""
        ptr = None
        if mean_increment is not None:
            _torch_ready()
            ptr = C.c_void_p(mean_increment.data_ptr())
        _check(self._lib.hzlb_learned_forecast(self._h, pod._h, mlp._h, dt, steps, ptr,
                                               1 if centre else 0))

    def mean_device(self, out) -> None:
        """Member mean of the compact state into out (CUDA tensor of the state's precision)."""
        _check(self._lib.hzlb_ensemble_mean_device(self._h, C.c_void_p(out.data_ptr())))

    def enable_ou(self, sigma: float, tau: float, kmin: int, kmax: int, initialize: bool = True):
        """Device OU shell forcing (hzlb_enable_ou)."""
        _check(self._lib.hzlb_enable_ou(self._h, sigma, tau, kmin, kmax, int(initialize)))

    def forcing_compact(self, first: int = 0, count: int | None = None) -> np.ndarray:
        """Per-member forcing, compact forcing layout, complex128 [count][cols * (2K+1)]."""
        count = self.members - first if count is None else count
        k = retained_k(self.n)
        cols = min(self.config.forcing_kmax + 1, k + 1)
        out = np.zeros((count, cols * (2 * k + 1)), np.complex128)
        _check(self._lib.hzlb_get_forcing_compact(self._h, out.view(np.float64).ctypes.data_as(_dp),
                                                  first, count))
        return out

    def weighted_mean_compact(self, weights) -> np.ndarray:
        """sum_m w[m] x_m, compact layout, complex128."""
        w = _f64(weights)
        out = np.zeros(self.compact_size, np.complex128)
        _check(self._lib.hzlb_weighted_mean(self._h, _p(w), out.view(np.float64).ctypes.data_as(_dp)))
        return out

    def mean_compact(self) -> np.ndarray:
        """Ensemble mean, compact layout, complex128."""
        out = np.zeros(self.compact_size, np.complex128)
        _check(self._lib.hzlb_ensemble_mean(self._h, out.view(np.float64).ctypes.data_as(_dp)))
        return out

    def state_device(self) -> int:
        """Device address of the compact state (see hzlb_state_device)."""
        ptr = C.c_void_p()
        _check(self._lib.hzlb_state_device(self._h, C.byref(ptr)))
        return ptr.value


def dgemm(a, b, c, alpha: float = 1.0, beta: float = 0.0, a_trans: bool = False,
          b_trans: bool = False) -> None:
    """c = alpha op(a) op(b) + beta c on the FP64 tensor cores (hzlb_dgemm), for contiguous
    CUDA float64 matrices; op(x) = x.T when the flag is set.  Runs on torch's current stream."""
    import torch
    for t in (a, b, c):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.dim() != 2:
            raise HzlbInvalidArgument(HZLB_EINVAL, "dgemm takes contiguous CUDA float64 matrices")
    m, k = (a.shape[1], a.shape[0]) if a_trans else (a.shape[0], a.shape[1])
    kb, n = (b.shape[1], b.shape[0]) if b_trans else (b.shape[0], b.shape[1])
    if kb != k or tuple(c.shape) != (m, n):
        raise HzlbInvalidArgument(HZLB_EINVAL, "dgemm shape mismatch")
    sam, sak = (1, a.shape[1]) if a_trans else (a.shape[1], 1)
    sbk, sbn = (1, b.shape[1]) if b_trans else (b.shape[1], 1)
    stream = torch.cuda.current_stream(c.device).cuda_stream
    _check(library().hzlb_dgemm(m, n, k, alpha, C.c_void_p(a.data_ptr()), sam, sak,
                                C.c_void_p(b.data_ptr()), sbk, sbn, beta, C.c_void_p(c.data_ptr()),
                                n, C.c_void_p(stream)))


def grf_spectrum(n: int, seed: int, member: int) -> np.ndarray:
    out = np.zeros((n, n), np.complex128)
    _check(library().hzlb_grf_spectrum(n, seed, member, out.view(np.float64).ctypes.data_as(_dp)))
    return out


def kolmogorov_forcing(n: int, amplitude: float = 0.1, wavenumber: int = 4) -> np.ndarray:
    out = np.zeros((n, n), np.complex128)
    _check(library().hzlb_kolmogorov_forcing(n, amplitude, wavenumber,
                                             out.view(np.float64).ctypes.data_as(_dp)))
    return out


def compact_to_full(compact: np.ndarray, n: int) -> np.ndarray:
    """Compact half-spectrum layout -> reference full-complex layout (Hermitian fill)."""
    k = retained_k(n)
    ld = 2 * k + 1
    c = np.asarray(compact).reshape(-1, k + 1, ld).astype(np.complex128)
    j = np.arange(ld)
    ypos = np.where(j <= k, j, n - ld + j)
    full = np.zeros((len(c), n, n), np.complex128)
    full[:, ypos[:, None], np.arange(k + 1)[None, :]] = c.transpose(0, 2, 1)
    kx = np.arange(1, k + 1)
    full[:, ((n - ypos) % n)[:, None], (n - kx)[None, :]] = np.conj(c[:, 1:, :]).transpose(0, 2, 1)
    return full


def full_to_compact(full: np.ndarray, n: int) -> np.ndarray:
    k = retained_k(n)
    ld = 2 * k + 1
    j = np.arange(ld)
    ypos = np.where(j <= k, j, n - ld + j)
    f = np.asarray(full).reshape(-1, n, n)
    out = f[:, ypos][:, :, : k + 1].transpose(0, 2, 1).copy()
    out[:, 0, 0] = 0
    return out.reshape(len(f), -1)


# ---- drop-ins for the reference's ensemble entry points ------------------------------------
@dataclass
class Parameters:
    """hzl::Parameters (include/hzl/solver.hpp:15-23) with the reference defaults."""
    viscosity: float = 0.01
    friction: float = 0.1
    forcing_sigma: float = 0.2
    forcing_tau: float = 0.5
    forcing_min: int = 2
    forcing_max: int = 3

    def to_c(self) -> hzlb_parameters:
        return hzlb_parameters(self.viscosity, self.friction, self.forcing_sigma,
                               self.forcing_tau, self.forcing_min, self.forcing_max)


def _dataset_c(ds: dict):
    count = len(ds["steps"])
    obs = (hzlb_observation * count)()
    for i in range(count):
        obs[i] = hzlb_observation(int(ds["steps"][i]), int(ds["x"][i]), int(ds["y"][i]),
                                  float(ds["value"][i]), float(ds["sd"][i]))
    c = hzlb_dataset(ds["n"], ds["dt"], int(ds.get("stochastic", 1)), ds["forcing_min"],
                     ds["forcing_max"], count, obs)
    return c, obs


def ensemble(n: int, p: Parameters, dt: float, steps: int, count: int, seed: int,
             precision: int = 8, device: int = 0) -> np.ndarray:
    """hzl::ensemble (src/inference.cpp:555-590): (count, 6) diagnostics in member order."""
    out = np.zeros((count, 6))
    pc = p.to_c()
    _check(library().hzlb_run_ensemble(n, C.byref(pc), dt, steps, count, seed, precision,
                                       device, _p(out)))
    return out


def bootstrap_filter(ds: dict, p: Parameters, particles: int, seed: int,
                     retain_states: bool = True, precision: int = 8, device: int = 0) -> dict:
    """hzl::bootstrap_filter (src/filter.cpp:38-126)."""
    dc, keep = _dataset_c(ds)
    cap = len(np.unique(ds["steps"])) + 1
    recs = (hzlb_filter_record * cap)()
    means = np.zeros((cap, ds["n"], ds["n"]), np.complex128)
    ll, ev, nrec = C.c_double(), C.c_uint64(), C.c_size_t()
    pc = p.to_c()
    _check(library().hzlb_bootstrap_filter(
        C.byref(dc), C.byref(pc), particles, seed, int(retain_states), precision, device,
        C.byref(ll), C.byref(ev), recs, cap, C.byref(nrec),
        means.view(np.float64).ctypes.data_as(_dp) if retain_states else None))
    k = nrec.value
    rec = np.array([[recs[i].step, recs[i].log_likelihood_increment,
                     recs[i].effective_particles, recs[i].maximum_weight] for i in range(k)])
    return dict(log_likelihood=ll.value, resampling_events=ev.value, records=rec.reshape(-1, 4),
                means=means[:k].copy())


def synthetic_observations(n: int, truth: Parameters, dt: float, steps: int, every: int,
                           noise: float, seed: int, precision: int = 8, device: int = 0,
                           truth_fields: bool = False):
    """hzl::synthetic_observations (src/inference.cpp:258-288) with the truth run on the
    device: the dataset dict the drivers take, and with truth_fields the (steps // every, n, n)
    physical vorticity at the observation times as a second value."""
    lib = library()
    pc = truth.to_c()
    header, count = hzlb_dataset(), C.c_size_t()
    _check(lib.hzlb_synthetic_observations(n, C.byref(pc), dt, steps, every, noise, seed,
                                           precision, device, C.byref(header), None, 0,
                                           C.byref(count), None))
    k = count.value
    obs = (hzlb_observation * max(k, 1))()
    fields = np.zeros((k // 8, n, n)) if truth_fields else None
    _check(lib.hzlb_synthetic_observations(
        n, C.byref(pc), dt, steps, every, noise, seed, precision, device, C.byref(header), obs,
        k, C.byref(count), _p(fields) if truth_fields else None))
    ds = dict(n=header.n, dt=header.dt, stochastic=header.stochastic,
              forcing_min=header.forcing_min, forcing_max=header.forcing_max,
              steps=np.array([obs[i].step for i in range(k)], np.uint64),
              x=np.array([obs[i].x for i in range(k)], np.uint32),
              y=np.array([obs[i].y for i in range(k)], np.uint32),
              value=np.array([obs[i].value for i in range(k)]),
              sd=np.array([obs[i].standard_deviation for i in range(k)]))
    return (ds, fields) if truth_fields else ds


def likelihood_adjoint(ds: dict, log_parameters, checkpoint_stride: int = 20,
                       device: int = 0) -> list[dict]:
    """hzl::likelihood_adjoint (src/adjoint.cpp:43-161) for one or many (log nu, log alpha)
    vectors at once: objective value, gradient and the checkpoint counters of each."""
    q = np.ascontiguousarray(log_parameters, dtype=np.float64).reshape(-1, 2)
    dc, keep = _dataset_c(ds)
    out = (hzlb_adjoint_evaluation * max(len(q), 1))()
    _check(library().hzlb_likelihood_adjoint(C.byref(dc), _p(q), len(q), checkpoint_stride,
                                             device, out))
    return [dict(value=out[i].value, gradient=np.array(out[i].gradient[:]),
                 checkpoint_fields=out[i].checkpoint_fields,
                 peak_block_fields=out[i].peak_block_fields,
                 replayed_steps=out[i].replayed_steps) for i in range(len(q))]


def _drift_pairs(fn, n, p, states, second, device):
    a = np.ascontiguousarray(states, dtype=np.complex128).reshape(-1, n, n)
    b = np.ascontiguousarray(second, dtype=np.complex128).reshape(-1, n, n)
    if a.shape != b.shape:
        raise HzlbInvalidArgument(HZLB_EINVAL, "drift state size mismatch")
    out = np.zeros_like(a)
    pc = p.to_c()
    _check(fn(n, C.byref(pc), a.view(np.float64).ctypes.data_as(_dp),
              b.view(np.float64).ctypes.data_as(_dp), a.shape[0], device,
              out.view(np.float64).ctypes.data_as(_dp)))
    return out


def linearized_drift(n: int, p: Parameters, states, directions, device: int = 0) -> np.ndarray:
    """hzl::Solver::linearized_drift (src/solver.cpp:264-292) for a batch of (state,
    direction) pairs, (count, n, n) complex spectra each."""
    return _drift_pairs(library().hzlb_linearized_drift, n, p, states, directions, device)


def adjoint_drift(n: int, p: Parameters, states, cotangents, device: int = 0) -> np.ndarray:
    """hzl::Solver::adjoint_drift (src/solver.cpp:293-324) for a batch of (state, cotangent)
    pairs, (count, n, n) complex spectra each."""
    return _drift_pairs(library().hzlb_adjoint_drift, n, p, states, cotangents, device)


class Solvers:
    """A set of hzl::Solver instances (src/solver.cpp:120-254) advanced together on the device,
    each savable as an HZL_CHECKPOINT_V1 file (Solver::save / Solver::load,
    src/solver.cpp:434-491).  Solver i is Solver(n, p, seeds[i]) initialised with `initial`;
    Solvers.load restores a set from checkpoint files written by either library."""

    def __init__(self, n: int, p: Parameters, seeds, initial: str = "multimode",
                 precision: int = 8, device: int = 0):
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        self._h = C.c_void_p()
        pc = p.to_c()
        _check(library().hzlb_solvers_create(n, C.byref(pc),
                                             seeds.ctypes.data_as(C.POINTER(C.c_uint64)),
                                             len(seeds), initial.encode(), precision, device,
                                             C.byref(self._h)))
        self.n, self.count = n, len(seeds)

    @classmethod
    def load(cls, paths, precision: int = 8, device: int = 0) -> "Solvers":
        arr = (C.c_char_p * len(paths))(*[str(p).encode() for p in paths])
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        _check(library().hzlb_solvers_load(arr, len(paths), precision, device, C.byref(self._h)))
        n, count = C.c_int(), C.c_uint64()
        _check(library().hzlb_solvers_shape(self._h, C.byref(n), C.byref(count)))
        self.n, self.count = n.value, count.value
        return self

    def step(self, dt: float, steps: int = 1) -> None:
        _check(library().hzlb_solvers_step(self._h, dt, steps))

    def diagnostics(self) -> np.ndarray:
        out = np.zeros((self.count, 6))
        _check(library().hzlb_solvers_diagnostics(self._h, _p(out)))
        return out

    def coefficients(self):
        """(omega, latent forcing), each (count, n, n) complex over the whole spectrum."""
        w = np.zeros((self.count, self.n, self.n), np.complex128)
        f = np.zeros_like(w)
        _check(library().hzlb_solvers_coefficients(self._h, w.view(np.float64).ctypes.data_as(_dp),
                                                   f.view(np.float64).ctypes.data_as(_dp)))
        return w, f

    def save(self, member: int, path) -> None:
        _check(library().hzlb_solvers_save(self._h, member, str(path).encode()))

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().hzlb_solvers_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def save_dataset(ds: dict, path) -> None:
    """hzl::Dataset::save (src/inference.cpp:214-226): HZL_OBSERVATIONS_V2 text."""
    dc, keep = _dataset_c(ds)
    _check(library().hzlb_dataset_save(C.byref(dc), str(path).encode()))


def validate_dataset(ds: dict) -> None:
    """hzl::Dataset::validate (src/inference.cpp:197-213)."""
    dc, keep = _dataset_c(ds)
    _check(library().hzlb_dataset_validate(C.byref(dc)))


def load_dataset(path) -> dict:
    """hzl::Dataset::load (src/inference.cpp:227-257): V1 or V2 files, as the dataset dict the
    drivers take (n, dt, stochastic, forcing_min, forcing_max, steps, x, y, value, sd)."""
    lib = library()
    header, count = hzlb_dataset(), C.c_size_t()
    _check(lib.hzlb_dataset_load(str(path).encode(), C.byref(header), None, 0, C.byref(count)))
    obs = (hzlb_observation * max(count.value, 1))()
    _check(lib.hzlb_dataset_load(str(path).encode(), C.byref(header), obs, count.value,
                                 C.byref(count)))
    k = count.value
    return dict(n=header.n, dt=header.dt, stochastic=header.stochastic,
                forcing_min=header.forcing_min, forcing_max=header.forcing_max,
                steps=np.array([obs[i].step for i in range(k)], np.uint64),
                x=np.array([obs[i].x for i in range(k)], np.uint32),
                y=np.array([obs[i].y for i in range(k)], np.uint32),
                value=np.array([obs[i].value for i in range(k)]),
                sd=np.array([obs[i].standard_deviation for i in range(k)]))


def particle_log_likelihood(ds: dict, log_parameters, particles: int, seed: int,
                            precision: int = 8, device: int = 0) -> float:
    """hzl::particle_log_likelihood (src/filter.cpp:141-149)."""
    return _particle_ll(ds, log_parameters, particles, 0, seed, 0, precision, device)


def averaged_particle_log_likelihood(ds: dict, log_parameters, particles: int, replicates: int,
                                     seed: int, precision: int = 8, device: int = 0) -> float:
    """hzl::averaged_particle_log_likelihood (src/filter.cpp:150-165): all replicates advance
    as one batched ensemble of replicates x particles members."""
    return _particle_ll(ds, log_parameters, particles, replicates, seed, 1, precision, device)


def _particle_ll(ds, log_parameters, particles, replicates, seed, averaged, precision, device):
    q = np.ascontiguousarray(log_parameters, dtype=np.float64)
    if q.shape != (4,):
        raise HzlbInvalidArgument(HZLB_EINVAL, "stochastic inference expects log(nu), "
                                  "log(alpha), log(sigma), log(tau)")
    dc, keep = _dataset_c(ds)
    out = C.c_double()
    _check(library().hzlb_particle_log_likelihood(C.byref(dc), _p(q), particles, replicates,
                                                  seed, averaged, precision, device,
                                                  C.byref(out)))
    return out.value


def ensemble_kalman_filter(ds: dict, p: Parameters, members: int, seed: int,
                           inflation: float = 1.0, localization_radius: float = 0.0,
                           forecast_steps: int = 0, forecast_every: int = 1,
                           precision: int = 8, device: int = 0) -> dict:
    """hzl::ensemble_kalman_filter (src/filter.cpp:204-356)."""
    dc, keep = _dataset_c(ds)
    cap = len(np.unique(ds["steps"])) + forecast_steps + 1
    recs = (hzlb_enkf_record * cap)()
    means = np.zeros((cap, ds["n"], ds["n"]), np.complex128)
    nrec = C.c_size_t()
    pc = p.to_c()
    opt = hzlb_enkf_options(inflation, localization_radius, forecast_steps, forecast_every)
    _check(library().hzlb_ensemble_kalman_filter(
        C.byref(dc), C.byref(pc), members, seed, C.byref(opt), precision, device, recs, cap,
        C.byref(nrec), means.view(np.float64).ctypes.data_as(_dp)))
    k = nrec.value
    rec = np.array([[recs[i].step, recs[i].forecast_sensor_rmse, recs[i].posterior_spread,
                     recs[i].is_forecast] for i in range(k)])
    return dict(records=rec.reshape(-1, 4), means=means[:k].copy())


def _torch_ready():
    """The library runs on its own non-blocking streams: wait for torch's pending work on the
    tensors passed in before handing them over."""
    import torch
    torch.cuda.current_stream().synchronize()


class Mlp:
    """Learned reduced forecast network (hzlb_mlp_*): r POD coefficients plus q noise-mode
    amplitudes -> r coefficients one window later, BF16 on the tcgen05 tensor cores.  Batches
    are CUDA tensors (torch) of FP32, row-major [batch][features]."""

    def __init__(self, r: int, q: int, hidden: int, max_batch: int, seed: int = 0,
                 device: int = 0):
        self._lib = library()
        self._h = C.c_void_p()
        _check(self._lib.hzlb_mlp_create(r, q, hidden, max_batch, device, seed,
                                         C.byref(self._h)))
        self.r, self.q, self.hidden, self.max_batch = r, q, hidden, max_batch
        self.count = int(self._lib.hzlb_mlp_param_count(self._h))

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.hzlb_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def layout(self) -> dict:
        """Offsets and shapes of W1, W2, W3, b1, b2, b3 in the parameter vector."""
        i, h, r = self.r + self.q, self.hidden, self.r
        shapes = [("W1", (h, i)), ("W2", (h, h)), ("W3", (r, h)), ("b1", (h,)), ("b2", (h,)),
                  ("b3", (r,))]
        out, off = {}, 0
        for name, shp in shapes:
            size = int(np.prod(shp))
            out[name] = (off, shp)
            off += size
        return out

    def unpack(self, flat: np.ndarray) -> dict:
        return {k: flat[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in self.layout().items()}

    def pack(self, parts: dict) -> np.ndarray:
        flat = np.zeros(self.count, np.float32)
        for k, (o, s) in self.layout().items():
            flat[o:o + int(np.prod(s))] = np.asarray(parts[k], np.float32).ravel()
        return flat

    def set_params(self, flat) -> None:
        a = np.ascontiguousarray(flat, np.float32)
        if a.size != self.count:
            raise ValueError(f"expected {self.count} parameters")
        _check(self._lib.hzlb_mlp_set_params(self._h, a.ctypes.data_as(_fp)))

    def params(self, grads: bool = False):
        p = np.zeros(self.count, np.float32)
        g = np.zeros(self.count, np.float32) if grads else None
        _check(self._lib.hzlb_mlp_get_params(self._h, p.ctypes.data_as(_fp),
                                             g.ctypes.data_as(_fp) if grads else None))
        return (p, g) if grads else p

    def set_scales(self, s_in, s_out) -> None:
        a = np.ascontiguousarray(s_in, np.float32)
        b = np.ascontiguousarray(s_out, np.float32)
        if a.size != self.r + self.q or b.size != self.r:
            raise ValueError("scale sizes must be r+q and r")
        _check(self._lib.hzlb_mlp_set_scales(self._h, a.ctypes.data_as(_fp), b.ctypes.data_as(_fp)))

    @staticmethod
    def _dev(t, cols: int):
        if not (t.is_cuda and t.dtype.is_floating_point and t.element_size() == 4 and
                t.is_contiguous() and t.dim() == 2 and t.shape[1] == cols):
            raise ValueError(f"expected a contiguous CUDA float32 [batch][{cols}] tensor")
        return C.c_void_p(t.data_ptr())

    def forward(self, x, out=None):
        import torch
        if out is None:
            out = torch.empty((x.shape[0], self.r), dtype=torch.float32, device=x.device)
        _torch_ready()
        _check(self._lib.hzlb_mlp_forward(self._h, self._dev(x, self.r + self.q), x.shape[0],
                                          self._dev(out, self.r), None))
        return out

    def train_step(self, x, target, lr: float) -> float:
        loss = C.c_double()
        _torch_ready()
        _check(self._lib.hzlb_mlp_train_step(self._h, self._dev(x, self.r + self.q),
                                             self._dev(target, self.r), x.shape[0], lr,
                                             C.byref(loss)))
        return loss.value


def fit_pod(snapshots, max_rank: int, fraction: float = 0.9999, device: int = 0) -> dict:
    """hzl::fit_pod (src/reduced.cpp:36-136) on the GPU: snapshots (m, ...) complex."""
    x = _c128(snapshots)
    m = x.shape[0]
    dim = x[0].size
    mean = np.zeros(dim, np.complex128)
    modes = np.zeros((max_rank, dim), np.complex128)
    sv = np.zeros(max_rank)
    rank, cap = C.c_size_t(), C.c_double()
    _check(library().hzlb_fit_pod(m, dim, x.view(np.float64).ctypes.data_as(_dp), max_rank,
                                  fraction, device, C.byref(rank), mean.view(np.float64).ctypes.data_as(_dp),
                                  modes.view(np.float64).ctypes.data_as(_dp), _p(sv), C.byref(cap)))
    r = rank.value
    shape = x.shape[1:]
    return dict(mean=mean.reshape(shape), modes=modes[:r].reshape((r,) + shape),
                singular_values=sv[:r].copy(), captured=cap.value)


class Pod:
    """POD basis of compact FP32 ensemble snapshots on the device (hzlb_pod_*)."""

    def __init__(self, n: int, snapshots, rank: int, oversample: int = 32, iterations: int = 60,
                 seed: int = 0, device: int = 0):
        self._lib = library()
        self._h = C.c_void_p()
        t = snapshots
        if not (t.is_cuda and t.is_contiguous() and t.dtype.is_floating_point and
                t.element_size() == 4 and t.dim() == 2):
            raise ValueError("snapshots: contiguous CUDA float32 [count][2 * compact] tensor")
        _torch_ready()
        _check(self._lib.hzlb_pod_fit(n, t.shape[0], C.c_void_p(t.data_ptr()), rank, oversample,
                                      iterations, seed, device, C.byref(self._h)))
        self.n, self.rank = n, rank

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.hzlb_pod_destroy(self._h)
            self._h = C.c_void_p()

    def info(self) -> dict:
        r = C.c_int()
        ev = np.zeros(self.rank)
        cap, res = C.c_double(), C.c_double()
        _check(self._lib.hzlb_pod_info(self._h, C.byref(r), _p(ev), C.byref(cap), C.byref(res)))
        return dict(rank=r.value, eigenvalues=ev, captured=cap.value, residual=res.value)

    def modes(self):
        k = retained_k(self.n)
        size = (k + 1) * (2 * k + 1)
        modes = np.zeros((self.rank, 2 * size), np.float32)
        mean = np.zeros(2 * size, np.float32)
        _check(self._lib.hzlb_pod_modes(self._h, modes.ctypes.data_as(_fp), mean.ctypes.data_as(_fp)))
        return modes, mean

    def project(self, states, out=None):
        import torch
        if out is None:
            out = torch.empty((states.shape[0], self.rank), dtype=torch.float32, device=states.device)
        return self.project_ptr(states.data_ptr(), states.shape[0], out)

    def project_ptr(self, ptr: int, count: int, out):
        """Projections of `count` compact FP32 states at device address ptr into out (CUDA
        float32, rows of stride out.stride(0))."""
        if out.shape[0] != count or out.shape[1] < self.rank or out.stride(1) != 1:
            raise ValueError("out must be [count][>= rank] with unit column stride")
        _torch_ready()
        _check(self._lib.hzlb_pod_project(self._h, C.c_void_p(ptr), count,
                                          C.c_void_p(out.data_ptr()), out.stride(0), None))
        return out


def noise_amplitudes(config: Config, dt: float, first_step: int, steps: int, count: int, out):
    """Noise-mode amplitudes of a forecast window into out[count][>= 8] (CUDA float32)."""
    cfg = config.to_c()
    _torch_ready()
    _check(library().hzlb_noise_amplitudes(C.byref(cfg), dt, first_step, steps, count,
                                           C.c_void_p(out.data_ptr()), out.stride(0), None))
    return out


def add_window_noise(config: Config, dt: float, first_step: int, steps: int, count: int,
                     ptr: int) -> None:
    """Adds a window's noise increments to `count` compact FP32 states at device address ptr."""
    cfg = config.to_c()
    _torch_ready()
    _check(library().hzlb_add_window_noise(C.byref(cfg), dt, first_step, steps, count,
                                           C.c_void_p(ptr), None))


class Mixed:
    """Mixed-resolution ensembles advanced by one graph per batch of steps (hzlb_mixed_*)."""

    def __init__(self, configs: list):
        self._lib = library()
        arr = (hzlb_config * len(configs))(*[c.to_c() for c in configs])
        self._h = C.c_void_p()
        _check(self._lib.hzlb_mixed_create(arr, len(configs), C.byref(self._h)))
        self.configs = list(configs)
        self.groups = [Ensemble.borrow(self._lib.hzlb_mixed_group(self._h, g), c, self)
                       for g, c in enumerate(configs)]

    def close(self):
        for g in getattr(self, "groups", []):
            g.close()
        if getattr(self, "_h", None) and self._h.value:
            self._lib.hzlb_mixed_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def step(self, dts, steps: int) -> None:
        d = _f64(dts)
        _check(self._lib.hzlb_mixed_step(self._h, _p(d), steps))

    def tune(self, dts, repeats: int = 2) -> float:
        d = _f64(dts)
        ms = C.c_double()
        _check(self._lib.hzlb_mixed_tune(self._h, _p(d), repeats, C.byref(ms)))
        return ms.value

    MODES = ("serial", "concurrent", "fused", "fused_branch")

    def schedule(self) -> dict:
        k = len(self.configs)
        serial = C.c_int()
        col, row = (C.c_int * k)(), (C.c_int * k)()
        _check(self._lib.hzlb_mixed_schedule(self._h, C.byref(serial), col, row))
        mode = C.c_int()
        tried = (C.c_double * 4)()
        _check(self._lib.hzlb_mixed_mode(self._h, C.byref(mode), tried))
        threads = (C.c_int * k)()
        _check(self._lib.hzlb_mixed_row_threads(self._h, threads))
        return dict(serial=bool(serial.value), mode=self.MODES[mode.value],
                    column_caps=list(col), row_caps=list(row), row_threads=list(threads),
                    tuned_ms={m: t for m, t in zip(self.MODES, tried) if t > 0})

    def set_row_threads(self, threads) -> None:
        """Row-kernel block shape per group, 64 or 128 threads (0: the resolution's default;
        hzlb_mixed_set_row_threads)."""
        arr = (C.c_int * len(self.configs))(*threads)
        _check(self._lib.hzlb_mixed_set_row_threads(self._h, arr))

    def set_mode(self, mode: str, column_caps=None, row_caps=None) -> None:
        """One of MODES (hzlb_mixed_set_mode); caps per group as in set_schedule."""
        k = len(self.configs)
        col = (C.c_int * k)(*column_caps) if column_caps is not None else None
        row = (C.c_int * k)(*row_caps) if row_caps is not None else None
        _check(self._lib.hzlb_mixed_set_mode(self._h, self.MODES.index(mode), col, row))

    def set_schedule(self, serial: bool, column_caps=None, row_caps=None) -> None:
        k = len(self.configs)
        col = (C.c_int * k)(*column_caps) if column_caps is not None else None
        row = (C.c_int * k)(*row_caps) if row_caps is not None else None
        _check(self._lib.hzlb_mixed_set_schedule(self._h, int(serial), col, row))


class GalerkinModel:
    """hzl::GalerkinModel (src/reduced.cpp:137-209) with its drifts evaluated on the GPU."""

    def __init__(self, n: int, p: "Parameters", mean, modes, device: int = 0):
        self._lib = library()
        m = _c128(mean).reshape(n * n)
        u = _c128(modes).reshape(-1, n * n)
        self.rank = len(u)
        self._h = C.c_void_p()
        pc = p.to_c()
        _check(self._lib.hzlb_galerkin_create(n, C.byref(pc), m.view(np.float64).ctypes.data_as(_dp),
                                              u.view(np.float64).ctypes.data_as(_dp), self.rank,
                                              device, C.byref(self._h)))

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.hzlb_galerkin_destroy(self._h)
            self._h = C.c_void_p()

    def coefficients(self):
        r = self.rank
        c, A, Q = np.zeros(r), np.zeros((r, r)), np.zeros((r, r, r))
        _check(self._lib.hzlb_galerkin_coefficients(self._h, _p(c), _p(A), _p(Q)))
        return c, A, Q

    def rhs(self, a) -> np.ndarray:
        a = _f64(a).reshape(-1, self.rank)
        out = np.zeros_like(a)
        _check(self._lib.hzlb_galerkin_rhs(self._h, _p(a), len(a), _p(out)))
        return out

    def step(self, a, dt: float, steps: int = 1) -> np.ndarray:
        a = _f64(a).reshape(-1, self.rank).copy()
        _check(self._lib.hzlb_galerkin_step(self._h, _p(a), len(a), dt, steps))
        return a
