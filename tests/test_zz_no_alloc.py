"""hzlb_step_noalloc, the stepping entry point for callers that may not allocate GPU memory
while they run (their device memory is owned by their own pool, or an allocation on their hot
loop is not acceptable).  It must give the same results as the ordinary entry point
(hzlb_ensemble_create + hzlb_step), on two calls in a row, using only the caller's buffers and
the library's fixed scratch array.  This file is collected last; the test passes both on its
own in a fresh process and after the rest of the suite."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, MEMBERS, DT, NU, SIGMA, SEED = 64, 6, 1e-3, 1e-3, 0.05, 17


def _bind(lib):
    import hzl_stochasticflowinference_b200 as hz
    fn = lib.hzlb_step_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(hz.hzlb_config), C.c_double, C.c_uint64, C.c_uint64, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    return fn


@pytest.mark.parametrize("precision,tol", [(8, 1e-12), (4, 2e-5)])
def test_noalloc_step_matches_ensemble_step(precision, tol):
    import torch
    import hzl_stochasticflowinference_b200 as hz

    lib = hz.library()
    step_noalloc = _bind(lib)
    cfg = hz.Config(n=N, members=MEMBERS, precision=precision, nu=NU, forcing_kmax=0,
                    noise_sigma=SIGMA, noise_kmax=4, seed=SEED)
    # ordinary entry point
    ens = hz.Ensemble(cfg)
    init = np.array([hz.grf_spectrum(N, SEED, m) for m in range(MEMBERS)])
    ens.set_state(init)
    forcing_full = hz.kolmogorov_forcing(N)
    ens.set_forcing(forcing_full[None])
    ens.set_time(0.0, 0)
    dtype = np.complex64 if precision == 4 else np.complex128
    compact0 = hz.full_to_compact(init, N).astype(dtype)
    # caller-owned device buffers (the caller allocates its own inputs and outputs)
    k = (N - 1) // 3
    ld = 2 * k + 1
    forcing_compact = hz.full_to_compact(forcing_full, N)[0].reshape(k + 1, ld)[:1].astype(dtype)
    tdtype = torch.complex64 if precision == 4 else torch.complex128
    state = torch.from_numpy(compact0.copy()).to("cuda", tdtype)
    forcing = torch.from_numpy(forcing_compact.copy()).to("cuda", tdtype)
    stream = torch.cuda.current_stream().cuda_stream
    c = cfg.to_c()
    status = C.c_uint32(0)
    first = 0
    for steps in (3, 2):   # two calls in a row
        ens.step(DT, steps)
        assert ens.status() == 0
        rc = step_noalloc(C.byref(c), DT, steps, first, C.c_void_p(state.data_ptr()),
                          C.c_void_p(forcing.data_ptr()), C.c_void_p(stream), C.byref(status))
        assert rc == 0, lib.hzlb_last_error().decode()
        assert status.value == 0
        first += steps
        torch.cuda.synchronize()
        got = state.cpu().numpy()
        want = ens.get_state_compact()
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= tol, err


def test_noalloc_rejects_sizes_beyond_the_scratch_limit():
    import hzl_stochasticflowinference_b200 as hz

    lib = hz.library()
    step_noalloc = _bind(lib)
    c = hz.Config(n=512, members=4096, precision=8, nu=1e-4).to_c()
    rc = step_noalloc(C.byref(c), 1e-4, 1, 0, C.c_void_p(1), None, None, None)
    assert rc == hz.HZLB_EINVAL
    assert "limit" in lib.hzlb_last_error().decode()
