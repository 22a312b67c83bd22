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


def _capacity(n: int, precision: int, limit: int = 32 << 20) -> int:
    """Largest member count whose scratch fits the array: the layout the entry point documents
    (twiddle region, control word, then state copy, stage input and accumulator with 16 bytes
    of slack each, velocity rows of the padded stride and product columns, each rounded up to
    256 bytes)."""
    def a256(b):
        return (b + 255) // 256 * 256
    k = (n - 1) // 3
    c, ld, cb = k + 1, 2 * k + 1, 2 * precision
    entries = 8 + 16 + 32 + 64 + 128 + 256 + 512
    fixed = a256(entries * 8) + a256(entries * 16) + 256
    # the velocity rows' padded stride (velocity_row_stride): whole column groups and sectors
    e = min(n, 16)
    t = n // e
    lpb = 1 if t >= 64 else 64 // t
    q = max(lpb, 32 // (2 * precision))
    stride = -(-c // q) * q
    m = 1
    while True:
        total = fixed + 3 * a256(cb * c * ld * (m + 1) + 16) + \
            a256(cb * 2 * n * stride * (m + 1)) + a256(cb * 2 * n * c * (m + 1))
        if total > limit:
            return m
        m += 1


def _compare(hz, lib, step_noalloc, cfg, init, forcing_full, forcing_dev_np, steps_list):
    """Runs the ordinary and the allocation-free entry points side by side on two or more
    calls in a row and checks that the states agree exactly (same kernels, same twiddles)."""
    import torch
    n, M, precision = cfg.n, cfg.members, cfg.precision
    ens = hz.Ensemble(cfg)
    ens.set_state(init)
    if forcing_full is not None:
        ens.set_forcing(forcing_full)
    ens.set_time(0.0, 0)
    dtype = np.complex64 if precision == 4 else np.complex128
    tdtype = torch.complex64 if precision == 4 else torch.complex128
    state = torch.from_numpy(hz.full_to_compact(init, n).astype(dtype)).to("cuda", tdtype)
    forcing = None if forcing_dev_np is None else \
        torch.from_numpy(forcing_dev_np.astype(dtype)).to("cuda", tdtype)
    stream = torch.cuda.current_stream().cuda_stream
    c = cfg.to_c()
    status = C.c_uint32(0)
    first = 0
    for steps in steps_list:
        ens.step(DT, steps)
        assert ens.status() == 0
        rc = step_noalloc(C.byref(c), DT, steps, first, C.c_void_p(state.data_ptr()),
                          None if forcing is None else C.c_void_p(forcing.data_ptr()),
                          C.c_void_p(stream), C.byref(status))
        assert rc == 0, lib.hzlb_last_error().decode()
        assert status.value == 0
        first += steps
        torch.cuda.synchronize()
        np.testing.assert_array_equal(state.cpu().numpy(), ens.get_state_compact())
    ens.close()


@pytest.mark.parametrize("precision", [8, 4])
def test_noalloc_step_matches_ensemble_step(precision):
    """Shared Kolmogorov forcing, noise: identical to hzlb_step over two calls in a row."""
    import hzl_stochasticflowinference_b200 as hz
    lib = hz.library()
    cfg = hz.Config(n=N, members=MEMBERS, precision=precision, nu=NU, forcing_kmax=0,
                    noise_sigma=SIGMA, noise_kmax=4, seed=SEED)
    init = np.array([hz.grf_spectrum(N, SEED, m) for m in range(MEMBERS)])
    full = hz.kolmogorov_forcing(N)
    k = (N - 1) // 3
    dev = hz.full_to_compact(full, N)[0].reshape(k + 1, 2 * k + 1)[:1]
    _compare(hz, lib, _bind(lib), cfg, init, full[None], dev, (3, 2))


def test_noalloc_per_member_forcing_and_no_forcing():
    """Per-member forcing (columns kx <= 3, one field per member) and no forcing at all."""
    import hzl_stochasticflowinference_b200 as hz
    lib = hz.library()
    n, M = 32, 5
    k = (n - 1) // 3
    init = np.array([hz.grf_spectrum(n, SEED, m) for m in range(M)])
    full = np.array([hz.kolmogorov_forcing(n, 0.05 * (m + 1), 1 + m % 3) for m in range(M)])
    dev = hz.full_to_compact(full, n).reshape(M, k + 1, 2 * k + 1)[:, :4]
    cfg = hz.Config(n=n, members=M, precision=8, nu=NU, forcing_kmax=3, forcing_per_member=True,
                    noise_sigma=SIGMA, noise_kmax=4, seed=SEED)
    _compare(hz, lib, _bind(lib), cfg, init, full, dev, (2, 3))
    cfg = hz.Config(n=n, members=M, precision=4, nu=NU, forcing_kmax=-1, noise_sigma=SIGMA,
                    noise_kmax=4, seed=SEED)
    _compare(hz, lib, _bind(lib), cfg, init, None, None, (2, 3))


def test_noalloc_fp64_128():
    import hzl_stochasticflowinference_b200 as hz
    lib = hz.library()
    n, M = 128, 3
    init = np.array([hz.grf_spectrum(n, SEED, m) for m in range(M)])
    full = hz.kolmogorov_forcing(n)
    k = (n - 1) // 3
    dev = hz.full_to_compact(full, n)[0].reshape(k + 1, 2 * k + 1)[:1]
    cfg = hz.Config(n=n, members=M, precision=8, nu=5e-4, forcing_kmax=0, noise_sigma=SIGMA,
                    noise_kmax=4, seed=SEED)
    _compare(hz, lib, _bind(lib), cfg, init, full[None], dev, (2, 2))


def test_noalloc_capacity_edge():
    """At 256^2 FP32 the largest member count that fits runs and matches hzlb_step; one more
    member is rejected before any work is queued (its buffer exists all the same)."""
    import torch
    import hzl_stochasticflowinference_b200 as hz
    lib = hz.library()
    step_noalloc = _bind(lib)
    n = 256
    cap = _capacity(n, 4)
    assert cap == 31
    init = np.array([hz.grf_spectrum(n, SEED, m) for m in range(cap)])
    full = hz.kolmogorov_forcing(n)
    k = (n - 1) // 3
    dev = hz.full_to_compact(full, n)[0].reshape(k + 1, 2 * k + 1)[:1]
    cfg = hz.Config(n=n, members=cap, precision=4, nu=2.5e-4, forcing_kmax=0,
                    noise_sigma=SIGMA, noise_kmax=4, seed=SEED)
    _compare(hz, lib, step_noalloc, cfg, init, full[None], dev, (2, 1))
    over = hz.Config(n=n, members=cap + 1, precision=4, nu=2.5e-4).to_c()
    state = torch.zeros((cap + 1) * (k + 1) * (2 * k + 1), dtype=torch.complex64, device="cuda")
    rc = step_noalloc(C.byref(over), 2.5e-4, 1, 0, C.c_void_p(state.data_ptr()), None, None, None)
    assert rc == hz.HZLB_EINVAL
    assert "limit" in lib.hzlb_last_error().decode()


def test_noalloc_rejects_sizes_beyond_the_scratch_limit():
    import hzl_stochasticflowinference_b200 as hz

    lib = hz.library()
    step_noalloc = _bind(lib)
    c = hz.Config(n=512, members=4096, precision=8, nu=1e-4).to_c()
    rc = step_noalloc(C.byref(c), 1e-4, 1, 0, C.c_void_p(1), None, None, None)
    assert rc == hz.HZLB_EINVAL
    assert "limit" in lib.hzlb_last_error().decode()
