"""hzlb_step_host: the ensemble state read from and written to host memory around the steps,
in member chunks whose copies overlap the stepping.  The results are bit-identical with
hzlb_set_state_compact + hzlb_step + hzlb_get_state_compact for every chunk size (odd sizes are
rounded so that each chunk's state stays 16-byte aligned), in FP32 and FP64, and the noise
counter and status carry over to later steps."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import device_synthetic

pytestmark = pytest.mark.gpu


def _pair(hzlb, n, members, precision):
    kmax = min(4, (n - 1) // 3)
    a = device_synthetic(hzlb, n, members, precision, 5e-4, 0.05, 11, wavenumber=kmax,
                         noise_kmax=kmax)
    b = device_synthetic(hzlb, n, members, precision, 5e-4, 0.05, 11, wavenumber=kmax,
                         noise_kmax=kmax)
    return a, b


def _pinned_state(e, dtype):
    state = e.get_state_compact()
    host = torch.from_numpy(np.ascontiguousarray(state).view(dtype)).pin_memory()
    return host, torch.empty_like(host).pin_memory()


@pytest.mark.parametrize("n,members,precision,chunk", [
    (256, 48, 4, 0), (256, 48, 4, 7), (256, 48, 4, 48), (256, 48, 4, 1000),
    (128, 33, 4, 5), (128, 33, 8, 3), (64, 10, 8, 1)])
def test_bit_identical_with_device_stepping(hzlb, n, members, precision, chunk):
    dt, steps = 5e-4, 3
    a, b = _pair(hzlb, n, members, precision)
    dtype = np.float32 if precision == 4 else np.float64
    host_in, host_out = _pinned_state(a, dtype)
    a.set_state_compact_ptr(host_in.data_ptr(), 0, members)
    a.step(dt, steps)
    want = a.get_state_compact()
    b.step_host_ptr(host_in.data_ptr(), host_out.data_ptr(), dt, steps, chunk)
    b.synchronize()
    got = host_out.numpy().view(want.dtype).reshape(want.shape)
    assert np.array_equal(got, want)
    assert b.status() == 0
    # the counter (noise) and the state carry on: one more ordinary step agrees too
    a.step(dt, 1)
    b.step(dt, 1)
    assert np.array_equal(a.get_state_compact(), b.get_state_compact())
    a.close()
    b.close()


def test_in_place_buffer_and_repeated_calls(hzlb):
    a, b = _pair(hzlb, 128, 16, 4)
    host, _ = _pinned_state(a, np.float32)
    for _ in range(3):
        a.set_state_compact_ptr(host.data_ptr(), 0, 16)
        a.step(5e-4, 1)
        a.get_state_compact_ptr(host.data_ptr(), 0, 16)
    a.synchronize()
    want = host.numpy().copy()
    host2, _ = _pinned_state(b, np.float32)
    for _ in range(3):
        b.step_host_ptr(host2.data_ptr(), host2.data_ptr(), 5e-4, 1, 4)
    b.synchronize()
    assert np.array_equal(host2.numpy(), want)
    a.close()
    b.close()


def test_cfl_violation_is_flagged_in_a_chunk(hzlb):
    a, _ = _pair(hzlb, 64, 8, 8)
    state = a.get_state_compact()
    state[5] *= 1e4                       # one member far too fast for dt
    host = torch.from_numpy(np.ascontiguousarray(state).view(np.float64)).pin_memory()
    a.step_host_ptr(host.data_ptr(), host.data_ptr(), 0.01, 1, 2)
    assert a.status() & hzlb.STATUS_CFL
    a.close()


def test_invalid_calls(hzlb):
    a, _ = _pair(hzlb, 32, 4, 4)
    host, out = _pinned_state(a, np.float32)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        a.step_host_ptr(host.data_ptr(), out.data_ptr(), -1.0, 1, 0)
    with pytest.raises(hzlb.HzlbInvalidArgument):
        a.step_host_ptr(0, out.data_ptr(), 1e-3, 1, 0)
    a.close()


def test_per_member_forcing_offsets(hzlb):
    """Per-member forcing: each chunk reads its own members' forcing."""
    n, members = 64, 12
    outs = []
    for use_host in (False, True):
        cfg = hzlb.Config(n=n, members=members, precision=8, nu=1e-3, alpha=0.05,
                          forcing_kmax=4, forcing_per_member=True, noise_sigma=0.02,
                          noise_kmax=4, seed=9)
        e = hzlb.Ensemble(cfg)
        e.set_state(np.array([hzlb.grf_spectrum(n, 9, m) for m in range(members)]))
        e.set_forcing(np.array([(1 + 0.1 * m) * hzlb.kolmogorov_forcing(n, 0.1, 4)
                                for m in range(members)]))
        e.set_time(0.0, 0)
        if use_host:
            host, out = _pinned_state(e, np.float64)
            e.step_host_ptr(host.data_ptr(), out.data_ptr(), 1e-3, 2, 3)
            e.synchronize()
            outs.append(out.numpy().copy())
        else:
            e.step(1e-3, 2)
            outs.append(np.ascontiguousarray(e.get_state_compact()).view(np.float64).reshape(-1))
        e.close()
    assert np.array_equal(outs[0].reshape(-1), outs[1].reshape(-1))


def test_consecutive_calls_chain_and_stay_exact(hzlb):
    """Back-to-back calls on one handle let each chunk's upload follow only the previous call's
    download of that chunk; with the state in place (in = out) and a call of another kind
    breaking the chain halfway, five calls still equal five device steps bit for bit."""
    n, members, dt = 256, 512, 5e-4
    a, b = _pair(hzlb, n, members, 4)
    host, _ = _pinned_state(a, np.float32)
    a.set_state_compact_ptr(host.data_ptr(), 0, members)
    a.step(dt, 5)
    want = a.get_state_compact()
    for i in range(5):
        b.step_host_ptr(host.data_ptr(), host.data_ptr(), dt, 1, 0)
        if i == 2:
            assert b.status() == 0   # another call in between: the next one starts afresh
    b.synchronize()
    got = host.numpy().view(want.dtype).reshape(want.shape)
    assert np.array_equal(got, want)
    assert b.status() == 0
    a.close()
    b.close()
