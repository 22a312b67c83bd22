"""OU shell forcing on the device (hzlb_enable_ou) against the statistics the reference's own
test asserts (tests/verification.cpp:109-140): 2048 members at 16^2, sigma 0.5, tau 0.3, one
step of 0.05 — stationary variance sigma^2 tau / 4 before and after within 5 standard errors,
lag correlation exp(-dt/tau) within 0.04 — plus the conjugate symmetry of the kx = 0 column and
that forcing outside the shell is left alone."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [8, 4])
def test_ou_moments_match_reference_test(hzlb, precision):
    n, count, sigma, tau, dt = 16, 2048, 0.5, 0.3, 0.05
    cfg = hzlb.Config(n=n, members=count, precision=precision, nu=0.01, alpha=0.1,
                      forcing_kmax=3, forcing_per_member=True, seed=123)
    e = hzlb.Ensemble(cfg)
    e.set_state(np.zeros((count, n, n), np.complex128))
    e.enable_ou(sigma, tau, 2, 3)
    k = (n - 1) // 3
    ld = 2 * k + 1
    f0 = e.forcing_compact().reshape(count, -1, ld)
    e.step(dt, 1)
    f1 = e.forcing_compact().reshape(count, -1, ld)
    a, b = f0[:, 2, 0].real, f1[:, 2, 0].real        # mode (kx, ky) = (2, 0), as the reference test
    variance = sigma ** 2 * tau / 4
    tol = 5 * np.sqrt(2.0 / (count - 1))
    assert abs(a.var(ddof=1) / variance - 1) < tol
    assert abs(b.var(ddof=1) / variance - 1) < tol
    corr = np.corrcoef(a, b)[0, 1]
    assert abs(corr - np.exp(-dt / tau)) < 0.04
    # kx = 0 column: (0, -ky) is the conjugate of (0, ky); modes outside the shell stay zero
    np.testing.assert_array_equal(f1[:, 0, ld - 2], np.conj(f1[:, 0, 2]))
    assert np.all(f1[:, 1, 1] == 0) and np.all(f1[:, 0, 1] == 0)   # |k|^2 = 2 and 1 < kmin^2
    assert np.all(f1[:, 3, 3] == 0)                                 # |k|^2 = 18 > kmax^2
    # the forcing drove the fields (they start at rest)
    assert np.all(np.isfinite(e.get_state_compact())) and np.abs(e.get_state_compact()).max() > 0
    e.close()


def test_ou_rejects_bad_configuration(hzlb):
    e = hzlb.Ensemble(hzlb.Config(n=16, members=2, precision=8, forcing_kmax=1,
                                  forcing_per_member=True))
    with pytest.raises(hzlb.HzlbInvalidArgument):
        e.enable_ou(0.5, 0.3, 2, 3)          # storage does not cover the shell
    shared = hzlb.Ensemble(hzlb.Config(n=16, members=2, precision=8, forcing_kmax=3))
    with pytest.raises(hzlb.HzlbInvalidArgument):
        shared.enable_ou(0.5, 0.3, 2, 3)     # one forcing for all members
