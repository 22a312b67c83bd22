"""CPU checks of the C ABI: the library loads, exports every symbol include/hzlb.h declares,
its host-only entry points (random fields, forcing, layouts) agree with the oracle, and device
entry points fail loudly (no CPU fallback) when no GPU is present."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> list[str]:
    text = (ROOT / "include" / "hzlb.h").read_text()
    return sorted(set(re.findall(r"HZLB_API\s+[\w\s\*]*?\b(hzlb_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "hzlb_ensemble_create" in names and "hzlb_step" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(hzlb):
    lib = hzlb.library()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_grf_matches_oracle(hzlb, oracle):
    for n in (16, 64, 256):
        for member in (0, 3):
            a = hzlb.grf_spectrum(n, 42, member)
            b = oracle.grf(n, 42, member)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-15 * np.abs(b).max())
            area = 4 * np.pi ** 2
            assert abs(area / 2 * np.sum(np.abs(a) ** 2) - 1) < 1e-13


def test_kolmogorov_matches_oracle(hzlb, oracle):
    np.testing.assert_array_equal(hzlb.kolmogorov_forcing(64), oracle.kolmogorov(64))


def test_resampling_needs_an_ensemble(hzlb):
    """Systematic resampling has no host path: a NULL handle is rejected."""
    w = np.array([0.5, 0.5])
    out = np.zeros(2, np.uint32)
    lib = hzlb.library()
    rc = lib.hzlb_systematic_resample(None, w.ctypes.data_as(hzlb._dp), 2, 0.5,
                                      out.ctypes.data_as(hzlb._u32p))
    assert rc == hzlb.HZLB_EINVAL


def test_compact_layout_round_trip(hzlb, oracle):
    n = 32
    w = oracle.grf(n, 1, 0)
    c = hzlb.full_to_compact(w, n)
    np.testing.assert_array_equal(hzlb.compact_to_full(c, n)[0], w)


def test_device_calls_fail_loudly_without_gpu(hzlb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hzlb.HzlbError):
        hzlb.Ensemble(hzlb.Config(n=32, members=1))
