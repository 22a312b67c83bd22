"""The drop-in hzl::CudaSolver (hzl_stochasticflowinference_b200/shim/cuda_solver_b200.cpp,
compiled against the reference's unchanged include/hzl/cuda_solver.hpp) passes the
reference's own CPU/GPU parity check (src/cuda_benchmark.cpp:37-80) at the sizes of the
reference's recorded evidence (docs/evidence/gpu-256.json: 256^2, 100 steps, dt 0.005;
README: 128^2, 200 steps, sigma 0.2)."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
BIN = Path(__file__).resolve().parent / "cpp" / "shim_parity"


@pytest.mark.parametrize("args", [("256", "100", "0.005"), ("128", "200", "0.005", "0.2"),
                                  ("64", "50", "0.005", "0.2")])
def test_cuda_solver_shim_parity(args):
    if not BIN.exists():
        pytest.skip("shim_parity not built (needs the reference headers at build time)")
    out = subprocess.run([str(BIN), *args], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    result = json.loads(out.stdout.strip().splitlines()[-1])
    assert result["relative_l2_error"] <= 1e-12
    assert result["invalid_argument_on_missing_forcing"]
    # a CFL violation throws before the state changes, and the instance steps on from it
    assert result["cfl_throws"] and result["cfl_state_unchanged"] and result["cfl_steps_on"]
