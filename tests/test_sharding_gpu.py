"""The sharded analysis on the device: the functions of sharding.py with sharding.DeviceAnalysis
(the library's FP64 particle weights and resampling, FP64 Cholesky and solve of the gathered
innovation system, FP64 tensor-core anomaly products) over an NCCL process group on CUDA
tensors.  One GPU is available, so the group has one rank; the communication logic with
several ranks is covered on CPU by tests/test_multirank.py."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from helpers import enkf_weight_matrix

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.fixture
def nccl_group():
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        yield dist
    finally:
        dist.destroy_process_group()


def test_device_analysis_matches_the_reference_formulas(hzlb, oracle, nccl_group):
    import torch
    from hzl_stochasticflowinference_b200 import sharding
    total, dim, p = 96, 132, 40
    e = hzlb.Ensemble(hzlb.Config(n=16, members=8, precision=8, nu=1e-3))
    analysis = sharding.DeviceAnalysis(e)
    rng = np.random.default_rng(7)
    logs = rng.normal(-30, 6, total)
    states = rng.normal(size=(total, dim))
    hx = rng.normal(size=(total, p))
    eps = rng.normal(size=(total, p))
    y, sd = rng.normal(size=p), np.full(p, 0.25)
    dev = torch.device("cuda", 0)
    # particle filter: the device weights against the oracle's restatement of the reference,
    # the ancestors bit for bit given the device weights
    w, inc, ess, mw, anc = sharding.pf_resample_distributed(
        torch.from_numpy(logs).to(dev), 0.41, analysis)
    w2, inc2, ess2, mw2 = oracle.pf_weights(logs)
    np.testing.assert_allclose(w, w2, rtol=1e-13, atol=0)
    np.testing.assert_allclose([inc, ess, mw], [inc2, ess2, mw2], rtol=1e-13)
    np.testing.assert_array_equal(anc, oracle.systematic_resample(w, 0.41))
    moved = sharding.exchange_members(torch.from_numpy(states).to(dev), anc)
    np.testing.assert_array_equal(moved.cpu().numpy(), states[anc])
    # EnKF: device Cholesky and solve of the gathered system, device anomaly products
    W = enkf_weight_matrix(hx, y, sd, eps)
    Wd = analysis.enkf_weights(torch.from_numpy(hx).to(dev), y, sd, torch.from_numpy(eps).to(dev))
    np.testing.assert_allclose(Wd.cpu().numpy(), W, rtol=0, atol=1e-11 * np.abs(W).max())
    xa = sharding.enkf_distributed(torch.from_numpy(states).to(dev), torch.from_numpy(hx).to(dev),
                                   y, sd, torch.from_numpy(eps).to(dev), analysis)
    expect = states + (states - states.mean(axis=0)).T.dot(W).T
    np.testing.assert_allclose(xa.cpu().numpy(), expect, rtol=0, atol=1e-11 * np.abs(expect).max())
    e.close()


@pytest.mark.parametrize("shape", [(64, 64, 64), (96, 132, 40), (1, 7, 300), (130, 3, 2)])
def test_dgemm_transposes_and_accumulates(hzlb, shape):
    """hzlb_dgemm: C = alpha op(A) op(B) + beta C on the FP64 tensor cores, every transpose
    combination, against numpy."""
    import torch
    m, n, k = shape
    rng = np.random.default_rng(3)
    dev = torch.device("cuda", 0)
    for at in (False, True):
        for bt in (False, True):
            a = rng.normal(size=(k, m) if at else (m, k))
            b = rng.normal(size=(n, k) if bt else (k, n))
            c0 = rng.normal(size=(m, n))
            c = torch.from_numpy(c0.copy()).to(dev)
            hzlb.dgemm(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev), c, alpha=0.5,
                       beta=-2.0, a_trans=at, b_trans=bt)
            expect = 0.5 * (a.T if at else a) @ (b.T if bt else b) - 2.0 * c0
            torch.cuda.synchronize()
            np.testing.assert_allclose(c.cpu().numpy(), expect, rtol=0,
                                       atol=1e-12 * max(1.0, np.abs(expect).max()) * k)
