"""Multi-rank member sharding on CPU (gloo, world size 2): the sharded particle-filter
resampling and the sharded EnKF analysis give the same result as the single-process
computation, and every member is owned exactly once."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hzl_stochasticflowinference_b200 import sharding


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges_cover_every_member_once():
    for total in (1, 7, 2048, 4099):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                first, count = sharding.shard_range(total, world, r)
                seen.extend(range(first, first + count))
                for i in range(count):
                    assert sharding.owner(first + i, total, world) == (r, i)
            assert seen == list(range(total))


def test_mixed_resolution_balance():
    # 4096 x 64^2, 1024 x 128^2, 128 x 256^2, 8 x 512^2 with bytes ~ N^2
    groups = [(64, 4096, 64.0 ** 2), (128, 1024, 128.0 ** 2), (256, 128, 256.0 ** 2),
              (512, 8, 512.0 ** 2)]
    for world in (1, 2, 4, 8):
        plan = sharding.balance_mixed(groups, world)
        counts = {gi: 0 for gi in range(len(groups))}
        loads = []
        for slices in plan:
            loads.append(sum(c * groups[gi][2] for gi, _, c in slices))
            for gi, first, c in slices:
                counts[gi] += c
        assert counts == {gi: g[1] for gi, g in enumerate(groups)}
        assert max(loads) <= 1.2 * (sum(loads) / world) + 512.0 ** 2


# 64 members of 16^2 states in the compact layout (2 x 66 reals each), 20 observations
TOTAL, DIM, P = 64, 132, 20


def _problem():
    rng = np.random.default_rng(5)
    logs = rng.normal(-20, 4, TOTAL)
    states = rng.normal(size=(TOTAL, DIM))
    hx = rng.normal(size=(TOTAL, P))
    eps = rng.normal(size=(TOTAL, P))
    y, sd = rng.normal(size=P), np.full(P, 0.3)
    return logs, states, hx, eps, y, sd


def _worker(rank, world, port, q):
    from helpers import HostAnalysis
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        logs, states, hx, eps, y, sd = _problem()
        analysis = HostAnalysis()
        first, count = sharding.shard_range(TOTAL, world, rank)
        sl = slice(first, first + count)
        # particle filter: identical weights and ancestors on every rank, then migration
        w, inc, ess, mw, anc = sharding.pf_resample_distributed(torch.from_numpy(logs[sl]), 0.37,
                                                                analysis)
        moved = sharding.exchange_members(torch.from_numpy(states[sl].copy()), anc)
        # EnKF: all-gather of HX, redundant solve, reduce-scatter of partial products
        xa = sharding.enkf_distributed(torch.from_numpy(states[sl].copy()),
                                       torch.from_numpy(hx[sl]), y, sd,
                                       torch.from_numpy(eps[sl]), analysis)
        q.put((rank, first, anc, inc, ess, moved.numpy(), xa.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_filters_match_single_process(world, oracle):
    """The sharded filters on `world` gloo ranks (member blocks of 32/32 and 22/21/21) equal
    the single-process computation: identical weights and ancestors on every rank, migrated
    members equal to their ancestors, and the analysed states of the reduce-scatter update."""
    from helpers import enkf_weight_matrix
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    logs, states, hx, eps, y, sd = _problem()
    w, inc, ess, mw = oracle.pf_weights(logs)
    anc = oracle.systematic_resample(w, 0.37)
    assert len(set(anc.tolist())) < TOTAL   # the weights are uneven enough to resample
    W = enkf_weight_matrix(hx, y, sd, eps)
    xa = states + (states - states.mean(axis=0)).T.dot(W).T
    moved_all, xa_all = np.zeros_like(states), np.zeros_like(states)
    for rank, first, a, i, e, moved, xa_local in results:
        np.testing.assert_array_equal(a, anc)
        assert i == inc and e == ess
        moved_all[first:first + len(moved)] = moved
        xa_all[first:first + len(xa_local)] = xa_local
    np.testing.assert_array_equal(moved_all, states[anc])
    np.testing.assert_allclose(xa_all, xa, rtol=1e-12, atol=1e-12)
