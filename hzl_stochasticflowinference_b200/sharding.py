"""Member sharding across GPUs (one process per GPU, torch.distributed).

Ensemble members are independent during the forecast, so each rank holds a contiguous block
of members and steps it with no communication (the multi-rank analogue of the reference's
round-robin MPI ensemble, src/mpi_ensemble.cpp:40-61, and of its worker pool,
src/inference.cpp:555-590).  Exchanges happen only in the analysis:

* particle filter (src/filter.cpp:76-120): one all-gather of the M log-weights; every rank
  then computes the same normalised weights and the same systematic-resampling ancestors from
  the shared uniform, and members whose ancestor lives on another rank are copied point to
  point (send/recv of the member state);
* EnKF (src/filter.cpp:265-321 in batched form): one all-gather of the predicted
  observations HX (and the perturbation draws); each rank factorises the same p x p
  innovation system and forms the same M x M weight matrix W; the update
  X_a[:, mine] = X[:, mine] + sum_r A_r W[rows of r, mine] is one reduce-scatter of the
  per-rank partial products A_r W[rows of r, :].

The arithmetic of both runs on the rank's GPU through the library (`DeviceAnalysis`: the
particle weights and resampling in FP64, the FP64 Cholesky and solve of the innovation system,
the FP64 anomaly products on the tensor cores); this module only moves data between ranks.
The collective functions take torch tensors (CUDA tensors over NCCL) and an analysis object
with the methods of `DeviceAnalysis`, which tests may replace to check the communication
logic on CPU ranks over gloo.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def shard_range(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced block of members [first, first + count) for `rank`."""
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def owner(member: int, total: int, world: int) -> tuple[int, int]:
    """(rank, local index) holding global `member` under shard_range."""
    base, extra = divmod(total, world)
    cut = extra * (base + 1)
    if member < cut:
        return member // (base + 1), member % (base + 1)
    r = extra + (member - cut) // base
    return r, (member - cut) % base


def balance_mixed(groups: list[tuple[int, int, float]], world: int) -> list[list[tuple[int, int, int]]]:
    """Splits a mixed-resolution ensemble [(n, members, bytes_per_member_step)] over ranks so
    that every rank carries about the same bytes per step.  Returns, per rank, the slices
    (group index, first member, count)."""
    total = sum(m * b for _, m, b in groups)
    target = total / world
    out: list[list[tuple[int, int, int]]] = [[] for _ in range(world)]
    rank, load = 0, 0.0
    for gi, (n, members, b) in enumerate(groups):
        first = 0
        while first < members:
            if rank == world - 1:
                take = members - first
            else:
                take = min(members - first, max(1, int(max(target - load, b) // b)))
            out[rank].append((gi, first, take))
            load += take * b
            first += take
            if load >= target - 0.5 * b and rank < world - 1:
                rank, load = rank + 1, 0.0
    return out


def _gather_concat(local: torch.Tensor, group=None) -> torch.Tensor:
    world = dist.get_world_size(group)
    sizes = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    all_sizes = [torch.zeros_like(sizes) for _ in range(world)]
    dist.all_gather(all_sizes, sizes, group=group)
    cap = int(max(s.item() for s in all_sizes))
    padded = torch.zeros((cap,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[: local.shape[0]] = local
    parts = [torch.zeros_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[: int(s.item())] for p, s in zip(parts, all_sizes)], dim=0)


class DeviceAnalysis:
    """The analysis arithmetic of a sharded filter on this rank's GPU, through the library:
    particle weights and systematic resampling (hzlb_pf_weights, hzlb_systematic_resample:
    FP64 in the reference's order), the ensemble-space EnKF solve of the gathered predicted
    observations (hzlb_enkf_weights: FP64 Cholesky and forward substitution) and the anomaly
    products (hzlb_dgemm, FP64 tensor cores).  `ensemble` is this rank's handle; the solves run
    on its device and stream."""

    def __init__(self, ensemble):
        from . import dgemm
        self.ensemble = ensemble
        self._dgemm = dgemm

    def pf_weights(self, logs: np.ndarray):
        """(weights, increment, ess, max weight) of all M log-weights (filter.cpp:76-92)."""
        return self.ensemble.pf_weights(logs)

    def resample(self, weights: np.ndarray, u: float) -> np.ndarray:
        """Ancestors of systematic resampling with uniform u (filter.cpp:102-112)."""
        return self.ensemble.resample(weights, u)

    def enkf_weights(self, hx: torch.Tensor, y, sd, eps: torch.Tensor) -> torch.Tensor:
        """W (M x M, rows: contributing member) of the gathered HX and perturbations."""
        w, _ = self.ensemble.enkf_weights(hx, y, sd, eps)
        return w

    def anomaly_products(self, anomalies: torch.Tensor, w_rows: torch.Tensor) -> torch.Tensor:
        """w_rows^T anomalies: (total, dim) from this rank's (count, dim) anomalies and its
        (count, total) rows of W."""
        out = torch.empty((w_rows.shape[1], anomalies.shape[1]), dtype=torch.float64,
                          device=anomalies.device)
        self._dgemm(w_rows.contiguous(), anomalies.contiguous(), out, a_trans=True)
        return out


def pf_resample_distributed(local_log_weights: torch.Tensor, u: float, analysis, group=None):
    """All-gathers the log-weights; returns (weights, increment, ess, max weight, ancestors),
    identical on every rank."""
    logs = _gather_concat(local_log_weights.to(torch.float64), group).cpu().numpy()
    w, inc, ess, mw = analysis.pf_weights(logs)
    return w, inc, ess, mw, analysis.resample(w, u)


def migration_plan(ancestors: np.ndarray, world: int) -> list[list[tuple[int, int, int]]]:
    """Per destination rank: (destination local slot, source rank, source local slot) for every
    member slot whose new state comes from `ancestors`."""
    total = len(ancestors)
    plan: list[list[tuple[int, int, int]]] = [[] for _ in range(world)]
    for g, a in enumerate(ancestors):
        dr, dl = owner(g, total, world)
        sr, sl = owner(int(a), total, world)
        plan[dr].append((dl, sr, sl))
    return plan


def exchange_members(local_states: torch.Tensor, ancestors: np.ndarray, group=None) -> torch.Tensor:
    """New local states after resampling: local copies plus point-to-point transfers of the
    members whose ancestor lives on another rank.  local_states: (local members, ...)."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    plan = migration_plan(ancestors, world)
    out = torch.empty_like(local_states)
    ops = []
    recv_bufs = []
    # sends: every (dst rank != me) entry whose source is me
    for dr in range(world):
        if dr == rank:
            continue
        for dl, sr, sl in plan[dr]:
            if sr == rank:
                ops.append(dist.P2POp(dist.isend, local_states[sl].contiguous(), dr, group))
    for dl, sr, sl in plan[rank]:
        if sr == rank:
            out[dl] = local_states[sl]
        else:
            buf = torch.empty_like(local_states[0])
            recv_bufs.append((dl, buf))
            ops.append(dist.P2POp(dist.irecv, buf, sr, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for dl, buf in recv_bufs:
        out[dl] = buf
    return out


def enkf_distributed(local_x: torch.Tensor, local_hx: torch.Tensor, y: np.ndarray,
                     sd: np.ndarray, local_eps: torch.Tensor, analysis, group=None) -> torch.Tensor:
    """Batched EnKF analysis of member-sharded states.  local_x: (local members, state dim)
    real; local_hx, local_eps: (local members, p).  Returns the analysed local states."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    hx = _gather_concat(local_hx.to(torch.float64), group)
    eps = _gather_concat(local_eps.to(torch.float64), group)
    total = hx.shape[0]
    w = analysis.enkf_weights(hx, np.asarray(y), np.asarray(sd), eps)
    first, count = shard_range(total, world, rank)
    xs = local_x.to(torch.float64)
    mean = xs.sum(dim=0, keepdim=True)
    dist.all_reduce(mean, group=group)
    mean /= total
    partial = analysis.anomaly_products(xs - mean, w[first:first + count, :])   # (total, dim)
    chunks = [partial[a:a + c] for a, c in (shard_range(total, world, r) for r in range(world))]
    mine = torch.empty((count,) + tuple(partial.shape[1:]), dtype=partial.dtype, device=partial.device)
    if world == 1:
        mine.copy_(chunks[0])
    elif all(c.shape[0] == chunks[0].shape[0] for c in chunks):
        dist.reduce_scatter(mine, chunks, group=group)
    else:   # uneven shards: reduce each destination's block to its owner
        for r, c in enumerate(chunks):
            buf = c.clone()
            dist.reduce(buf, dst=r, group=group)
            if r == rank:
                mine.copy_(buf)
    return (xs + mine).to(local_x.dtype)
