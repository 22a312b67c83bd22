"""HZL_CHECKPOINT_V1 files of device-resident solver sets (hzlb_solvers_*) against the reference
library's own hzl::Solver::save / Solver::load (src/solver.cpp:434-491) on the same inputs:
the files agree line by line (random streams and latent forcing exactly, vorticity to FP64
roundoff), each library restarts from the other's files, and a restart continues the same
trajectory as an uninterrupted run."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_l2
from oracle.oracle import params6

pytestmark = pytest.mark.gpu

N, DT, STEPS = 32, 0.005, 40
P = (0.02, 0.1, 0.2, 0.5, 2, 3)


def _seeds(reference):
    return [42, 7, reference.stream_seed(5, 2)]


def _parse(path):
    lines = path.read_text().splitlines()
    rows = np.array([[float(v) for v in line.split()] for line in lines[5:]])
    return lines[:5], rows


def _reference_run(reference, seed, steps, initial="multimode"):
    s = reference.solver(N, params6(*P), seed)
    s.initialize(initial)
    s.step(DT, steps)
    return s


def test_saved_files_match_reference(hzlb, reference, tmp_path):
    seeds = _seeds(reference)
    ours = hzlb.Solvers(N, hzlb.Parameters(*P), seeds, "multimode")
    ours.step(DT, STEPS)
    for i, seed in enumerate(seeds):
        ours.save(i, tmp_path / f"ours{i}.txt")
        _reference_run(reference, seed, STEPS).save(tmp_path / f"ref{i}.txt")
        head_o, rows_o = _parse(tmp_path / f"ours{i}.txt")
        head_r, rows_r = _parse(tmp_path / f"ref{i}.txt")
        # magic, "n time", parameters, the mt19937_64 state, the cached normal
        assert head_o == head_r
        assert rows_o.shape == (N * N, 4)
        np.testing.assert_array_equal(rows_o[:, 2:], rows_r[:, 2:])          # latent forcing
        w_o = rows_o[:, 0] + 1j * rows_o[:, 1]
        w_r = rows_r[:, 0] + 1j * rows_r[:, 1]
        assert rel_l2(w_o, w_r) <= 1e-12
        np.testing.assert_array_equal(w_o == 0, w_r == 0)                   # inactive modes
    ours.close()


def test_reference_restarts_from_our_checkpoint(hzlb, reference, tmp_path):
    seeds = _seeds(reference)
    ours = hzlb.Solvers(N, hzlb.Parameters(*P), seeds, "multimode")
    ours.step(DT, STEPS)
    for i in range(len(seeds)):
        ours.save(i, tmp_path / f"ours{i}.txt")
    ours.step(DT, 20)
    w, f = ours.coefficients()
    for i, seed in enumerate(seeds):
        restarted = reference.solver_load(tmp_path / f"ours{i}.txt")
        restarted.step(DT, 20)
        assert rel_l2(w[i], restarted.coefficients()) <= 1e-12
        np.testing.assert_allclose(f[i], restarted.forcing(), rtol=0, atol=1e-15)
        straight = _reference_run(reference, seed, STEPS + 20)
        assert rel_l2(restarted.coefficients(), straight.coefficients()) <= 1e-12
    ours.close()


def test_restart_from_reference_checkpoints(hzlb, reference, tmp_path):
    seeds = _seeds(reference)
    paths = []
    for i, seed in enumerate(seeds):
        _reference_run(reference, seed, STEPS, "taylor-green").save(tmp_path / f"ref{i}.txt")
        paths.append(tmp_path / f"ref{i}.txt")
    ours = hzlb.Solvers.load(paths)
    assert (ours.n, ours.count) == (N, len(seeds))
    ours.step(DT, 25)
    w, f = ours.coefficients()
    d = ours.diagnostics()
    for i, seed in enumerate(seeds):
        straight = _reference_run(reference, seed, STEPS + 25, "taylor-green")
        assert rel_l2(w[i], straight.coefficients()) <= 1e-12
        np.testing.assert_allclose(f[i], straight.forcing(), rtol=0, atol=1e-15)
        dr = straight.diagnostics()
        assert d[i, 0] == dr[0]                                   # time: the same sum of dt
        np.testing.assert_allclose(d[i, 1:5], dr[1:5], rtol=1e-11, atol=1e-14)
    # save -> load -> save reproduces the file
    ours.save(1, tmp_path / "again.txt")
    again = hzlb.Solvers.load([tmp_path / "again.txt"])
    again.save(0, tmp_path / "again2.txt")
    assert (tmp_path / "again.txt").read_bytes() == (tmp_path / "again2.txt").read_bytes()
    ours.close()
    again.close()


def test_create_matches_reference_ensemble_members(hzlb, reference):
    """seeds[i] = stream_seed(seed, i) gives hzl::ensemble's members."""
    seeds = [reference.stream_seed(77, i) for i in range(4)]
    ours = hzlb.Solvers(16, hzlb.Parameters(), seeds, "zero")
    ours.step(0.01, 4)
    got = ours.diagnostics()
    ref = reference.ensemble(16, params6(0.01, 0.1, 0.2, 0.5, 2, 3), 0.01, 4, 4, 2, 77)
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=1e-15)
    np.testing.assert_allclose(got[:, 1:5], ref[:, 1:5], rtol=1e-11, atol=1e-14)
    ours.close()
