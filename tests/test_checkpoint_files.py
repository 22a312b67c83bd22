"""Malformed and inconsistent HZL_CHECKPOINT_V1 files are refused by hzlb_solvers_load with the
messages of the reference's hzl::Solver::load (src/solver.cpp:453-491).  Every case fails while
the files are read, before any device work, so this runs without a GPU; the reference writes
the valid file that each case corrupts."""
from __future__ import annotations

import pytest

from oracle.oracle import OracleError, params6

N = 16
P = params6(0.02, 0.1, 0.2, 0.5, 2, 3)


@pytest.fixture
def good(reference, tmp_path):
    s = reference.solver(N, P, 11)
    s.initialize("multimode")
    s.step(0.01, 5)
    s.save(tmp_path / "good.txt")
    return (tmp_path / "good.txt").read_text().splitlines()


def _corrupt(lines, name):
    lines = list(lines)
    if name == "magic":
        lines[0] = "HZL_CHECKPOINT_V2"
    elif name == "negative time":
        lines[1] = f"{N} -1"
    elif name == "grid":
        lines[1] = "12 " + lines[1].split()[1]
    elif name == "parameters":
        lines[2] = "0.02 0.1 0.2 0 2 3"            # tau must be positive
    elif name == "shell":
        lines[2] = "0.02 0.1 0.2 0.5 2 7"          # beyond the dealiased band of 16
    elif name == "random stream":
        lines[3] = "not-a-state"
    elif name == "nonfinite field":
        lines[6] = "nan 0 0 0"
    elif name == "short field":
        lines = lines[:-3]
    elif name == "inactive mode":
        lines[5 + 8] = "1 0 0 0"                   # kx = 8: outside the retained band
    elif name == "mean mode":
        lines[5] = "1e-3 0 0 0"                    # k = 0
    elif name == "forcing symmetry":
        a, b, c, d = lines[5 + 2].split()         # (kx, ky) = (2, 0), a forced mode
        lines[5 + 2] = f"{a} {b} {float(c) + 1e-9!r} {d}"
    elif name == "trailing":
        lines.append("42")
    return "\n".join(lines) + "\n"


CASES = ["magic", "negative time", "grid", "parameters", "shell", "random stream",
         "nonfinite field", "short field", "inactive mode", "mean mode", "forcing symmetry",
         "trailing"]


@pytest.mark.parametrize("name", CASES)
def test_refused_with_reference_message(hzlb, reference, good, tmp_path, name):
    bad = tmp_path / "bad.txt"
    bad.write_text(_corrupt(good, name))
    with pytest.raises(OracleError) as theirs:
        reference.solver_load(bad)
    with pytest.raises(hzlb.HzlbError) as ours:
        hzlb.Solvers.load([bad])
    assert str(ours.value) == str(theirs.value)


def test_a_set_shares_grid_parameters_and_time(hzlb, reference, good, tmp_path):
    (tmp_path / "a.txt").write_text("\n".join(good) + "\n")
    s = reference.solver(N, P, 12)
    s.initialize("multimode")
    s.step(0.01, 6)                                # a different time
    s.save(tmp_path / "b.txt")
    with pytest.raises(hzlb.HzlbInvalidArgument, match="share grid, parameters and time"):
        hzlb.Solvers.load([tmp_path / "a.txt", tmp_path / "b.txt"])


def test_grids_beyond_the_device_limit(hzlb, reference, tmp_path):
    """The reference's solver runs up to 4096^2 on the CPU; the device path stops at 512^2."""
    s = reference.solver(1024, params6(0.02, 0.1, 0.2, 0.5, 2, 3), 1)
    s.initialize("zero")
    s.save(tmp_path / "big.txt")
    reference.solver_load(tmp_path / "big.txt")
    with pytest.raises(hzlb.HzlbInvalidArgument, match="between 8 and 512"):
        hzlb.Solvers.load([tmp_path / "big.txt"])
