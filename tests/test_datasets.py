"""Observation dataset files (HZL_OBSERVATIONS_V1/V2) against the reference library's own
hzl::Dataset::save / load / validate (src/inference.cpp:197-257): the files are byte-identical,
each side reads the other's files, and malformed or invalid files fail with the reference's
messages.  Host code only: no GPU."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import OracleError, params6


def _reference_dataset(reference, sigma=0.2):
    p6 = params6(0.03, 0.1, sigma, 0.5, 2, 3)
    return reference.synthetic_observations(16, 0.01, 150, 10, p6, 0.02, 314159)


def _same(a: dict, b: dict):
    for key in ("n", "stochastic", "forcing_min", "forcing_max"):
        assert int(a[key]) == int(b[key]), key
    assert a["dt"] == b["dt"]
    for key in ("steps", "x", "y"):
        np.testing.assert_array_equal(np.asarray(a[key]), np.asarray(b[key]))
    for key in ("value", "sd"):
        np.testing.assert_array_equal(np.asarray(a[key], np.float64), np.asarray(b[key], np.float64))


def test_save_is_byte_identical(hzlb, reference, tmp_path):
    for sigma in (0.2, 0.0):
        ds = _reference_dataset(reference, sigma)
        ours, theirs = tmp_path / f"ours{sigma}.csv", tmp_path / f"theirs{sigma}.csv"
        hzlb.save_dataset(ds, ours)
        reference.dataset_save(ds, theirs)
        assert ours.read_bytes() == theirs.read_bytes()
        assert ours.read_text().startswith(f"HZL_OBSERVATIONS_V2,16,0.01,{int(sigma > 0)},2,3\n")


def test_each_reads_the_others_files(hzlb, reference, tmp_path):
    ds = _reference_dataset(reference)
    rng = np.random.default_rng(5)
    ds["value"] = ds["value"] + rng.normal(size=len(ds["value"])) * 1e-3   # full-precision values
    hzlb.save_dataset(ds, tmp_path / "ours.csv")
    reference.dataset_save(ds, tmp_path / "theirs.csv")
    _same(hzlb.load_dataset(tmp_path / "theirs.csv"), ds)
    _same(reference.dataset_load(tmp_path / "ours.csv"), ds)
    _same(hzlb.load_dataset(tmp_path / "ours.csv"), reference.dataset_load(tmp_path / "ours.csv"))


def test_version_1_header_and_blank_lines(hzlb, reference, tmp_path):
    f = tmp_path / "v1.csv"
    f.write_text("HZL_OBSERVATIONS_V1,32,0.005\nstep,x,y,vorticity,standard_deviation\n"
                 "\n10,1,2,0.5,0.1\n\n20,3,4,-0.25,0.2\n")
    got, ref = hzlb.load_dataset(f), reference.dataset_load(f)
    _same(got, ref)
    assert (got["n"], got["stochastic"], got["forcing_min"], got["forcing_max"]) == (32, 0, 2, 3)
    assert list(got["steps"]) == [10, 20]


BAD_FILES = {
    "empty": "",
    "magic": "HZL_OBSERVATIONS_V3,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n1,0,0,1,1\n",
    "metadata": "HZL_OBSERVATIONS_V2,16,0.01\nstep,x,y,vorticity,standard_deviation\n1,0,0,1,1\n",
    "columns": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,value,sd\n1,0,0,1,1\n",
    "extra token": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n"
                   "1,0,0,1,1,7\n",
    "short row": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n1,0,0,1\n",
    "no rows": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n",
    "unordered": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n"
                 "5,0,0,1,1\n4,0,0,1,1\n",
    "out of grid": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n"
                   "5,16,0,1,1\n",
    "zero sd": "HZL_OBSERVATIONS_V2,16,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n"
               "5,0,0,1,0\n",
    "grid": "HZL_OBSERVATIONS_V2,12,0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n5,0,0,1,1\n",
    "small grid": "HZL_OBSERVATIONS_V2,8,0.01,1,1,2\nstep,x,y,vorticity,standard_deviation\n"
                  "5,0,0,1,1\n",
    "shell": "HZL_OBSERVATIONS_V2,16,0.01,1,2,6\nstep,x,y,vorticity,standard_deviation\n5,0,0,1,1\n",
    "dt": "HZL_OBSERVATIONS_V2,16,-0.01,1,2,3\nstep,x,y,vorticity,standard_deviation\n5,0,0,1,1\n",
}


@pytest.mark.parametrize("name", sorted(BAD_FILES))
def test_bad_files_fail_with_the_reference_messages(hzlb, reference, tmp_path, name):
    f = tmp_path / "bad.csv"
    f.write_text(BAD_FILES[name])
    with pytest.raises(OracleError) as theirs:
        reference.dataset_load(f)
    with pytest.raises(hzlb.HzlbError) as ours:
        hzlb.load_dataset(f)
    assert str(ours.value) == str(theirs.value)


def test_invalid_dataset_is_not_written(hzlb, reference, tmp_path):
    ds = _reference_dataset(reference)
    ds["sd"] = ds["sd"].copy()
    ds["sd"][3] = -1.0
    with pytest.raises(hzlb.HzlbInvalidArgument, match="positive uncertainty"):
        hzlb.save_dataset(ds, tmp_path / "x.csv")
    with pytest.raises(hzlb.HzlbInvalidArgument, match="positive uncertainty"):
        hzlb.validate_dataset(ds)
    assert not (tmp_path / "x.csv").exists()
    with pytest.raises(hzlb.HzlbError, match="observation write failed"):
        hzlb.save_dataset(_reference_dataset(reference), tmp_path / "missing" / "x.csv")
