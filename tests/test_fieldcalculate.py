"""fieldCalculate without a GPU: the oracle's arithmetic and the executable's
command-line handling (no device call is made on these paths)."""
import os
import subprocess
import tempfile

import numpy as np

import fieldcalc_oracle as fo
from cudalbm_b200 import casefiles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cudalbm_b200", "bin", "fieldCalculate")


def test_oracle_mean_is_the_sequential_float_sum():
    rng = np.random.default_rng(0)
    x = rng.normal(size=3000).astype(np.float32)
    s = np.float32(0.0)
    for v in x:
        s = np.float32(s + v)
    assert fo.spatial_mean(x) == np.float32(s / np.float32(x.size))
    # the reference's float accumulation saturates: 2^25 values of 0.1 give 0.0625
    assert fo.spatial_mean(np.full(1 << 25, 0.1, np.float32)) == np.float32(0.0625)
    assert fo.fmt(np.float32(1.0)) == "1" and fo.fmt(np.float32(0.00012345678)) == "0.000123457"


def test_oracle_nan_block():
    f = np.zeros((3, 8), np.float32)
    f[1, 2] = np.nan
    f[2, 0] = np.inf
    lines = fo.time_block("containsNaN", 7, ["a", "b", "c"], f)
    assert lines == ["Time: 7", "{", "    NaN detected in field b", "    Total number of fields with NaN values: 1",
                     "};", ""]


def case_dir():
    d = tempfile.mkdtemp()
    casefiles.write_case(d, casefiles.CaseSpec(nx=16, ny=8, nz=8, Re=100.0, u_inf=0.05, n_steps=10, save_interval=5,
                                                       info_interval=5))
    return d


def test_executable_without_a_calculation_prints_the_startup_blocks_only():
    r = subprocess.run([EXE], cwd=case_dir(), capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    assert "programControl:" in r.stdout and "latticeMesh:" in r.stdout and "deviceList: [0];" in r.stdout
    lines = r.stdout.splitlines()
    assert not any(s.startswith("Time: ") for s in lines) and "End" not in lines


def test_executable_rejects_the_calculations_it_does_not_provide():
    for kind in ("vorticity", "div[U]"):
        r = subprocess.run([EXE, "-calculationType", kind], cwd=case_dir(), capture_output=True, text=True,
                           timeout=60)
        assert r.returncode == 1 and "is not provided" in r.stderr
    r = subprocess.run([EXE, "-GPU", "x"], cwd=case_dir(), capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "-GPU is not numeric" in r.stderr
