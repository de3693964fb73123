"""fieldCalculate containsNaN / spatialMean on the GPU.

* lbm_field_statistics: NaN counts, the reference's left-to-right float mean
  (bit for bit against oracle/fieldcalc_oracle.py) and the FP64 mean, for
  both layouts, partial last chunks, NaN and infinity;
* the fieldCalculate executable prints, per saved time, the oracle's block;
* its output equals the reference's own fieldCalculate (built from its
  sources into oracle/_ref) line for line from the first time block on.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import fieldcalc_oracle as fo
from cudalbm_b200 import casefiles, lbmbin
from cudalbm_b200.solver import field_statistics

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cudalbm_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")
MOMENTS = ["rho", "u", "v", "w", "m_xx", "m_xy", "m_xz", "m_yy", "m_yz", "m_zz"]


def random_fields(shape, nf=4, seed=0):
    rng = np.random.default_rng(seed)
    f = rng.normal(0.0, 1.0, (nf,) + shape).astype(np.float32)
    f[0] += 1.0  # a density-like field: the float sum loses digits as it grows
    f[1] *= 1e-3
    if nf > 2:
        f[2] = np.float32(0.1)  # constant: the float sum saturates on large meshes
    return f


@pytest.mark.parametrize("shape", [(8, 8, 8), (40, 8, 24), (16, 24, 40), (64, 256, 256)])
@pytest.mark.parametrize("tiled", [False, True])
def test_statistics_match_the_oracle(shape, tiled):
    f = random_fields(shape)
    data = lbmbin.global_to_tiled(f) if tiled else f
    nan, mean_ref, mean = field_statistics(data, shape=shape, tiled=tiled)
    ref = np.array([fo.spatial_mean(x) for x in f], np.float32)
    assert np.array_equal(mean_ref.view(np.uint32), ref.view(np.uint32))
    exact = f.reshape(len(f), -1).astype(np.float64).mean(axis=1)
    assert np.allclose(mean, exact, rtol=1e-12, atol=1e-15)
    assert np.all(nan == 0)


def test_nan_counts_and_infinities():
    shape = (24, 16, 32)
    f = random_fields(shape, nf=5, seed=3)
    f[1].flat[[0, 7, 5000]] = np.nan
    f[3].flat[-1] = np.nan
    f[4].flat[100] = np.inf  # not a NaN
    nan, mean_ref, mean = field_statistics(lbmbin.global_to_tiled(f), shape=shape, tiled=True)
    assert list(nan) == [0, 3, 0, 1, 0]
    assert np.isnan(mean_ref[1]) and np.isinf(mean_ref[4]) and np.isinf(mean[4])
    ok = np.isfinite(f[1])
    assert np.isclose(mean[1], f[1][ok].astype(np.float64).sum() / f[1].size, rtol=1e-12)
    assert [fo.contains_nan(x) for x in f] == [False, True, False, True, False]


def test_statistics_argument_errors():
    f = np.zeros((2, 8, 8, 8), np.float32)
    with pytest.raises(RuntimeError, match="multiples of 8"):
        field_statistics(f.reshape(2, -1)[:, :500], shape=(5, 10, 10), tiled=True)
    with pytest.raises(RuntimeError, match="device ordinal"):
        field_statistics(f, device=999)


def solver_case(nx=32, ny=24, nz=16, steps=41, save=20):
    spec = casefiles.CaseSpec(nx=nx, ny=ny, nz=nz, Re=300.0, u_inf=0.05, n_steps=steps, save_interval=save,
                              info_interval=save)
    case = tempfile.mkdtemp()
    casefiles.write_case(case, spec)
    subprocess.run([os.path.join(BIN, "momentBasedD3Q19"), "-GPU", "0"], cwd=case, capture_output=True,
                   timeout=300, check=True)
    return case, spec


def calculate(exe, case, *args):
    r = subprocess.run([exe, *args], cwd=case, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    first = next((i for i, s in enumerate(lines) if s.startswith("Time: ")), None)
    return lines[first:] if first is not None else lines[lines.index("End"):]


def expected(case, kind, latest=False):
    files = sorted((f for f in os.listdir(case) if f.endswith(".LBMBin")),
                   key=lambda f: int(f.rsplit("_", 1)[1].split(".")[0]))
    if latest:
        files = files[-1:]
    out = []
    for name in files:
        ff = lbmbin.read(os.path.join(case, name))
        out += fo.time_block(kind, ff.time_step, ff.names, ff.data)
    return out + ["End", ""]


def inject(case, t, field_values):
    """Rewrite <case>_<t>.LBMBin with values[field] = [(flat index, value), ...]."""
    path = [os.path.join(case, f) for f in os.listdir(case) if f.endswith(f"_{t}.LBMBin")][0]
    ff = lbmbin.read(path)
    data = ff.data.copy()
    for name, items in field_values.items():
        for i, v in items:
            data[ff.names.index(name)].flat[i] = v
    lbmbin.write(path, ff.names, data, ff.time_step)


def test_executable_prints_the_oracle_blocks():
    case, _ = solver_case()
    exe = os.path.join(BIN, "fieldCalculate")
    for kind in ("spatialMean", "containsNaN"):
        assert calculate(exe, case, "-calculationType", kind) == expected(case, kind)
        assert calculate(exe, case, "-calculationType", kind, "-latestTime") == expected(case, kind, latest=True)
    inject(case, 20, {"u": [(5, np.nan)], "m_xy": [(0, np.nan), (99, np.nan)], "w": [(3, np.inf)]})
    got = calculate(exe, case, "-calculationType", "containsNaN", "-GPU", "0")
    assert got == expected(case, "containsNaN")
    assert "    NaN detected in field u" in got and "    Total number of fields with NaN values: 2" in got
    assert "    No NaN values detected in any field." in got  # the other saved times
    shutil.rmtree(case)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "fieldCalculate")), reason="reference fieldCalculate not built")
def test_executable_output_identical_to_reference_fieldcalculate():
    case, _ = solver_case(nx=64, ny=48, nz=40, steps=61, save=30)
    ours, ref = os.path.join(BIN, "fieldCalculate"), os.path.join(REF, "fieldCalculate")
    # -GPU 0 given: the reference makes -GPU optional only when argv[0] is the
    # bare name "fieldCalculate" (inputControl.cuh:218), not a path
    runs = [("-GPU", "0", "-calculationType", "spatialMean"), ("-GPU", "0", "-calculationType", "containsNaN"),
            ("-GPU", "0", "-calculationType", "spatialMean", "-latestTime")]
    for args in runs:
        assert calculate(ours, case, *args) == calculate(ref, case, *args), args
    inject(case, 30, {"v": [(17, np.nan)], "m_zz": [(0, np.nan)], "rho": [(1, np.inf)]})
    for args in runs[:2]:
        a, b = calculate(ours, case, *args), calculate(ref, case, *args)
        assert a == b, args
    assert "    NaN detected in field m_zz" in a
    shutil.rmtree(case)
