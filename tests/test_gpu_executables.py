"""The momentBasedD3Q19 / momentBasedD3Q27 executables as drop-in
replacements: same case directory, same command line, and every .LBMBin file
identical byte for byte to what the reference executables write."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from cudalbm_b200 import casefiles, lbmbin

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cudalbm_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def run(exe, case, check=True):
    return subprocess.run([exe, "-GPU", "0"], cwd=case, capture_output=True, text=True, timeout=600, check=check)


def lbmbin_files(d):
    return sorted(f for f in os.listdir(d) if f.endswith(".LBMBin"))


@pytest.mark.parametrize("q", [19, 27])
def test_outputs_identical_to_reference_executable(q):
    if not os.path.exists(os.path.join(REF, f"momentBasedD3Q{q}")):
        pytest.skip("reference executables not built")
    spec = casefiles.CaseSpec(nx=32, ny=24, nz=16, Re=300.0, u_inf=0.05, n_steps=61, save_interval=20,
                              info_interval=10, function_objects=("S", "SMean", "k", "kMean", "momentsMean"))
    ours, ref = tempfile.mkdtemp(), tempfile.mkdtemp()
    casefiles.write_case(ours, spec)
    casefiles.write_case(ref, spec)
    out = run(os.path.join(BIN, f"momentBasedD3Q{q}"), ours)
    run(os.path.join(REF, f"momentBasedD3Q{q}"), ref)
    files = lbmbin_files(ref)
    assert len(files) == 4 * 6 and lbmbin_files(ours) == files
    for f in files:
        a = open(os.path.join(ours, f), "rb").read()
        b = open(os.path.join(ref, f), "rb").read()
        assert a == b, f
    assert "Time: 60" in out.stdout and "MLUPS" in out.stdout


def test_restart_continues_like_one_run():
    spec = casefiles.CaseSpec(nx=16, ny=16, nz=24, Re=200.0, u_inf=0.05, n_steps=41, save_interval=20,
                              info_interval=20)
    one, two = tempfile.mkdtemp(), tempfile.mkdtemp()
    casefiles.write_case(one, spec)
    casefiles.write_case(two, casefiles.CaseSpec(**{**spec.__dict__, "n_steps": 21}))
    exe = os.path.join(BIN, "momentBasedD3Q19")
    run(exe, one)
    run(exe, two)
    casefiles.write_case(two, spec)  # extend nTimeSteps, keep lidDrivenCavity_20.LBMBin
    out = run(exe, two)
    assert "latestTime = 20" in out.stdout
    a = lbmbin.read(os.path.join(one, "lidDrivenCavity_40.LBMBin")).data
    b = lbmbin.read(os.path.join(two, "lidDrivenCavity_40.LBMBin")).data
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_command_line_and_case_errors():
    exe = os.path.join(BIN, "momentBasedD3Q19")
    d = tempfile.mkdtemp()
    casefiles.write_case(d, casefiles.CaseSpec(nx=12, ny=16, nz=16, Re=100.0, u_inf=0.05, n_steps=2,
                                               save_interval=1, info_interval=1))
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True)
    assert r.returncode != 0 and "-GPU argument is mandatory" in r.stderr
    r = run(exe, d, check=False)
    assert r.returncode != 0 and "multiples of 8" in r.stderr
    os.remove(os.path.join(d, "latticeMesh"))
    r = run(exe, d, check=False)
    assert r.returncode != 0 and "latticeMesh file not opened" in r.stderr


FO_ALL = ("S", "SMean", "k", "kMean", "momentsMean")
FO_PREFIXES = ("lidDrivenCavity", "S", "SMean", "k", "kMean", "momentsMean")


def restart_pair(q, opts):
    """Run 0..40 in one go, and 0..20 then a restart to 40, with the same
    b200Options; returns the two case directories."""
    spec = casefiles.CaseSpec(nx=16, ny=16, nz=24, Re=200.0, u_inf=0.05, n_steps=41, save_interval=20,
                              info_interval=20, function_objects=FO_ALL, extra_files=opts)
    one, two = tempfile.mkdtemp(), tempfile.mkdtemp()
    casefiles.write_case(one, spec)
    casefiles.write_case(two, casefiles.CaseSpec(**{**spec.__dict__, "n_steps": 21}))
    exe = os.path.join(BIN, f"momentBasedD3Q{q}")
    run(exe, one)
    run(exe, two)
    casefiles.write_case(two, spec)  # extend nTimeSteps, keep the files of t = 20
    out = run(exe, two)
    assert "latestTime = 20" in out.stdout
    return one, two


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("precision", [32, 64])
def test_restart_with_restored_means_continues_like_one_run(q, precision):
    """b200Options `restoreMeans 1;`: the running means (FP32 or FP64
    accumulators) and S/k saved at the restart time are read back, so every
    file of the restarted run -- moments and all five function objects, at the
    restart step and at the end -- is byte-identical to the uninterrupted run's."""
    one, two = restart_pair(q, {"b200Options": f"meanPrecision {precision};\nrestoreMeans 1;\n"})
    for t in (20, 40):
        for p in FO_PREFIXES:
            f = f"{p}_{t}.LBMBin"
            assert open(os.path.join(one, f), "rb").read() == open(os.path.join(two, f), "rb").read(), f
    if precision == 64:
        h = lbmbin.read(os.path.join(two, "SMean_40.LBMBin"))
        assert h.data.dtype == np.float64


def test_restart_without_restored_means_keeps_the_reference_behaviour():
    """Default (the reference's rule): the moments continue exactly, the
    running means restart from zero with 1/(t+1) at the absolute step."""
    one, two = restart_pair(19, {})
    a = lbmbin.read(os.path.join(one, "lidDrivenCavity_40.LBMBin")).data
    b = lbmbin.read(os.path.join(two, "lidDrivenCavity_40.LBMBin")).data
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    ma = lbmbin.read(os.path.join(one, "kMean_40.LBMBin")).data
    mb = lbmbin.read(os.path.join(two, "kMean_40.LBMBin")).data
    assert not np.array_equal(ma, mb)
    # after the restart the means hold only steps 20..39, weighted by 1/(t+1)
    assert np.abs(mb).max() < np.abs(ma).max()


@pytest.mark.parametrize("q", [19, 27])
def test_autotuned_run_writes_the_same_files(q):
    """b200Options `autotune 1;` (the default from 1000 steps on) times the
    kernel shapes on the run's own state before the loop; the files are
    those of the default shape, byte for byte."""
    spec = casefiles.CaseSpec(nx=32, ny=32, nz=40, Re=500.0, u_inf=0.05, n_steps=41, save_interval=20,
                              info_interval=20, function_objects=("S", "SMean", "k", "kMean"))
    plain, tuned = tempfile.mkdtemp(), tempfile.mkdtemp()
    for d, flag in ((plain, 0), (tuned, 1)):
        casefiles.write_case(d, spec)
        with open(os.path.join(d, "b200Options"), "w") as fh:
            fh.write(f"autotune {flag};\n")
        out = run(os.path.join(BIN, f"momentBasedD3Q{q}"), d)
        assert "autotune skipped" not in out.stderr
    files = lbmbin_files(plain)
    assert files and lbmbin_files(tuned) == files
    for f in files:
        assert open(os.path.join(plain, f), "rb").read() == open(os.path.join(tuned, f), "rb").read(), f
