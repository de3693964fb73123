"""fieldConvert: .LBMBin -> VTS, whole fields and cut planes (CPU).

The cut plane of the drop-in executable reproduces the reference's arithmetic
(applications/fieldConvert/fieldConvert.cuh:236-326), including its weight
coordinate - floor(index); the expectations below restate it in float32
numpy and must match bit for bit.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from cudalbm_b200 import casefiles, lbmbin
from helpers import ROOT, read_vts

EXE = os.path.join(ROOT, "cudalbm_b200", "bin", "fieldConvert")
NX, NY, NZ = 16, 8, 24


def make_case(tmp_path, times=(0, 5), prefix=None, names=casefiles.MOMENT_NAMES, seed=0):
    spec = casefiles.CaseSpec(nx=NX, ny=NY, nz=NZ, Re=100.0, u_inf=0.05, n_steps=10, save_interval=5,
                              info_interval=5)
    casefiles.write_case(str(tmp_path), spec)
    rng = np.random.default_rng(seed)
    data = {}
    for t in times:
        a = rng.standard_normal((len(names), NZ, NY, NX)).astype(np.float32)
        lbmbin.write(str(tmp_path / f"{prefix or 'lidDrivenCavity'}_{t}.LBMBin"), list(names), a, t)
        data[t] = a
    return data


def run(tmp_path, *args):
    return subprocess.run([EXE, *args], cwd=tmp_path, capture_output=True, text=True, timeout=60)


def reference_cut(a, axis, coord):
    """The reference's cut plane in float32: a is [var][z][y][x]."""
    n = a.shape[3 - axis]
    f32 = np.float32
    index = f32(n - 1) * (f32(coord) * f32(1.0))
    i0, i1 = int(np.floor(index)), int(np.ceil(index))
    w = f32(coord) - f32(i0)
    take = lambda i: np.take(a, i, axis=3 - axis)
    return (f32(1) - w) * take(i0) + w * take(i1)


@pytest.mark.skipif(not os.path.exists(EXE), reason="fieldConvert not built")
def test_whole_fields_to_vts(tmp_path):
    data = make_case(tmp_path)
    r = run(tmp_path, "-fileType", "vts")
    assert r.returncode == 0, r.stderr
    for t, a in data.items():
        extent, arrays, points = read_vts(tmp_path / "postProcess" / f"lidDrivenCavity_{t}.vts")
        assert extent == [0, NX - 1, 0, NY - 1, 0, NZ - 1]
        assert list(arrays) == list(casefiles.MOMENT_NAMES)
        for k, name in enumerate(casefiles.MOMENT_NAMES):
            assert np.array_equal(arrays[name], a[k].ravel())
        assert points.shape == (NX * NY * NZ, 3)
        assert np.allclose(points[NX - 1], [1.0, 0.0, 0.0]) and np.allclose(points[-1], [1.0, 1.0, 1.0])
    assert "writeStatus: success" in r.stdout


@pytest.mark.skipif(not os.path.exists(EXE), reason="fieldConvert not built")
@pytest.mark.parametrize("arg,axis,coord", [("x=0", 0, 0.0), ("y=1", 1, 1.0), ("z=0.5", 2, 0.5),
                                            ("y=0.5", 1, 0.5), ("x=0.25", 0, 0.25)])
def test_cut_planes_match_reference_arithmetic(tmp_path, arg, axis, coord):
    data = make_case(tmp_path, times=(5,))
    r = run(tmp_path, "-fileType", "vts", "-cutPlane", arg, "-latestTime")
    assert r.returncode == 0, r.stderr
    extent, arrays, points = read_vts(tmp_path / "postProcess" / f"lidDrivenCavityCutPlane_{arg}_5.vts")
    dims = [NX, NY, NZ]
    dims[axis] = 1
    assert extent == [0, dims[0] - 1, 0, dims[1] - 1, 0, dims[2] - 1]
    expect = reference_cut(data[5], axis, coord)
    for k, name in enumerate(casefiles.MOMENT_NAMES):
        assert np.array_equal(arrays[name].view(np.uint32), expect[k].ravel().view(np.uint32)), name
    assert np.all(points[:, axis] == 0.0)


@pytest.mark.skipif(not os.path.exists(EXE), reason="fieldConvert not built")
def test_custom_field_and_errors(tmp_path):
    names = ["S_xx", "S_xy", "S_xz", "S_yy", "S_yz", "S_zz"]
    data = make_case(tmp_path, times=(3,), prefix="S", names=names)
    r = run(tmp_path, "-fileType", "vts", "-fieldName", "S")
    assert r.returncode == 0, r.stderr
    _, arrays, _ = read_vts(tmp_path / "postProcess" / "S_3.vts")
    assert np.array_equal(arrays["S_yz"], data[3][4].ravel())
    r = run(tmp_path, "-fileType", "vtu")
    assert r.returncode != 0 and "Supported formats are: vts" in r.stderr
    r = run(tmp_path, "-fileType", "vts", "-fieldName", "nope")
    assert r.returncode != 0 and "-fieldName" in r.stderr
    r = run(tmp_path, "-fileType", "vts", "-cutPlane", "q=0.5")
    assert r.returncode != 0
    r = run(tmp_path, "-fileType", "vts", "-fieldName", "S", "-cutPlane", "x=1.5")
    assert r.returncode != 0 and "outside" in r.stderr
    empty = tmp_path / "empty"
    empty.mkdir()
    for f in ("programControl", "latticeMesh"):
        shutil.copy(tmp_path / f, empty / f)
    r = run(empty, "-fileType", "vts")
    assert r.returncode != 0 and "LBMBin" in r.stderr
