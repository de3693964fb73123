"""fieldConvert and cut planes on real solver output (GPU).

* The drop-in fieldConvert writes the same .vts files, byte for byte, as the
  reference's own fieldConvert (built from its sources into oracle/_ref; it
  needs a GPU to start) on a case directory produced by our solver.
* lbm_cut_plane, evaluated on the device from the live state, equals linear
  interpolation of the read-back fields computed in float32 on the host.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from cudalbm_b200 import casefiles
from cudalbm_b200.solver import Cavity

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cudalbm_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def convert(exe, case, *args):
    return subprocess.run([exe, "-GPU", "0", *args], cwd=case, capture_output=True, text=True, timeout=300,
                          check=True)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "fieldConvert")), reason="reference fieldConvert not built")
def test_vts_files_identical_to_reference_fieldconvert():
    spec = casefiles.CaseSpec(nx=32, ny=24, nz=16, Re=300.0, u_inf=0.05, n_steps=41, save_interval=20,
                              info_interval=20, function_objects=("S", "k"))
    case = tempfile.mkdtemp()
    casefiles.write_case(case, spec)
    subprocess.run([os.path.join(BIN, "momentBasedD3Q19"), "-GPU", "0"], cwd=case, capture_output=True,
                   timeout=300, check=True)
    runs = [(), ("-cutPlane", "y=0.5"), ("-cutPlane", "x=0"), ("-cutPlane", "z=1"), ("-latestTime",),
            ("-fieldName", "S"), ("-fieldName", "k", "-cutPlane", "y=0.25")]
    for args in runs:
        ours, ref = tempfile.mkdtemp(), tempfile.mkdtemp()
        for d in (ours, ref):
            shutil.rmtree(d)
            shutil.copytree(case, d)
        convert(os.path.join(BIN, "fieldConvert"), ours, "-fileType", "vts", *args)
        convert(os.path.join(REF, "fieldConvert"), ref, "-fileType", "vts", *args)
        files = sorted(os.listdir(os.path.join(ref, "postProcess")))
        assert files and sorted(os.listdir(os.path.join(ours, "postProcess"))) == files, args
        for f in files:
            a = open(os.path.join(ours, "postProcess", f), "rb").read()
            b = open(os.path.join(ref, "postProcess", f), "rb").read()
            assert a == b, (args, f)


def host_cut(a, axis, pos):
    """Linear interpolation in float32 between the bracketing node planes."""
    f32 = np.float32
    n = a.shape[3 - axis]
    index = f32(n - 1) * f32(pos)
    i0, i1 = int(np.floor(index)), int(np.ceil(index))
    w = index - f32(i0)
    take = lambda i: np.take(a, i, axis=3 - axis)
    return (f32(1) - w) * take(i0) + w * take(i1)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_cut_plane_on_device(storage):
    with Cavity(19, 32, 24, 16, 400.0, 0.05, function_objects=("S", "kMean"), mean_bits=64, storage=storage) as c:
        c.init_regions()
        c.step(30)
        c.synchronize()
        m = c.read()
        for axis, pos in [(0, 0.5), (1, 0.0), (1, 1.0), (2, 0.3), (0, 0.77)]:
            got = c.cut_plane(axis, pos)
            want = host_cut(m, axis, pos)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (axis, pos)
        s = c.read("S")
        assert np.array_equal(c.cut_plane(2, 0.5, "S").view(np.uint32), host_cut(s, 2, 0.5).view(np.uint32))
        km = c.read("kMean", dtype=np.float64).astype(np.float32)
        assert np.array_equal(c.cut_plane(1, 0.6, "kMean").view(np.uint32), host_cut(km, 1, 0.6).view(np.uint32))
        from cudalbm_b200 import _lib

        with pytest.raises(_lib.LBMError):
            c.cut_plane(0, 1.5)
