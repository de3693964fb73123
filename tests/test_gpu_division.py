"""The strain-rate divisions of the step kernel use a correctly rounded
reciprocal and one FMA correction (Markstein) instead of a divide, with an
exact rescaling path for numerators outside [2^-64, 2^64).  This checks, on
the GPU, that the result equals IEEE division bit for bit for every float
numerator (all 2^32 patterns) and the divisors of the benchmarked and tested
cases."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from cudalbm_b200.casefiles import relaxation

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def divlib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("div") / "libdivcheck.so")
    subprocess.run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
                    "-shared", "-I" + os.path.join(ROOT, "cudalbm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cuda", "div_exhaustive.cu"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    L.div_exhaustive.argtypes = [ctypes.c_float, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_uint),
                                 ctypes.POINTER(ctypes.c_ulonglong)]
    return L


CASES = [(0.05, 100.0, 64), (0.05, 1000.0, 256), (0.05, 10000.0, 512), (0.0256, 10000.0, 256), (0.05, 400.0, 24),
         (0.05, 250.0, 24), (0.05, 100.0, 16)]


@pytest.mark.parametrize("u,Re,nx", CASES)
def test_markstein_division_is_ieee_for_all_numerators(divlib, u, Re, nx):
    tau = relaxation(u, Re, nx)[0]
    for d in (np.float32(2.0) * np.float32(4.5) * tau, np.float32(2.0) * np.float32(9.0) * tau):
        bad = ctypes.c_ulonglong()
        first = ctypes.c_uint()
        hist = (ctypes.c_ulonglong * 256)()
        assert divlib.div_exhaustive(float(d), ctypes.byref(bad), ctypes.byref(first), hist) == 0
        unguarded = {e - 127: hist[e] for e in range(256) if hist[e]}
        print(f"d={float(d)!r}: unguarded Markstein mismatches by unbiased exponent {unguarded}")
        assert bad.value == 0, (float(d), bad.value, hex(first.value))
        # the guard window [2^-64, 2^64) holds no unguarded mismatch
        assert all(not (-64 <= e < 64) for e in unguarded), unguarded
