"""The roundings the step kernel writes out explicitly (lbm_core.cuh) are
the reference's: its strain-rate numerator is 3 * fma(u_a, u_b, -m_ab) and its
kinetic energy sqrtf(fma(w, w, fma(u, u, v*v))) * 0.5
(src/functionObjects/strainRateTensor.cuh:78-82, kineticEnergy.cuh:72-85,
as nvcc contracts them).  Checked on CPU against the reference's own outputs
in the golden fixtures: the stated forms reproduce every sampled S_xx and k
bit for bit, and the other plausible contractions do not."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from cudalbm_b200.casefiles import relaxation
from helpers import load_golden

FORMS = r"""
#include <math.h>
float s_fused(float a, float b, float m) { return 3.0f * fmaf(a, b, -m); }
float s_plain(float a, float b, float m) { volatile float p = a * b; return 3.0f * (p - m); }
float k_ref(float u, float v, float w) { volatile float vv = v * v; return sqrtf(fmaf(w, w, fmaf(u, u, vv))) * 0.5f; }
float k_alt(float u, float v, float w) { volatile float uu = u * u; return sqrtf(fmaf(w, w, fmaf(v, v, uu))) * 0.5f; }
"""


@pytest.fixture(scope="module")
def forms(tmp_path_factory):
    d = tmp_path_factory.mktemp("forms")
    src, lib = d / "forms.c", d / "libforms.so"
    src.write_text(FORMS)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-shared", "-fPIC", str(src), "-o", str(lib), "-lm"], check=True)
    L = ctypes.CDLL(str(lib))
    for f in ("s_fused", "s_plain", "k_ref", "k_alt"):
        getattr(L, f).restype = ctypes.c_float
        getattr(L, f).argtypes = [ctypes.c_float] * 3
    return L


@pytest.mark.parametrize("name", ["q27_16x24x32_fo", "q19_24x16x8_fo"])
def test_strain_rate_and_kinetic_energy_forms(forms, name):
    meta, arr = load_golden(name)
    m, S, k = arr["moments"].reshape(10, -1), arr["S"].reshape(6, -1), arr["k"].reshape(-1)
    s = meta["spec"]
    d = np.float32(2.0) * np.float32(4.5) * np.float32(relaxation(s["u_inf"], s["Re"], s["nx"])[0])
    u, v, w, mxx = m[1], m[2], m[3], m[4]
    idx = np.arange(0, m.shape[1], max(1, m.shape[1] // 2000))

    def hits(fn, args, ref, post=lambda x: x):
        return sum(int(np.float32(post(np.float32(fn(*(float(a[i]) for a in args))))).view(np.uint32)
                       == ref[i].view(np.uint32)) for i in idx)

    assert hits(forms.s_fused, (u, u, mxx), S[0], lambda x: x / d) == len(idx)
    assert hits(forms.s_plain, (u, u, mxx), S[0], lambda x: x / d) < len(idx)
    assert hits(forms.k_ref, (u, v, w), k) == len(idx)
    assert hits(forms.k_alt, (u, v, w), k) < len(idx)
