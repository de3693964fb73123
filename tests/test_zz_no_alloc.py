"""lbm_reduce_moments_noalloc: the global sums of lbm_reduce for callers that
must not allocate device memory (a framework whose caching allocator owns the
GPU, a monitor of buffers it does not own).  It reads a caller-owned device
array and keeps its scratch in a fixed device array of the library.

This file is collected last on purpose, and each test creates everything it
uses, so it passes alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from cudalbm_b200 import _lib
from cudalbm_b200.solver import Cavity

pytestmark = pytest.mark.gpu


def noalloc(ptr, nodes):
    out = (ctypes.c_double * 3)()
    _lib.check(_lib.lib().lbm_reduce_moments_noalloc(ctypes.c_void_p(ptr), nodes, out, None))
    return np.array(out[:])


def test_matches_lbm_reduce_on_two_calls_in_a_row():
    import torch

    with Cavity(19, 48, 32, 24, 300.0, 0.05) as c:
        c.init_regions()
        c.step(25)
        c.synchronize()
        ref = c.reduce()  # the existing entry point, on the handle's own buffers
        host = c.read("moments")
    nodes = 48 * 32 * 24
    dev = torch.from_numpy(np.ascontiguousarray(host).reshape(-1)).to("cuda:0")  # caller-owned device copy
    torch.cuda.synchronize()
    first = noalloc(dev.data_ptr(), nodes)
    second = noalloc(dev.data_ptr(), nodes)
    expect = np.array([ref["mass"], ref["kinetic_energy"], ref["nonfinite"]])
    np.testing.assert_allclose(first, expect, rtol=1e-12)
    assert first[2] == 0
    assert np.array_equal(first, second)  # fixed summation order: same bits every call


def test_counts_nonfinite_values_and_rejects_oversized_input():
    import torch

    nodes = 64 * 64 * 8
    dev = torch.zeros(10 * nodes, dtype=torch.float32, device="cuda:0")
    dev[3 * nodes + 17] = float("nan")
    dev[9 * nodes + 5] = float("inf")
    torch.cuda.synchronize()
    r = noalloc(dev.data_ptr(), nodes)
    assert r[0] == nodes and r[2] == 2
    # sizes beyond the fixed scratch are refused before any device work
    out = (ctypes.c_double * 3)()
    st = _lib.lib().lbm_reduce_moments_noalloc(ctypes.c_void_p(dev.data_ptr()), (1 << 30) + 1, out, None)
    assert st == 1 and b"fixed scratch limit" in _lib.lib().lbm_last_error()
