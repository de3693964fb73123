"""Failure detection without a GPU fault: a device wait that nothing
completes gives up after its limit, reports LBM_ERR_TIMEOUT with where it
stopped, and the context keeps working (the next solver step is exact)."""
import time

import numpy as np
import pytest

from cudalbm_b200 import _lib
from cudalbm_b200.solver import Cavity

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports():
    L = _lib.lib()
    t0 = time.perf_counter()
    status = L.lbm_selftest_wait_timeout(0, 1_000_000)  # 1 ms
    dt = time.perf_counter() - t0
    assert status == 4, L.lbm_last_error()
    msg = L.lbm_last_error().decode()
    assert "timed out" in msg and "mbarrier" in msg
    assert dt < 5.0


def test_context_survives_the_timeout():
    L = _lib.lib()
    assert L.lbm_selftest_wait_timeout(0, 500_000) == 4
    with Cavity(19, 16, 16, 16, 100.0, 0.05) as a, Cavity(19, 16, 16, 16, 100.0, 0.05) as b:
        a.init_regions()
        b.init_regions()
        a.step(3)
        b.step(3)
        a.synchronize()
        b.synchronize()
        assert np.array_equal(a.read().view(np.uint32), b.read().view(np.uint32))
