"""The checked build (cudalbm_b200/lib/liblbm_b200_checked.so, -DLBM_CHECKED).

compute-sanitizer is not available here, so the library is also built with
index checks compiled into its step kernels: every shared-memory index,
global node index and TMA coordinate is verified before use, a failure is
recorded and the access skipped, and the call reports LBM_ERR_STATE.  Every
kernel path is run under it (tests/checked_cases.py) in a child process that
loads the checked library; none may report a failed check, and the results
must be the ordinary library's bit for bit.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "cudalbm_b200", "lib", "liblbm_b200_checked.so")


def test_checked_build_finds_nothing_and_changes_nothing():
    if not os.path.exists(CHECKED):
        pytest.fail("the checked library is not built (python -m cudalbm_b200.build)")
    import checked_cases

    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "checked.npz")
        env = dict(os.environ, LBM_B200_LIBRARY=CHECKED)
        r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_cases.py"), path], env=env,
                           capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
        assert "liblbm_b200_checked.so" in r.stdout
        got = dict(np.load(path))
    want = checked_cases.run_all()
    assert set(got) == set(want)
    for k, w in want.items():
        g = got[k]
        if k.endswith("/mass"):
            np.testing.assert_allclose(g, w, rtol=1e-12, err_msg=k)
            continue
        view = np.uint64 if w.dtype == np.float64 else np.uint32
        assert g.dtype == w.dtype and np.array_equal(g.view(view), w.view(view)), k
