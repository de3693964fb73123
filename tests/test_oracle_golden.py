"""The CPU oracle against outputs of the reference solver itself.

The fixtures in tests/golden were written by the reference executables
(oracle/_ref, built from the reference's sources) on a B200; see
tests/golden/make_golden.py.  The reference computes in FP32, the oracle in
FP64, so the two differ by the reference's own rounding: a few ulp per node.
Fields dominated by cancellation (rho-1 and m_zz, both near zero in the
cavity) show relative L2 differences up to ~5e-4 for that reason, while the
absolute per-node difference stays at FP32 rounding level (< 2e-6), except
for rho-1, whose FP32 rounding accumulates a small drift of total mass in the
reference (~4e-6 after 200 steps).
"""
import numpy as np
import pytest

from cudalbm_b200 import casefiles
from helpers import GOLDEN_CASES, lattice_q, load_golden, max_abs, rel_l2, spec_of

from pyoracle import Oracle

REL_L2_TOL = 1e-3   # per moment / function-object component
MAX_ABS_TOL = np.array([1e-5] + [2.5e-6] * 9)  # per node and moment, stored (scaled) units


def run_oracle(meta, precision="f64"):
    s = meta["spec"]
    o = Oracle(lattice_q(meta), s["nx"], s["ny"], s["nz"], s["Re"], s["u_inf"], precision)
    m = o.initial(casefiles.scaled_region_values(spec_of(meta).initial_values()))
    fo = o.new_function_objects(s.get("function_objects", []))
    o.run(m, meta["t"], 0, fo)
    return m, fo


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_oracle_matches_reference_output(name, precision):
    meta, arr = load_golden(name)
    m, fo = run_oracle(meta, precision)
    assert np.all(rel_l2(m, arr["moments"]) < REL_L2_TOL), rel_l2(m, arr["moments"])
    assert np.all(max_abs(m, arr["moments"]) < MAX_ABS_TOL), max_abs(m, arr["moments"])
    for k, v in fo.items():
        assert np.all(rel_l2(v, arr[k]) < REL_L2_TOL), (k, rel_l2(v, arr[k]))


def test_oracle_detects_a_planted_error():
    """A mistake planted in the oracle's output must fail the comparison."""
    meta, arr = load_golden("q19_16c_re100")
    m, _ = run_oracle(meta)
    m[1, 5, 5, 5] += 1e-4  # one node of u
    assert max_abs(m, arr["moments"])[1] > MAX_ABS_TOL[1]
