"""What the trained network gains over the method without it (GPU).

A reduced closure study (cudalbm_b200/closure_study.py): D3Q27 cavity on a
32^3 grid at the coarse relaxation time 0.5077 (Re 604), trained on eight
perturbed 64^3 runs, shrink factor calibrated on a ninth, measured against the
unperturbed 64^3 run box-filtered 2:1 (and sampled at the coarse nodes).
Samples and training are deterministic, so the numbers below repeat.
"""
import json
import os

import pytest

from cudalbm_b200.closure_study import run_study

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def study():
    r = run_study(nc=32, coarse_steps=5000, log=lambda s: None)
    out = os.environ.get("LBM_B200_STUDY_JSON")
    if out:
        with open(out, "w") as fh:
            json.dump(r, fh, indent=1, default=float)
    return r


def test_network_learns_the_targets(study):
    t = study["training"]
    assert t["samples"] > 100000
    assert t["loss_last"] < 0.5 * t["loss_first"]
    assert t["r2_held_out"] > 0.8
    lo, hi = study["config"]["dtau_range"]
    assert lo <= study["dtau"]["mean"] <= hi and study["dtau"]["max"] <= hi
    assert study["dtau"]["nonzero_fraction"] > 0.0


def test_learned_closure_lowers_the_final_centreline_error(study):
    T = study["config"]["coarse_steps"]
    plain, learned = study["plain"][T], study["learned"][T]
    assert learned["centreline_box"] < plain["centreline_box"]
    assert learned["centreline_pos"] < plain["centreline_pos"]
