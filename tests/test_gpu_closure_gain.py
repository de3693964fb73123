"""What the trained network gains over the method without it (GPU).

Reduced closure studies (cudalbm_b200/closure_study.py): D3Q27 cavity on a
32^3 grid (Re 604; 5,000 coarse steps) and on a 64^3 grid (Re 1227; 10,000
coarse steps, the largest that fits the test budget: about a minute) at the
coarse relaxation time 0.5077, each trained on eight perturbed runs at twice
the resolution, shrink factor calibrated on a ninth, measured against the
unperturbed fine run box-filtered 2:1 (and sampled at the coarse nodes).
Samples and training are deterministic, so the numbers repeat.
"""
import json
import os

import numpy as np
import pytest

from cudalbm_b200.closure_study import run_study

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(32, 5000), (64, 10000)], ids=["32", "64"])
def study(request):
    nc, steps = request.param
    r = run_study(nc=nc, coarse_steps=steps, log=lambda s: None)
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
    # the clamp bounds are float32 values (float32(0.05) > 0.05)
    lo, hi = (float(np.float32(v)) for v in study["config"]["dtau_range"])
    assert lo <= study["dtau"]["mean"] <= hi and study["dtau"]["max"] <= hi
    assert study["dtau"]["nonzero_fraction"] > 0.0


def test_learned_closure_lowers_the_final_centreline_error(study):
    T = study["config"]["coarse_steps"]
    plain, learned = study["plain"][T], study["learned"][T]
    assert learned["centreline_box"] < plain["centreline_box"]
    assert learned["centreline_pos"] < plain["centreline_pos"]
