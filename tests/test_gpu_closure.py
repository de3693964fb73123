"""The learned closure's machinery on the GPU.

* training samples: features are the FP32 restatement's, bit for bit;
* training kernels: the gradient of the mean squared error equals the FP64
  oracle's (oracle/mlp_oracle.py) to FP32 accumulation error;
* tensor-core inference (tcgen05, FP16 weights and activations, FP32
  accumulation) equals the oracle evaluated with the same FP16 roundings,
  and the FP32 CUDA-core path equals the plain FP64 network;
* the closure step is the plain step, bit for bit, when the network gives
  dtau = 0 or every input lies outside the training range (the fallback);
* training lowers the loss.
"""
import numpy as np
import pytest

from cudalbm_b200 import _lib
from cudalbm_b200.closure import Trainer, mlp_infer
from cudalbm_b200.solver import Cavity

import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def make_samples(q=27, n=32, steps=40, seed=0, snapshots=2):
    tr = Trainer(capacity=200000)
    with Cavity(q, n, n, n, 400.0, 0.05) as fine, Cavity(q, n // 2, n // 2, n // 2, 400.0, 0.05) as coarse:
        fine.init_regions()
        fine.perturb_velocity(1e-3, seed)
        fine.step(steps)
        states, taus = [], []
        for _ in range(snapshots):
            coarse.filter_from(fine)
            states.append(coarse.read().reshape(10, -1))
            taus.append(coarse.info()["tau"])
            fine.step(2)
            tr.add(coarse, fine, stride=1)
            fine.step(4)
    return tr, states, taus


def random_net(feats, targets, seed=1, scale=0.4):
    rng = np.random.default_rng(seed)
    net = _lib.MLP()
    net.w1[:] = list(rng.normal(0, scale, 512))
    net.b1[:] = list(rng.normal(0, 0.1, 32))
    net.w2[:] = list(rng.normal(0, scale, 1024))
    net.b2[:] = list(rng.normal(0, 0.1, 32))
    net.w3[:] = list(rng.normal(0, scale, 32))
    net.b3 = 0.05
    mean, std = feats.mean(axis=0), feats.std(axis=0)
    net.in_mean[:] = list(mean)
    net.in_scale[:] = list(1.0 / np.where(std > 0, std, 1.0))
    net.in_lo[:] = list(feats.min(axis=0))
    net.in_hi[:] = list(feats.max(axis=0))
    net.out_scale = float(np.sqrt(np.mean(np.clip(targets, -0.002, 0.05) ** 2)) or 1.0)
    net.dtau_lo, net.dtau_hi = -0.002, 0.05
    return net


@pytest.fixture(scope="module")
def samples():
    tr, states, taus = make_samples()
    feats, targ = tr.samples()
    yield tr, feats, targ, states, taus
    tr.close()


def test_sample_features_are_the_fp32_restatement(samples):
    tr, feats, targ, states, taus = samples
    assert len(feats) > 1000 and np.all(np.isfinite(targ))
    ref = np.concatenate([mo.features(s, t) for s, t in zip(states, taus)])
    known = {row.tobytes() for row in ref}
    assert all(row.tobytes() in known for row in feats)


def test_gradient_matches_fp64_oracle(samples):
    tr, feats, targ, _, _ = samples
    net = random_net(feats, targ)
    n = 700
    g, loss = tr.gradient(net, 0, n)
    p = mo.params_of(net)
    ref, ref_loss = mo.gradient(p, feats[:n], targ[:n])
    assert abs(loss - ref_loss) <= 1e-4 * ref_loss
    gp = mo.params_of(g)
    for name in mo.WEIGHTS:
        a, b = np.ravel(gp[name]), np.ravel(ref[name])
        assert np.linalg.norm(a - b) <= 2e-4 * np.linalg.norm(b) + 1e-12, name


def test_inference_tensor_cores_and_fp32_paths(samples):
    _, feats, targ, _, _ = samples
    net = random_net(feats, targ, seed=3, scale=0.5)
    rng = np.random.default_rng(7)
    x = feats[rng.integers(0, len(feats), 1000)]  # 1000 rows: a partial last tile
    p = mo.params_of(net)
    y_tc = mlp_infer(net, x, tensor_cores=True)
    y_32 = mlp_infer(net, x, tensor_cores=False)
    ref16 = mo.forward(p, x, fp16=True)
    ref64 = mo.forward(p, x)
    scale = np.max(np.abs(ref64))
    assert np.max(np.abs(y_32 - ref64)) <= 1e-5 * scale
    assert np.max(np.abs(y_tc - ref16)) <= 2e-3 * scale
    assert np.mean(np.abs(y_tc - ref16)) <= 2e-4 * scale
    # the FP16 operands cost about 3 decimal digits against the FP64 network
    assert np.max(np.abs(y_tc - ref64)) <= 2e-2 * scale


def run_pair(q, net, steps=6, n=(24, 16, 16)):
    with Cavity(q, *n, 300.0, 0.05) as plain, Cavity(q, *n, 300.0, 0.05) as cl:
        for c in (plain, cl):
            c.init_regions()
        cl.set_closure(net)
        plain.step(steps)
        cl.step(steps)
        cl.synchronize()
        return plain.read(), cl.read(), cl.closure_dtau()


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("q", [19, 27])
def test_zero_network_and_fallback_are_the_plain_step(q):
    zero = _lib.MLP()
    zero.in_lo[:] = [-1e30] * 16
    zero.in_hi[:] = [1e30] * 16
    zero.in_scale[:] = [1.0] * 16
    zero.dtau_lo, zero.dtau_hi = -0.01, 0.01
    a, b, dt = run_pair(q, zero)
    assert np.array_equal(bits(a), bits(b)) and np.all(dt == 0.0)
    # a network that would change tau, but no input lies in its range
    off = _lib.MLP()
    off.in_scale[:] = [1.0] * 16
    off.in_lo[:] = [1e29] * 16
    off.in_hi[:] = [1e30] * 16
    off.b3, off.out_scale, off.dtau_lo, off.dtau_hi = 1.0, 0.01, -0.01, 0.05
    a, b, dt = run_pair(q, off)
    assert np.array_equal(bits(a), bits(b)) and np.all(dt == 0.0)


def test_constant_network_sets_dtau_everywhere():
    net = _lib.MLP()
    net.in_lo[:] = [-1e30] * 16
    net.in_hi[:] = [1e30] * 16
    net.in_scale[:] = [1.0] * 16
    net.b3, net.out_scale, net.dtau_lo, net.dtau_hi = 1.0, 0.01, -0.01, 0.05
    a, b, dt = run_pair(27, net, steps=4)
    assert np.allclose(dt, 0.01, rtol=0, atol=1e-6)
    assert not np.array_equal(bits(a), bits(b))  # more viscous interior
    assert np.all(np.isfinite(b))
    # the lid drives the plain run harder than the more viscous one
    assert np.abs(b[1]).sum() != np.abs(a[1]).sum()


def test_training_lowers_the_loss(samples):
    tr, _, _, _, _ = samples
    net, rep = tr.fit(steps=300, batch=2048, lr=3e-3, seed=0)
    assert rep["samples"] == len(tr) and rep["steps"] == 300
    assert rep["loss_last"] < rep["loss_first"]
    assert np.all(np.isfinite(np.array(net.w2)))


def test_samples_and_training_are_reproducible():
    tr1, _, _ = make_samples(q=19, n=32, steps=20, seed=5, snapshots=1)
    tr2, _, _ = make_samples(q=19, n=32, steps=20, seed=5, snapshots=1)
    f1, t1 = tr1.samples()
    f2, t2 = tr2.samples()
    assert np.array_equal(f1.view(np.uint32), f2.view(np.uint32))
    assert np.array_equal(t1.view(np.uint32), t2.view(np.uint32))
    n1, r1 = tr1.fit(steps=50, batch=1024, seed=3)
    n2, r2 = tr2.fit(steps=50, batch=1024, seed=3)
    assert np.array_equal(np.array(n1.w2), np.array(n2.w2)) and r1["loss_last"] == r2["loss_last"]
    tr1.close()
    tr2.close()


def test_closure_range_must_keep_the_viscosity_positive():
    net = _lib.MLP()
    net.in_scale[:] = [1.0] * 16
    with Cavity(19, 16, 16, 16, 300.0, 0.05) as c:
        tau = c.info()["tau"]
        net.dtau_lo, net.dtau_hi = 0.5 - tau, 0.01  # tau + dtau_lo = 0.5
        with pytest.raises(RuntimeError, match="tau \\+ dtau_lo > 0.5"):
            c.set_closure(net)
        net.dtau_lo, net.dtau_hi = 0.02, 0.01
        with pytest.raises(RuntimeError, match="dtau_lo <= dtau_hi"):
            c.set_closure(net)
        net.dtau_lo = 0.5 - tau + 1e-3
        c.set_closure(net)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("nx", [32, 16], ids=["tile32", "tile16"])
def test_fused_network_equals_separate_kernels(samples, q, nx):
    """The closure step with the network inside the step kernel (tcgen05
    MMAs per plane, no dtau array) gives the bits of the separate inference
    kernel followed by the closure step kernel: moments after several steps
    and the dtau field of the last step."""
    _, feats, targ, _, _ = samples
    net = random_net(feats, targ, seed=11, scale=0.5)
    shape = (nx, 16, 24)
    with Cavity(q, *shape, 300.0, 0.05) as a, Cavity(q, *shape, 300.0, 0.05) as b:
        for c in (a, b):
            c.init_regions()
            c.set_closure(net)
        b.closure_fused(False)
        a.step(7)
        b.step(7)
        a.synchronize()
        b.synchronize()
        assert a.info()["tile_x"] == nx
        # one launch per fused step, two per separate step
        assert b.info()["kernel_launches"] - a.info()["kernel_launches"] == 7
        da, db = a.closure_dtau(), b.closure_dtau()
        assert np.count_nonzero(db) > 0  # the network changes tau somewhere
        assert np.array_equal(bits(da), bits(db))
        assert np.array_equal(bits(a.read()), bits(b.read()))
        # a replaced state: both report the field the next step will use
        state = a.read()
        state[1] *= np.float32(0.5)
        for c in (a, b):
            c.write(state)
        da2, db2 = a.closure_dtau(), b.closure_dtau()
        assert np.array_equal(bits(da2), bits(db2)) and not np.array_equal(bits(da2), bits(da))


def test_autotune_picks_the_closure_evaluation_and_keeps_the_state(samples):
    """With a closure set, the autotuner times the closure kernel shapes and
    both evaluations of the network (inside the step kernel, or a separate
    inference kernel), keeps the faster, and leaves the state as it was."""
    _, feats, targ, _, _ = samples
    net = random_net(feats, targ, seed=5, scale=0.5)
    with Cavity(27, 32, 16, 24, 300.0, 0.05) as a, Cavity(27, 32, 16, 24, 300.0, 0.05) as b:
        for c in (a, b):
            c.init_regions()
            c.set_closure(net)
            c.step(3)
        t = b.autotune(3)
        assert t["closure_fused"] in (0, 1) and t["ms_per_step"] > 0
        for c in (a, b):
            c.step(5)
            c.synchronize()
        assert b.info()["step"] == 8
        assert np.array_equal(bits(a.read()), bits(b.read()))


def window_samples(window, q=27, n=32, steps=40):
    """Samples of one snapshot of a perturbed fine run: lbm_trainer_add
    (window 0 here) or lbm_trainer_add_window."""
    tr = Trainer(capacity=200000)
    with Cavity(q, n, n, n, 400.0, 0.05) as fine, Cavity(q, n // 2, n // 2, n // 2, 400.0, 0.05) as coarse:
        fine.init_regions()
        fine.perturb_velocity(1e-3, 0)
        fine.step(steps)
        coarse.filter_from(fine)
        if window == 0:
            fine.step(2)
            tr.add(coarse, fine)
        else:
            tr.add_window(coarse, fine, window)
        fine.synchronize()
        assert fine.info()["step"] == steps + 2 * max(window, 1)
        out = tr.samples()
    tr.close()
    return out


def test_window_targets():
    """A window of one coarse step gives exactly lbm_trainer_add's samples; a
    window of four fits one dtau per node to four transitions (same features
    at the window's start, finite targets that differ)."""
    f0, t0 = window_samples(0)
    f1, t1 = window_samples(1)
    assert len(t0) > 1000
    assert np.array_equal(f0.view(np.uint32), f1.view(np.uint32))
    assert np.array_equal(t0.view(np.uint32), t1.view(np.uint32))
    f4, t4 = window_samples(4)
    assert len(t4) > 1000 and np.all(np.isfinite(t4))
    common = min(len(t0), len(t4))
    assert not np.array_equal(t4[:common], t0[:common])
    assert np.std(t4) < np.std(t0)  # the window averages out transition noise
