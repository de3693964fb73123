"""Self-check of the FP64 network oracle (CPU): its analytic gradient equals
central finite differences, so it can check the GPU training kernels."""
import numpy as np

from cudalbm_b200 import _lib

import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    net = _lib.MLP()
    for name, size in (("w1", 512), ("b1", 32), ("w2", 1024), ("b2", 32), ("w3", 32)):
        getattr(net, name)[:] = list(rng.normal(0, 0.4, size))
    net.b3, net.out_scale, net.dtau_lo, net.dtau_hi = 0.1, 0.02, -0.01, 0.05
    net.in_scale[:] = [1.0] * 16
    x = rng.normal(0, 1, (64, 16))
    t = rng.normal(0.01, 0.01, 64)
    p = mo.params_of(net)
    g, loss = mo.gradient(p, x, t)
    h = 1e-6
    for name, idx in (("w1", (3, 5)), ("b1", (7,)), ("w2", (11, 2)), ("b2", (30,)), ("w3", (9,))):
        plus = {k: v.copy() for k, v in p.items()}
        minus = {k: v.copy() for k, v in p.items()}
        plus[name][idx] += h
        minus[name][idx] -= h
        fd = (mo.gradient(plus, x, t)[1] - mo.gradient(minus, x, t)[1]) / (2 * h)
        assert abs(fd - g[name][idx]) <= 1e-6 * max(1.0, abs(fd)), name
    plus = dict(p, b3=p["b3"] + h)
    minus = dict(p, b3=p["b3"] - h)
    fd = (mo.gradient(plus, x, t)[1] - mo.gradient(minus, x, t)[1]) / (2 * h)
    assert abs(fd - float(g["b3"])) <= 1e-6 * max(1.0, abs(fd))


def test_oracle_features_shape_and_strain_formula():
    rng = np.random.default_rng(1)
    m = rng.normal(0, 0.01, (10, 50)).astype(np.float32)
    f = mo.features(m, 0.51)
    assert f.shape == (50, 16)
    assert np.array_equal(f[:, :10], m.T)
    s_xy = 3.0 * (m[1].astype(np.float64) * m[2] - m[5]) / (2 * 9.0 * 0.51)
    assert np.allclose(f[:, 11], s_xy, rtol=1e-5, atol=1e-9)
