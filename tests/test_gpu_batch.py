"""Batched cavities: one persistent launch per step over many meshes.

Every cavity of a batch must compute exactly the bits it computes alone
(same scheme, same expressions; only the assignment of tiles to CTAs
differs), whatever the kernel shape, the z-chunks chosen per size class, an
odd number of steps (graph replays plus one direct launch) or a cavity
stepped on its own in between.
"""
import numpy as np
import pytest

from cudalbm_b200 import _lib, casefiles
from cudalbm_b200.solver import Batch, Cavity

pytestmark = pytest.mark.gpu

SPECS19 = [dict(lattice=19, nx=32, ny=32, nz=32, Re=150.0),
           dict(lattice=19, nx=48, ny=48, nz=48, Re=700.0),
           dict(lattice=19, nx=24, ny=16, nz=8, Re=100.0),
           dict(lattice=19, nx=64, ny=40, nz=24, Re=1999.0),
           dict(lattice=19, nx=32, ny=32, nz=32, Re=1200.0)]
SPECS27 = [dict(lattice=27, nx=32, ny=32, nz=32, Re=400.0),
           dict(lattice=27, nx=48, ny=16, nz=40, Re=1000.0),
           dict(lattice=27, nx=16, ny=24, nz=32, Re=100.0)]


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def alone(sp, steps):
    with Cavity(sp["lattice"], sp["nx"], sp["ny"], sp["nz"], sp["Re"], sp.get("u_inf", 0.05)) as c:
        c.init_regions()
        c.step(steps)
        c.synchronize()
        return c.read()


@pytest.mark.parametrize("specs", [SPECS19, SPECS27], ids=["d3q19", "d3q27"])
def test_batch_is_bitwise_equal_to_single_cavities(specs):
    with Batch(specs) as b:
        b.init_regions()
        b.step(5)  # two graph replays and one direct launch
        b.step(4)
        b.synchronize()
        info = b.info()
        assert info["cavities"] == len(specs) and info["step"] == 9
        assert info["graph_launches"] == 4 and info["kernel_launches"] == 9
        for i, sp in enumerate(specs):
            assert b[i].info()["step"] == 9
            assert np.array_equal(bits(b[i].read()), bits(alone(sp, 9))), i


def test_batch_shapes_and_chunks_do_not_change_results():
    ref = [alone(sp, 6) for sp in SPECS19]
    with Batch(SPECS19) as b:
        b.init_regions()
        tuned = b.autotune(trial_steps=2)
        assert tuned["candidates"] >= 6 and tuned["size_classes"] == 4
        b.step(6)
        b.synchronize()
        for i in range(len(SPECS19)):
            assert np.array_equal(bits(b[i].read()), bits(ref[i])), i


def test_cavity_stepped_alone_inside_a_batch():
    with Batch(SPECS19[:3]) as b:
        b.init_regions()
        b[1].step(1)        # its own kernel, on the batch stream
        b.step(2)
        b[0].step(3)
        b.step(1)
        b.synchronize()
        counts = [6, 4, 3]
        for i, n in enumerate(counts):
            assert b[i].info()["step"] == n
            assert np.array_equal(bits(b[i].read()), bits(alone(SPECS19[i], n))), i


def test_batch_autotune_restores_states():
    with Batch(SPECS27) as b:
        b.init_regions()
        b.step(3)
        b.synchronize()
        before = [b[i].read() for i in range(len(SPECS27))]
        b.autotune(trial_steps=2)
        info = b.info()
        assert info["step"] == 3 and info["graph_launches"] == 1
        for i in range(len(SPECS27)):
            assert b[i].info()["step"] == 3
            assert np.array_equal(bits(b[i].read()), bits(before[i]))


def test_batch_members_cannot_be_destroyed_alone():
    with Batch(SPECS19[:2]) as b:
        h = ctypes_handle(b, 0)
        assert _lib.lib().lbm_destroy(h) == 7  # LBM_ERR_STATE
        with pytest.raises(_lib.LBMError):
            _lib.check(_lib.lib().lbm_batch_cavity(b._b, 2, None))


def ctypes_handle(b, i):
    import ctypes

    h = ctypes.c_void_p()
    _lib.check(_lib.lib().lbm_batch_cavity(b._b, i, ctypes.byref(h)))
    return h


def test_seeded_64_cavity_batch_runs_and_conserves_mass():
    specs = casefiles.random_cavities(64, seed=0)
    with Batch(specs) as b:
        b.init_regions()
        m0 = [b[i].reduce()["mass"] for i in range(len(b))]
        b.step(20)
        b.synchronize()
        info = b.info()
        assert info["nodes"] == sum(s["nx"] ** 3 for s in specs)
        for i in range(len(b)):
            r = b[i].reduce()
            assert r["nonfinite"] == 0
            assert abs(r["mass"] - m0[i]) / m0[i] < 1e-3
        # spot-check two cavities bitwise against solo runs
        for i in (0, 63):
            assert np.array_equal(bits(b[i].read()), bits(alone(specs[i], 20))), i
