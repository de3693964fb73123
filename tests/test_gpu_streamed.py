"""lbm_run_streamed: a whole job between host buffers with the copies
overlapping the steps (z-slabs of each step shifted down by the step index;
a job longer than 32 steps skews only its first and last 16 steps).

The slab launches update the same nodes with the same arithmetic as whole-mesh
launches, so moments and function objects must equal those of
lbm_write_fields + lbm_step(n) + lbm_read_fields bit for bit, for every slab
height, z-chunk and step count (fewer and more steps than a slab has planes),
and the handle must continue from the same state afterwards.  The per-step
monitor sums are FP64 atomics in a different order: equal to 1e-12 relative.
"""
import numpy as np
import pytest

from cudalbm_b200 import _lib
from cudalbm_b200.solver import NVARS, Cavity

pytestmark = pytest.mark.gpu

LBM_ERR_ARG, LBM_ERR_STATE = 1, 7


def bits_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    view = np.uint64 if a.dtype == np.float64 else np.uint32
    return a.dtype == b.dtype and np.array_equal(a.view(view), b.view(view))


def prepared(q, shape, fo, mean_bits, warm):
    nx, ny, nz = shape
    c = Cavity(q, nx, ny, nz, 400.0, 0.05, function_objects=fo, mean_bits=mean_bits)
    c.init_regions()
    c.step(warm)
    c.synchronize()
    return c


_KEEP = []  # owners of the page-locked buffers handed out below (freed with the process)


def pinned(shape, dtype):
    p = _lib.PinnedArray(shape, dtype)
    _KEEP.append(p)
    return p.array


def out_arrays(c, fo, mean_bits):
    nz, ny, nx = c.shape
    sets = ("moments",) + tuple(fo)
    return {s: pinned((NVARS[s], nz, ny, nx), np.float64 if (mean_bits == 64 and "Mean" in s) else np.float32)
            for s in sets}


CASES = [
    # lattice, mesh, function objects, mean bits, warm-up steps, steps, slab, z-chunk
    (27, (40, 48, 72), ("S", "SMean", "k", "kMean"), 32, 30, 5, 16, 4),
    (27, (64, 64, 64), ("S", "SMean", "k", "kMean"), 32, 12, 23, 8, 3),
    (19, (64, 32, 56), (), 32, 40, 17, 16, 16),
    (19, (32, 32, 40), ("S", "SMean", "k", "kMean", "momentsMean"), 64, 20, 9, 4, 2),
    (27, (32, 32, 64), ("k",), 32, 10, 3, 128, 0),
    (19, (32, 40, 48), (), 32, 5, 1, 0, 0),
    # long jobs: skewed first and last 16 steps around whole-mesh steps
    (19, (32, 32, 48), ("S", "SMean", "k", "kMean"), 32, 5, 41, 8, 4),
    (27, (32, 40, 64), (), 32, 3, 70, 16, 0),
]


@pytest.mark.parametrize("q,shape,fo,mean_bits,warm,n,slab,zc", CASES)
def test_streamed_job_equals_step_loop(q, shape, fo, mean_bits, warm, n, slab, zc):
    a = prepared(q, shape, fo, mean_bits, warm)
    b = prepared(q, shape, fo, mean_bits, warm)
    try:
        state = pinned((10,) + a.shape, np.float32)
        a.read("moments", out=state)
        # reference path: upload, n monitored steps, download
        a.write(state)
        mon_a = a.step_monitored(n)
        a.synchronize()
        ref = {s: a.read(s, dtype=np.float64 if (mean_bits == 64 and "Mean" in s) else np.float32)
               for s in ("moments",) + tuple(fo)}
        # streamed job
        outs = out_arrays(b, fo, mean_bits)
        for arr in outs.values():
            arr[...] = np.nan  # every node must be written
        mon_b = pinned((n,), np.dtype(_lib.MONITOR_DTYPE))
        b.run_streamed(state, n, outs, monitor=mon_b, slab=slab, z_chunk=zc)
        for s, r in ref.items():
            assert bits_equal(outs[s], r), (s, np.argwhere(outs[s] != r)[:4])
        np.testing.assert_allclose(mon_b["mass"], mon_a["mass"], rtol=1e-12)
        np.testing.assert_allclose(mon_b["rho_u2"], mon_a["rho_u2"], rtol=1e-12)
        assert np.array_equal(mon_b["nonfinite"], mon_a["nonfinite"])
        ia, ib = a.info(), b.info()
        assert ia["step"] == ib["step"]
        # both handles continue from the same state
        a.step(3)
        b.step(3)
        a.synchronize()
        b.synchronize()
        assert bits_equal(b.read("moments"), a.read("moments"))
    finally:
        a.close()
        b.close()


def test_streamed_job_twice_in_a_row():
    """Two jobs on one handle (the second starts from the first's results)
    equal one loop of 2n steps with an upload in the middle."""
    fo = ("S", "SMean", "k", "kMean")
    a = prepared(27, (32, 32, 48), fo, 32, 8)
    b = prepared(27, (32, 32, 48), fo, 32, 8)
    try:
        state = a.read("moments")
        outs1 = out_arrays(b, fo, 32)
        b.run_streamed(np.ascontiguousarray(state), 6, outs1, slab=8, z_chunk=4)
        outs2 = out_arrays(b, fo, 32)
        b.run_streamed(np.ascontiguousarray(outs1["moments"]), 6, outs2, slab=8, z_chunk=4)
        a.step(12)
        a.synchronize()
        for s in ("moments",) + fo:
            assert bits_equal(outs2[s], a.read(s)), s
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
@pytest.mark.parametrize("q,n,slab", [(19, 7, 16), (27, 40, 8)])
def test_streamed_job_16bit_storage(storage, q, n, slab):
    """16-bit storage: the host values pass through staging blocks and the
    storage conversion on the copy streams; the results (FP32 on the host)
    equal write + step + read of the same handle type bit for bit."""
    fo = ("S", "SMean", "k", "kMean")
    shapes = (32, 40, 56)
    hs = []
    try:
        for _ in range(2):
            c = Cavity(q, *shapes, 400.0, 0.05, function_objects=fo, storage=storage)
            c.init_regions()
            c.step(6)
            c.synchronize()
            hs.append(c)
        a, b = hs
        state = pinned((10,) + a.shape, np.float32)
        a.read("moments", out=state)
        a.write(state)
        a.step(n)
        a.synchronize()
        ref = {s: a.read(s) for s in ("moments",) + fo}
        outs = out_arrays(b, fo, 32)
        b.run_streamed(state, n, outs, slab=slab)
        for s, r in ref.items():
            assert bits_equal(outs[s], r), s
    finally:
        for c in hs:
            c.close()


def test_streamed_job_refusals():
    c = Cavity(27, 16, 16, 16, 200.0, 0.05)
    try:
        c.init_regions()
        net = _lib.MLP()
        net.in_lo[:] = [-1e30] * 16
        net.in_hi[:] = [1e30] * 16
        net.in_scale[:] = [1.0] * 16
        c.set_closure(net)
        state = c.read("moments")
        with pytest.raises(_lib.LBMError) as e:  # not with the learned closure
            c.run_streamed(state, 2, {"moments": np.zeros_like(state)})
        assert e.value.status == LBM_ERR_STATE
    finally:
        c.close()
    c = Cavity(19, 32, 32, 32, 100.0, 0.05)
    try:
        c.init_regions()
        state = c.read("moments")
        with pytest.raises(_lib.LBMError) as e:
            c.run_streamed(state, 0, {"moments": np.zeros_like(state)})
        assert e.value.status == LBM_ERR_ARG
        with pytest.raises(_lib.LBMError) as e:  # no function objects on this handle
            c.run_streamed(state, 2, {"k": np.zeros((1, 32, 32, 32), np.float32)})
        assert e.value.status == LBM_ERR_STATE
    finally:
        c.close()
