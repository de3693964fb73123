"""Small runs of every step-kernel path, for the checked-build test.

run_all() drives the library that this process loaded (the ordinary one, or
the checked build when LBM_B200_LIBRARY names it) through every kernel shape
and mode -- tile widths 32/16/8, one and two population planes, four CTAs per
SM, three TMA stages, the checked and the compile-time function-object
kernels, FP64 means, monitored steps, FP16/BF16 storage, streamed jobs,
batches and both closure evaluations -- and returns the results by name.

    python tests/checked_cases.py OUT.npz   # run_all() into an .npz file
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from cudalbm_b200 import _lib  # noqa: E402
from cudalbm_b200.solver import NVARS, Batch, Cavity  # noqa: E402

FO4 = ("S", "SMean", "k", "kMean")
FO_OTHER = ("S", "kMean", "momentsMean")  # a set the run-time-checked kernel serves


def _cavity(out, name, q, shape, steps, fo=(), mean_bits=32, storage="f32", mon=0, **kw):
    with Cavity(q, *shape, 350.0, 0.05, function_objects=fo, mean_bits=mean_bits, storage=storage, **kw) as c:
        c.init_regions()
        c.step(steps)
        if mon:
            m = c.step_monitored(mon)
        c.synchronize()
        out[f"{name}/moments"] = c.read("moments")
        for f in fo:
            out[f"{name}/{f}"] = c.read(f, dtype=np.float64 if (mean_bits == 64 and "Mean" in f) else np.float32)
        if mon:
            out[f"{name}/mass"] = np.array(m["mass"])


def run_all():
    out = {}
    shape = (48, 40, 56)  # 48 is not a multiple of the 32-node tile
    for q in (19, 27):
        shapes = [((32, 8, 2), 1), ((32, 8, 2), 2), ((16, 8, 2), 1), ((8, 8, 2), 1)]
        if q == 19:
            shapes += [((32, 8, 2), 4), ((32, 8, 3), 1)]
        for tile, npb in shapes:
            tag = f"q{q}_t{tile[0]}_s{tile[2]}_p{npb}"
            _cavity(out, tag + "_fo", q, shape, 9, fo=FO_OTHER, mon=3, tile=tile, pop_buffers=npb, z_chunk=5)
            _cavity(out, tag + "_plain", q, shape, 7, tile=tile, pop_buffers=npb, z_chunk=16)
        _cavity(out, f"q{q}_fo4", q, shape, 8, fo=FO4, tile=(32, 8, 2), pop_buffers=1, z_chunk=7)
        _cavity(out, f"q{q}_fo4_64", q, shape, 8, fo=FO4, mean_bits=64, tile=(32, 8, 2), pop_buffers=1)
        for st in ("f16", "bf16"):
            _cavity(out, f"q{q}_{st}", q, shape, 6, fo=FO4, storage=st, tile=(32, 8, 2), pop_buffers=1)
            if q == 19:
                _cavity(out, f"q{q}_{st}_p4", q, shape, 6, storage=st, tile=(32, 8, 2), pop_buffers=4)
        # streamed jobs (z-slab launches): short and long
        for n, slab in ((9, 8), (40, 16)):
            with Cavity(q, *shape, 350.0, 0.05, function_objects=FO4) as c:
                c.init_regions()
                c.step(3)
                state = c.read("moments")
                nz, ny, nx = c.shape
                outs = {s: np.empty((NVARS[s], nz, ny, nx), np.float32) for s in ("moments",) + FO4}
                c.run_streamed(state, n, outs, slab=slab)
                for s, a in outs.items():
                    out[f"q{q}_streamed{n}/{s}"] = a
        # a batch of three meshes (persistent kernel)
        specs = [dict(lattice=q, nx=32, ny=32, nz=32, Re=150.0), dict(lattice=q, nx=48, ny=16, nz=40, Re=700.0),
                 dict(lattice=q, nx=16, ny=24, nz=8, Re=100.0)]
        with Batch(specs) as b:
            for i in range(len(b)):
                b[i].init_regions()
            b.step(5)
            b.synchronize()
            for i in range(len(b)):
                out[f"q{q}_batch/{i}"] = b[i].read()
        # the learned closure with a zero network (fused and separate evaluation)
        net = _lib.MLP()
        net.in_lo[:] = [-1e30] * 16
        net.in_hi[:] = [1e30] * 16
        net.in_scale[:] = [1.0] * 16
        for fused in (True, False):
            with Cavity(q, 32, 32, 24, 350.0, 0.05) as c:
                c.init_regions()
                c.set_closure(net)
                c.closure_fused(fused)
                c.step(4)
                c.synchronize()
                out[f"q{q}_closure_{int(fused)}"] = c.read()
    return out


if __name__ == "__main__":
    res = run_all()
    np.savez(sys.argv[1], **res)
    print(f"{len(res)} results from {_lib.LIB_PATH}")
