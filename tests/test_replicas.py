"""Multi-process replicas on CPU (gloo, world size 2): the barrier and the
max/sum over ranks the benchmark uses for N GPUs, and a rank that leaves
early: the other one gets an error from the process group's timeout
instead of waiting for ever."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from cudalbm_b200.replicas import Replicas

    if mode == "collectives":
        g = Replicas("gloo", timeout_s=30)
        g.barrier()
        out[rank] = (g.max(1.5 * (rank + 1)), g.sum(rank + 0.25), g.world, g.rank)
        g.barrier()
        g.close()
    else:  # rank 1 leaves before the barrier; rank 0 must see an error
        g = Replicas("gloo", timeout_s=3)
        if rank == 1:
            g.close()
            out[rank] = "left"
            return
        try:
            g.barrier()
            g.max(1.0)
            out[rank] = "no error"
        except Exception as exc:
            out[rank] = "error: " + type(exc).__name__


def _run(mode):
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, mode, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        alive = [p for p in procs if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive, "a rank hung"
        return dict(out)


def test_barrier_and_max_over_ranks():
    out = _run("collectives")
    assert out[0] == (3.0, 1.5, 2, 0)
    assert out[1] == (3.0, 1.5, 2, 1)


def test_rank_leaving_early_is_an_error_not_a_hang():
    out = _run("leave")
    assert out[1] == "left"
    assert out[0].startswith("error")
