"""The N>1 replica path of bench.py on CPU: two gloo ranks go through the same plumbing the
GPU run uses (process-group set-up from the torchrun variables, evenly spread orbit phases,
barrier, max-over-ranks timing) without a GPU.  The path has no data-path collective: each
replica renders its own views, and only the timing is reduced."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    w, r, local = bench.dist_init("gloo")
    assert (w, r, local) == (world, rank, rank)
    phase = bench.orbit_phase(r, w, 120)
    bench.barrier(w)
    slowest = bench.max_over_ranks(10.0 + 5.0 * r, w)
    out[r] = (phase, slowest)
    dist.destroy_process_group()


def test_two_replicas_over_gloo():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == 0 and res[1][0] == 60          # replicas start half an orbit apart
    assert res[0][1] == res[1][1] == 15.0               # both report the slower rank's time

