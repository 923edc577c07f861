"""The multi-process path of bench.py on CPU: two ranks over gloo on
127.0.0.1, as torchrun starts them.  Checks the rank bookkeeping, the barrier,
the max-over-ranks timing reduction and that only rank 0 of the reference arm
does work (the other ranks leave at once)."""
from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup(collective=True, backend="gloo")
    bench.barrier(w)
    # each rank reports its own "device time"; every rank must see the max
    worst = bench.allreduce_max(1.5 + r, w)

    class Args:  # the reference arm's arguments; rank 1 must return at once
        nx, scheme, steps, warmup, gpus = 64, "hllc", 1, 1, w
    if r != 0:
        bench.run_reference(Args, w, r)
    bench.barrier(w)
    out.put((r, w, local, worst))
    dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(200)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 0, 2.5), (1, 2, 1, 2.5)]
