"""The multi-process paths of bench.py on CPU: two gloo ranks (127.0.0.1) check the
max-over-ranks timing, that every rank of the batched workload gets its own batch, and that
the reference arm does its work on rank 0 only."""
import io
import os
import socket
import contextlib

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    import datetime
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from swcholesky_b200 import workloads as W
        ms = bench.max_over_ranks(10.0 + rank, world, "cpu")
        src, sides = W.batch_sources(count=3, seed=bench.batch_seed(rank), lo=5, hi=12)
        buf = io.StringIO()

        class Args:
            workload = "grid2d_100"
            steps = 1
            warmup = 0
        with contextlib.redirect_stdout(buf):
            if rank != 0:
                bench.run_reference(Args, rank, world)   # must return at once, no output
        out.put((rank, ms, [int(s) for s in sides], buf.getvalue()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, sides0, _), (r1, ms1, sides1, out1) = res
    assert ms0 == ms1 == 11.0            # both ranks see the slowest rank's time
    assert sides0 != sides1              # each rank factors its own batch
    assert out1 == ""                    # the reference arm runs on rank 0 only
