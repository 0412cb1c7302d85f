"""The multi-process paths on CPU: two gloo ranks (127.0.0.1) check the max-over-ranks
timing of bench.py, the split of ONE batch across ranks by factorization flops (every
matrix on exactly one rank, the work balanced, the per-matrix results gathered on the host
equal to a single-rank run), and that the reference arm does its work on rank 0 only."""
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


def _batch():
    """A small batch of the batched workload's kind (weighted grids of uneven sides)."""
    import sys
    sys.path.insert(0, ROOT)
    from swcholesky_b200 import batch_shard as BS
    from swcholesky_b200 import matrices as M
    from swcholesky_b200 import workloads as W
    src, _ = W.batch_sources(count=12, seed=3, lo=6, hi=30)
    mats = [M.permute_lower(A, p) for A, p in src]
    return mats, [BS.matrix_flops(m) for m in mats]


def _logdet(m):
    """A per-matrix result computed on the host (log det by a dense Cholesky)."""
    import scipy.sparse as sp
    low = sp.csc_matrix((m.data, m.indices, m.indptr), shape=(m.n, m.n)).toarray()
    full = low + np.tril(low, -1).T
    return float(2.0 * np.log(np.diag(np.linalg.cholesky(full))).sum())


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
        from swcholesky_b200 import batch_shard as BS
        ms = bench.max_over_ranks(10.0 + rank, world, "cpu")
        mats, costs = _batch()
        mine = BS.split_by_cost(costs, world)[rank]
        local = [_logdet(mats[i]) for i in mine]
        gathered = BS.gather_results(mine, local, len(mats), world)
        buf = io.StringIO()

        class Args:
            workload = "grid2d_100"
            steps = 1
            warmup = 0
        with contextlib.redirect_stdout(buf):
            if rank != 0:
                bench.run_reference(Args, rank, world)   # must return at once, no output
        out.put((rank, ms, mine.tolist(), gathered.tolist(), buf.getvalue()))
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
    (r0, ms0, mine0, got0, _), (r1, ms1, mine1, got1, out1) = res
    assert ms0 == ms1 == 11.0            # both ranks see the slowest rank's time
    mats, costs = _batch()
    # every matrix on exactly one rank
    assert sorted(mine0 + mine1) == list(range(len(mats)))
    # balanced: the busier rank within the list-scheduling bound (4/3 of the optimum,
    # which is at least the mean and at least the largest matrix)
    loads = [sum(costs[i] for i in mine0), sum(costs[i] for i in mine1)]
    bound = max(sum(costs) / 2, max(costs))
    assert max(loads) <= 4.0 / 3.0 * bound
    # the gathered per-matrix results are the single-rank results, on both ranks
    single = [_logdet(m) for m in mats]
    assert got0 == got1 == single
    assert out1 == ""                    # the reference arm runs on rank 0 only
