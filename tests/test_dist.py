"""CPU, world size 2 over gloo: the multi-process plumbing bench.py uses for
N > 1 (one replica per GPU): the job value is the units all ranks processed
over the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, local, w = bench.dist_env()
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, w, "cpu")   # rank 1 is slower
        units = bench.sum_over_ranks(1000 * (rank + 1), w, "cpu")  # ranks build different collections
        out.put((r, local, w, ms, units, units / (ms / 1000.0)))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions():
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
    for rank, (r, local, w, ms, units, value) in enumerate(res):
        assert (r, local, w) == (rank, rank, 2)
        assert ms == 150.0
        assert units == 3000.0
        assert value == pytest.approx(3000.0 / 0.150)


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.sum_over_ranks(7, 1, "cpu") == 7
