"""The N > 1 path of bench.py on CPU: two gloo ranks (replicas, no collective
on the data path) agree on the slowest rank's time, and the whole-job value
counts every rank's cells."""
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
    import datetime

    import torch
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench.dist_setup(None)
        assert (w, r, local) == (world, rank, rank)
        slowest = bench.max_over_ranks(10.0 + rank, world)       # rank times 10 s, 11 s
        out[rank] = (slowest, bench.job_throughput(1000, world, 5, slowest))
        torch.distributed.barrier()
    finally:
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_agree():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        got = dict(out)
    assert got[0] == got[1]
    slowest, value = got[0]
    assert slowest == 11.0
    assert value == pytest.approx(1000 * 2 * 5 / 11.0 / 1e6)


def test_single_rank_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_throughput(2097152, 1, 10, 1.0) == pytest.approx(20.97152)
