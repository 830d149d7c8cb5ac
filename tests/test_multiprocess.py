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


def _serve_rank(rank, world, port, out):
    import datetime
    from importlib import import_module

    import numpy as np
    import torch
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    import bench
    x = ge.load_package()
    serve = import_module(x.__name__ + ".serve")
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        reqs = serve.make_requests(11, seed=3, n_max=3e4, rate=4.0)
        mine = serve.shard_requests(reqs, rank, world)
        assert [r.rid for r in mine] == list(range(rank, 11, world))
        # a stand-in for each rank's Server: every request done 0.5 s after arrival
        res = [serve.Result(rid=r.rid, n_cells=100 * (r.rid + 1), arrival=r.arrival, admitted=r.arrival,
                            finished=r.arrival + 0.5, iterations=10 + r.rid, converged=True,
                            residuals=np.zeros(0)) for r in mine]
        merged, wall = bench.gather_served(res, 5.0 + rank, world, serve)
        out[rank] = ([r.rid for r in merged], wall, serve.summarize(merged, wall))
        torch.distributed.barrier()
    finally:
        torch.distributed.destroy_process_group()


def test_serving_sharded_over_gloo_ranks():
    """Serving sharded by request over two gloo ranks: rank r takes requests
    r, r + 2, ...; after the run every rank holds all 11 results once, the
    slowest rank's wall time, and the same summary over every request."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        ps = [ctx.Process(target=_serve_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(180)
            assert p.exitcode == 0
        got = dict(out)
    assert got[0][0] == list(range(11)) and got[1][0] == list(range(11))
    assert got[0][1] == got[1][1] == 6.0
    s = got[0][2]
    assert s == got[1][2]
    assert s["cases"] == 11 and s["converged"] == 11
    assert s["mcell_iters_per_s"] == pytest.approx(sum(100 * (i + 1) * (10 + i) for i in range(11)) / 6.0 / 1e6)
    assert s["p50_ms"] == pytest.approx(500.0)
