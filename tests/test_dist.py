"""The multi-GPU plumbing of bench.py on the CPU: two ranks on the gloo
backend (127.0.0.1) run the same collective calls the GPU run makes --
barrier, max over ranks, sum -- build their own replica boxes (seed + rank),
and agree on the whole-job rate, which counts every rank's units over the
slowest rank's time.  The path shards into independent replicas, so no
collective touches the data."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.init(backend="gloo", timeout_s=60)
    try:
        d.barrier()
        ms_local = 10.0 + 5.0 * rank                  # rank 1 is the slower one
        ms = d.max(ms_local)
        total = d.sum(1.0)
        w = bench.make_workload("ocp", 11 + rank, 300)
        rate = bench.job_rate(d.world, 1000, ms)
        d.barrier()
        q.put((rank, ms, total, float(w.x[0]), rate))
    finally:
        d.close()


def test_two_gloo_ranks_agree():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [15.0, 15.0]          # max over ranks
    assert [o[2] for o in out] == [2.0, 2.0]
    assert out[0][3] != out[1][3]                       # each rank its own replica box
    assert out[0][4] == out[1][4] == pytest.approx(2 * 1000 / 15e-3)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.init()
    assert not d.pg and d.max(3.0) == 3.0 and d.sum(2.0) == 2.0
    d.barrier()
    d.close()
