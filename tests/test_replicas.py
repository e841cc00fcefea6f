"""The multi-GPU replica logic on CPU: two processes over gloo take the
slowest rank's time, compute whole-job throughput from it, split work
evenly, and each compiles the query pipelines in its own compile-only
engine (no GPU: the data path has no collective, so gloo exercises all of
the host side)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from kushdb_b200 import replicas
    from kushdb_b200 import workloads as wl
    from kushdb_b200.engine import Engine
    r, w, local = replicas.rank_info()
    dist = replicas.init("gloo", timeout_s=60)
    try:
        slowest = replicas.max_over_ranks(10.0 * (r + 1), dist)
        rate = replicas.whole_job_rate(1_000_000, 4, w, slowest)
        b, e = replicas.share(1001, r, w)
        eng = Engine(-1)
        t = wl.group_by_table(rows=2000, seed=r)
        eng.register_table(t)
        eng.execute(wl.group_by_plan(t), fetch=False)
        launches = eng.kernel_launches()
        eng.close()
        replicas.barrier(dist)
        out.put((r, slowest, rate, b, e, launches))
    finally:
        replicas.finish(dist)


def test_two_rank_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(2))
    # both ranks see the slowest rank's time and the same whole-job rate
    assert [x[1] for x in res] == [20.0, 20.0]
    assert res[0][2] == res[1][2] == pytest.approx(1_000_000 * 4 * 2 / 0.020)
    # the shares tile the work exactly once
    assert (res[0][3], res[0][4], res[1][3], res[1][4]) == (0, 500, 500, 1001)
    # every rank ran the same pipelines
    assert res[0][5] == res[1][5] > 0
