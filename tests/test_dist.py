"""The multi-process plumbing of bench.py on CPU: one process per rank over
gloo, world size 2.  The survey path has no data-path collective (jobs are
replicated per GPU); ranks only meet to align the timed region (barrier) and
to take the slowest rank's time (max).  These run without a GPU."""
import multiprocessing as mp
import os
import socket

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, value, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "RANK": str(rank), "WORLD_SIZE": str(world),
                       "LOCAL_RANK": str(rank)})
    import bench
    r, w, local = bench.dist_env()
    d = bench.Dist(w)
    d.barrier()
    out = d.max(value)
    d.barrier()
    d.close()
    q.put((r, w, local, out))


def test_dist_max_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, [1.5, 4.25][r], q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 2 for r in res)
    assert all(r[3] == 4.25 for r in res)


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(1)
    d.barrier()
    assert d.max(3.0) == 3.0
    d.close()
