"""The multi-rank plumbing of bench.py on CPU: two gloo ranks, barrier,
max-over-ranks timing and the replica aggregation (value = N * K / max time)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    sys.path.insert(0, REPO)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    r, w, l = bench.dist_env()
    dist = bench.dist_init(w, "gloo")
    try:
        bench.barrier(dist)
        # each replica reports its own elapsed time; the job time is the max
        mine = 10.0 * (rank + 1)
        ms = bench.max_over_ranks(dist, mine)
        q.put((r, w, l, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 for o in out)
    assert all(o[3] == 20.0 for o in out)  # max over ranks on every rank


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.dist_init(1, "gloo") is None
    assert bench.max_over_ranks(None, 3.5) == 3.5
