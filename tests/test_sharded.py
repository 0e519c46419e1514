"""One embedding split by rows over ranks (sgtsne_b200.sharded).

CPU: two gloo ranks drive the orchestration (the order of scatter, grid
all-reduce, gather, Z all-reduce, update and all-gather) over the FP64 CPU
restatement of the phases (tests/shard_oracle.py); the coordinates after a
few iterations equal those of one rank holding every row (rel <= 1e-10: the
split only reorders FP64 sums) and those of the oracle's own loop.
GPU: the engine's shard phases on one rank (a one-rank NCCL group) follow
the whole-embedding job within the parity tolerance of iterations.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import REPO, make_problem

ITERS = 6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    rp, col, val, _ = make_problem(n=1500, dim=12, k=10, seed=5)
    n = len(rp) - 1
    Y0 = np.random.default_rng(1).standard_normal((n, 2)) * 3
    return rp, col, val, Y0


def _run_local(world_rank, world, rp, col, val, Y0, group=None):
    from shard_oracle import OracleShard

    from sgtsne_b200.sharded import ShardedEmbedding
    b = OracleShard(rp, col, val, len(rp) - 1, 2, world_rank, world, early_iter=2)
    b.set_y(Y0)
    ShardedEmbedding(b, group).run(ITERS)
    return b.Y().copy()


def _rank(rank, world, port, q):
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "tests"))
    sys.path.insert(0, os.path.join(REPO, "gpu-sg-sne_b200", "python"))
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        rp, col, val, Y0 = _problem()
        q.put((rank, _run_local(rank, world, rp, col, val, Y0)))
    finally:
        dist.destroy_process_group()


def _solo(q):
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "tests"))
    sys.path.insert(0, os.path.join(REPO, "gpu-sg-sne_b200", "python"))
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    try:
        rp, col, val, Y0 = _problem()
        q.put(_run_local(0, 1, rp, col, val, Y0))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_rank(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    p1 = ctx.Process(target=_solo, args=(q,))
    p1.start()
    one = q.get(timeout=300)
    p1.join(timeout=60)
    assert p1.exitcode == 0
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    # every rank holds the same coordinates, equal to the one-rank run's
    assert rel(got[0], got[1]) == 0.0
    assert rel(got[0], one) <= 1e-10
    # and to the oracle's own loop (centred each iteration in h mode)
    rp, col, val, Y0 = _problem()
    Yo = oracle.kl_minimization(rp, col, val, Y0, ITERS, early_iter=2, alpha=12.0, h=0.7,
                                grid_mode=0)
    c = one - one.mean(0)
    assert rel(c, Yo - Yo.mean(0)) <= 1e-9


def test_stretches_cover_every_row_once():
    from sgtsne_b200.sharded import local_rows, stretch
    rp, col, val, _ = make_problem(n=1000, k=8, seed=2)
    n = len(rp) - 1
    for world in (1, 2, 3, 7):
        seen = []
        cat_col = []
        for r in range(world):
            lo, hi, c = stretch(n, world, r)
            assert c * world >= n and hi - lo <= c
            seen.extend(range(lo, hi))
            lrp, lc, lv = local_rows(rp, col, val, lo, hi)
            assert lrp[0] == 0 and len(lrp) == hi - lo + 1 and lrp[-1] == len(lc) == len(lv)
            cat_col.append(lc)
        assert seen == list(range(n))
        assert np.array_equal(np.concatenate(cat_col), col)


@pytest.mark.gpu
def test_engine_shard_follows_the_whole_embedding():
    """One rank holding every row through the shard phases and a one-rank
    NCCL group, against sgt_job_run on the same P and Y0: the grid decision
    is recomputed from all coordinates each iteration (a different
    summation order of the mean), so the trajectories agree to rounding."""
    import torch
    import torch.distributed as dist

    import sgtsne_b200 as S
    from sgtsne_b200.sharded import EngineShard, ShardedEmbedding
    rp, col, val, _ = make_problem(n=4000, k=12, seed=9)
    n = len(rp) - 1
    Y0 = (np.random.default_rng(4).standard_normal((n, 2)) * 1e-2).astype(np.float32)
    p = S.default_params(d=2, format=S.FORMAT_CSR, max_iter=60, early_iter=20, max_grid=128)
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = S.Context(0)
    ctx.set_stream(stream.cuda_stream)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    try:
        sh = EngineShard(ctx, p, n, 0, 1, rp, col, val.astype(np.float32), "cuda:0")
        sh.set_y(Y0)
        ShardedEmbedding(sh).run(20)
        Ys = sh.get_y()
        assert sh.info().iter == 20 and sh.info().error_flags == 0
        sh.close()
        job = S.Job(ctx, p, rp, col, val.astype(np.float32), device_mem=False)
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(20)
        Yj = job.get_y(np.empty((n, 2), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
        job.close()
    finally:
        dist.destroy_process_group()
        torch.cuda.set_stream(torch.cuda.default_stream())
        ctx.close()
    assert float(np.linalg.norm(Ys - Yj) / np.linalg.norm(Yj)) <= 1e-3
