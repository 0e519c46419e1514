"""Batches (one CUDA graph over many jobs) and the continuous-batching server.

Each result must be the same alone and in the mix, within a stated
tolerance.  The FP32 atomics of S2G accumulate in a different order from run
to run, and the t-SNE iteration amplifies such last-bit differences (a
difference in maxy that flips the grid-size decision moves the forces by the
interpolation error, ~1e-3): two plain runs of one job from the same Y0
differ by rel-L2 ~1e-7 after 2 iterations, up to ~1e-4 after 5 and up to
~1e-2 after 40.  KL is compared once the early exaggeration has ended and
the embedding has relaxed (exaggeration for 100 iterations, KL after 300):
there, four plain runs of each job below spread by at most 0.4 % in KL,
where during the exaggeration they spread by up to 1.1 %.  So:

  after 2 iterations     Y alone vs in the mix        rel-L2 <= 1e-5
  after 300 iterations   KL alone vs in the mix       within 1 %
"""
import numpy as np
import pytest

from conftest import make_problem

pytestmark = pytest.mark.gpu

TOL_Y = 1e-5     # Y after SHORT iterations
SHORT = 2
LONG = 300
EARLY = 100      # iterations of early exaggeration
TOL_KL = 0.01    # relative KL after LONG iterations


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def problems():
    """Uneven sizes, d = 2 and 3, P from the oracle's pipeline."""
    specs = [(1500, 2, 1), (4000, 3, 2), (9000, 2, 3), (2500, 2, 4), (6000, 3, 5), (12000, 2, 6)]
    out = []
    for n, d, seed in specs:
        rp, col, val, _ = make_problem(n=n, dim=20, ncomp=5, k=12, seed=seed)
        y0 = (np.random.default_rng(seed).standard_normal((n, d)) * 1e-2).astype(np.float32)
        out.append((rp, col, val.astype(np.float32), d, y0))
    return out


def params(S, d, iters):
    return S.default_params(d=d, format=S.FORMAT_CSR, max_iter=iters, early_iter=EARLY,
                            h=0.7 if d == 2 else 1.2)


def run_alone(S, ctx, prob, iters):
    rp, col, val, d, y0 = prob
    job = S.Job(ctx, params(S, d, iters), rp, col, val, device_mem=False)
    job.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
    job.run(iters)
    out = np.empty_like(y0)
    job.get_y(out, S.LAYOUT_POINT_MAJOR, False, 1)
    job.close()
    return out


def kl_of(oracle, prob, Y):
    """KL (alpha = 1) of coordinates Y, with Z from the oracle's repulsion."""
    rp, col, val, d, _ = prob
    h = 0.7 if d == 2 else 1.2
    _, Z, _, _ = oracle.repulsive_interp(Y.astype(np.float64), h)
    return oracle.kl(rp, col, val.astype(np.float64), Y.astype(np.float64), 1.0, Z)


@pytest.mark.parametrize("iters", [SHORT, LONG])
def test_batch_matches_alone(problems, oracle, iters):
    import sgtsne_b200 as S
    ctx = S.Context(0)
    alone = [run_alone(S, ctx, p, iters) for p in problems]
    jobs = []
    for rp, col, val, d, y0 in problems:
        j = S.Job(ctx, params(S, d, iters), rp, col, val, device_mem=False)
        j.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
        jobs.append(j)
    batch = S.Batch(ctx, jobs, iters_per_launch=8)
    batch.run(iters // 2)  # launches of 8 chained iterations, then single ones
    batch.run(iters - iters // 2)
    for j, ref, prob in zip(jobs, alone, problems):
        out = np.empty_like(ref)
        j.get_y(out, S.LAYOUT_POINT_MAJOR, False, 1)
        assert j.info().iter == iters
        assert j.info().error_flags == 0
        if iters == SHORT:
            assert rel(out, ref) <= TOL_Y
        else:
            ka, kb = kl_of(oracle, prob, ref), kl_of(oracle, prob, out)
            assert abs(kb - ka) <= TOL_KL * ka, (ka, kb)
    batch.close()
    for j in jobs:
        j.close()
    ctx.close()


def test_batch_of_mixed_formats(problems):
    """A batch holding a COO job runs one graph branch per job instead of the
    fused launches of an all-CSR batch; results match alone runs."""
    import sgtsne_b200 as S
    ctx = S.Context(0)
    fmts = [S.FORMAT_CSR, S.FORMAT_COO, S.FORMAT_CSR]
    alone, jobs = [], []
    for prob, fmt in zip(problems[:3], fmts):
        rp, col, val, d, y0 = prob
        p = params(S, d, SHORT)
        p.format = fmt
        for dest in (alone, jobs):
            j = S.Job(ctx, p, rp, col, val, device_mem=False)
            j.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
            dest.append(j)
    for j in alone:
        j.run(SHORT)
    batch = S.Batch(ctx, jobs, iters_per_launch=1)
    batch.run(SHORT)
    for a, j, prob in zip(alone, jobs, problems):
        ya, yb = np.empty_like(prob[4]), np.empty_like(prob[4])
        a.get_y(ya, S.LAYOUT_POINT_MAJOR, False, 1)
        j.get_y(yb, S.LAYOUT_POINT_MAJOR, False, 1)
        assert rel(yb, ya) <= TOL_Y
    batch.close()
    for j in alone + jobs:
        j.close()
    ctx.close()


def test_batch_step_matches_alone(problems):
    """sgt_batch_step: the fused launches without a batch object, over a set
    of jobs that changes between calls (two jobs, then three)."""
    import sgtsne_b200 as S
    ctx = S.Context(0)
    alone = [run_alone(S, ctx, p, SHORT) for p in problems[:3]]
    jobs = []
    for rp, col, val, d, y0 in problems[:3]:
        j = S.Job(ctx, params(S, d, SHORT), rp, col, val, device_mem=False)
        j.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
        jobs.append(j)
    S.batch_step(ctx, jobs[:2], 1)
    S.batch_step(ctx, jobs[2:], 1)
    S.batch_step(ctx, jobs, SHORT - 1)
    for j, ref in zip(jobs, alone):
        out = np.empty_like(ref)
        j.get_y(out, S.LAYOUT_POINT_MAJOR, False, 1)
        assert j.info().iter == SHORT
        assert rel(out, ref) <= TOL_Y
    for j in jobs:
        j.close()
    ctx.close()


def test_batch_rejects_foreign_and_relayout(problems):
    import sgtsne_b200 as S
    c1, c2 = S.Context(0), S.Context(0)
    rp, col, val, d, y0 = problems[0]
    j1 = S.Job(c1, params(S, d, 10), rp, col, val, device_mem=False)
    j2 = S.Job(c2, params(S, d, 10), rp, col, val, device_mem=False)
    with pytest.raises(S.SgtError) as e:
        S.Batch(c1, [j1, j2])
    assert e.value.status == 1
    p = params(S, d, 10)
    p.relayout_every = 5
    j3 = S.Job(c1, p, rp, col, val, device_mem=False)
    with pytest.raises(S.SgtError) as e:
        S.Batch(c1, [j1, j3])
    assert e.value.status == 4
    for j in (j1, j2, j3):
        j.close()
    c1.close()
    c2.close()


def test_server_matches_alone_and_overlaps(problems, oracle):
    """Six requests, at most three running: later requests are admitted
    while earlier ones still run, and every result equals its plain run."""
    import sgtsne_b200 as S
    ctx = S.Context(0)
    iters = [SHORT, LONG, SHORT, LONG + 16, SHORT, LONG - 24]
    alone = [run_alone(S, ctx, p, it) for p, it in zip(problems, iters)]
    ctx.close()
    srv = S.Server(0, max_active=3, iters_per_round=8, rounds_ahead=2)
    outs = {}
    for (rp, col, val, d, y0), it in zip(problems, iters):
        rid, out = srv.submit(params(S, d, it), rp, col, val, y0)
        outs[rid] = out
    done = []
    for _ in range(600):
        done += srv.poll(wait_ms=100)
        if len(done) == len(problems):
            break
    assert sorted(done) == list(range(len(problems)))
    infos = [srv.info(r) for r in range(len(problems))]
    for r, inf in enumerate(infos):
        assert inf.state == S.REQ_DONE, (r, inf.status)
        assert inf.t_submit <= inf.t_admit <= inf.t_done
        if iters[r] == SHORT:
            assert rel(outs[r], alone[r]) <= TOL_Y
        else:
            ka = kl_of(oracle, problems[r], alone[r])
            kb = kl_of(oracle, problems[r], outs[r])
            assert abs(kb - ka) <= TOL_KL * ka, (r, ka, kb)
    # never more than three running at once
    events = sorted([(i.t_admit, 1) for i in infos] + [(i.t_done, -1) for i in infos])
    live = peak = 0
    for _, e in events:
        live += e
        peak = max(peak, live)
    assert peak <= 3
    # continuous: some request was admitted while another was still running
    assert any(infos[a].t_admit < infos[b].t_done and infos[b].t_admit < infos[a].t_admit
               for a in range(len(infos)) for b in range(len(infos)) if a != b)
    srv.close()


def test_server_budget_and_oversize(problems):
    import sgtsne_b200 as S
    fps = [S.job_footprint(params(S, p[3], 24), len(p[0]) - 1, int(p[0][-1])) for p in problems]
    budget = max(fps) + min(fps) // 2  # never room for the two largest together
    srv = S.Server(0, hbm_budget=budget, max_active=8, iters_per_round=8)
    for p in problems:
        srv.submit(params(S, p[3], 24), p[0], p[1], p[2], p[4])
    done = []
    for _ in range(600):
        done += srv.poll(wait_ms=100)
        if len(done) == len(problems):
            break
    infos = [srv.info(r) for r in range(len(problems))]
    assert all(i.state == S.REQ_DONE for i in infos)
    # the admitted footprints never exceed the budget
    events = sorted([(i.t_admit, i.footprint) for i in infos] +
                    [(i.t_done, -i.footprint) for i in infos], key=lambda e: (e[0], e[1]))
    live = 0
    for _, f in events:
        live += f
        assert live <= budget
    big = problems[-1]
    with pytest.raises(S.SgtError) as e:
        tiny = S.Server(0, hbm_budget=min(fps) // 4)
        try:
            tiny.submit(params(S, big[3], 24), big[0], big[1], big[2], big[4])
        finally:
            tiny.close()
    assert e.value.status == 3
    srv.close()


def test_one_dimensional_batch_and_server(problems):
    """d = 1 jobs (and a COO and a hybrid one) in a batch and through the
    server: the same after two iterations as alone."""
    import sgtsne_b200 as S
    ctx = S.Context(0)
    probs = []
    for fmt, (rp, col, val, _, y0) in zip((0, 2, 3), problems[:3]):
        probs.append((rp, col, val, y0[:, :1].copy(), fmt))

    def par(fmt, it):
        return S.default_params(d=1, format=fmt, max_iter=it, early_iter=EARLY, h=0.5)
    alone = []
    for rp, col, val, y0, fmt in probs:
        j = S.Job(ctx, par(fmt, SHORT), rp, col, val, device_mem=False)
        j.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
        j.run(SHORT)
        alone.append(j.get_y(np.empty_like(y0), S.LAYOUT_POINT_MAJOR, False, 1))
        j.close()
    jobs = []
    for rp, col, val, y0, fmt in probs:
        j = S.Job(ctx, par(fmt, SHORT), rp, col, val, device_mem=False)
        j.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
        jobs.append(j)
    b = S.Batch(ctx, jobs, iters_per_launch=4)
    b.run(SHORT)
    for j, ref in zip(jobs, alone):
        assert rel(j.get_y(np.empty_like(ref), S.LAYOUT_POINT_MAJOR, False, 1), ref) <= TOL_Y
    b.close()
    for j in jobs:
        j.close()
    ctx.close()
    srv = S.Server(0, max_active=2, iters_per_round=4)
    outs = [srv.submit(par(fmt, SHORT), rp, col, val, y0)[1] for rp, col, val, y0, fmt in probs]
    done = []
    for _ in range(300):
        done += srv.poll(wait_ms=50)
        if len(done) == len(probs):
            break
    for r, (out, ref) in enumerate(zip(outs, alone)):
        assert srv.info(r).state == S.REQ_DONE
        assert rel(out, ref) <= TOL_Y
    srv.close()
