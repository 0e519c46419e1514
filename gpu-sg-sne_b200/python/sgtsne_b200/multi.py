"""Many embeddings at once: the batched workload (many independent jobs in
one CUDA graph) and the served workload (an open-loop request stream through
the continuous-batching server), each beside its plain form (the same jobs
run one after another through sgt_job_run).

Used by bench.py.  P of every instance is built on the device through the
engine (exact kNN, lambda bisection, symmetrisation), as for the
single-embedding benchmark.
"""
from __future__ import annotations

import time

import numpy as np

from . import workloads as W


def _csr_from_knn(ctx, idx, d2, lam, dev):
    import torch
    n, k = idx.shape
    rp = torch.arange(0, (n + 1) * k, k, dtype=torch.int32, device=dev)
    vals = d2.reshape(-1).contiguous().clone()
    col = idx.reshape(-1).to(torch.int32).contiguous()
    # the engine works on its own stream: the tensors torch just wrote on
    # its stream must be complete before the engine reads them
    torch.cuda.synchronize(dev)
    ctx.lambda_bisect(n, rp, vals, float(lam), 1)
    nnz = n * k
    srp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    sc = torch.empty(2 * nnz, dtype=torch.int32, device=dev)
    sv = torch.empty(2 * nnz, dtype=torch.float32, device=dev)
    m = ctx.symmetrize(n, nnz, rp, col, vals, 1.0 / (2 * n), srp, sc, sv)
    return srp.cpu().numpy(), sc[:m].cpu().numpy(), sv[:m].cpu().numpy()


def batched_instances(ctx, count, seed, dev, n_lo=2000, n_hi=200000, k=30):
    """The batched configuration: n log-uniform in [n_lo, n_hi], dimension
    uniform in 20..100, isotropic mixture (centres N(0, 16 I), unit variance)
    with 5..30 components and a seed per instance, k = 30, lambda = 1, half
    d = 2 and half d = 3.  Returns a list of dicts."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        dim = int(rng.integers(20, 101))
        ncomp = int(rng.integers(5, 31))
        d = 2 if i % 2 == 0 else 3
        X, _ = W.gmm_isotropic(n, dim, ncomp, 16.0, seed * 100003 + i, dtype=np.float32)
        idx, d2 = W.knn_engine(ctx, X, k, dev)
        rp, col, val = _csr_from_knn(ctx, idx, d2, 1.0, dev)
        y0 = (np.random.default_rng(seed + 7 + i).standard_normal((n, d)) * 1e-2).astype(np.float32)
        out.append({"n": n, "d": d, "dim": dim, "rp": rp, "col": col, "val": val, "y0": y0})
    return out


def request_instances(ctx, count, seed, dev, n_lo=1000, n_hi=500000, k=30):
    """The served configuration: n log-uniform in [n_lo, n_hi], d in {2, 3},
    lambda in {1, 10, 30}, 500..1000 iterations, P from the 50-D 40-component
    Zipf(1.1) mixture with a seed per request."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        d = int(rng.choice([2, 3]))
        lam = float(rng.choice([1.0, 10.0, 30.0]))
        iters = int(rng.integers(500, 1001))
        X, _ = W.gmm_zipf(n, 50, 40, 1.1, 25.0, seed * 100003 + i)
        idx, d2 = W.knn_engine(ctx, X, k, dev)
        rp, col, val = _csr_from_knn(ctx, idx, d2, lam, dev)
        y0 = (np.random.default_rng(seed + 11 + i).standard_normal((n, d)) * 1e-2).astype(np.float32)
        out.append({"n": n, "d": d, "lambda": lam, "iters": iters, "rp": rp, "col": col,
                    "val": val, "y0": y0})
    return out


# sgt_params.locality_order of the jobs these helpers create (1: the
# engine's default, a locality order of the points at creation)
LOCALITY_ORDER = 1


def job_params(S, d, iters, lam=1.0):
    p = S.default_params(d=d, format=S.FORMAT_CSR, max_iter=iters, early_iter=250,
                         h=0.7 if d == 2 else 1.2)
    p.lambda_ = lam
    p.locality_order = LOCALITY_ORDER
    return p


def run_batched(S, ctx, inst, iters, stream, iters_per_launch=8):
    """Plain (each job's iterations through sgt_job_run, one job after
    another) and batched (all jobs in one graph) on the same device-resident
    jobs from the same Y0; CUDA-event time of each."""
    import torch
    jobs = []
    for it in inst:
        j = S.Job(ctx, job_params(S, it["d"], iters), torch.from_numpy(it["rp"]).cuda(),
                  torch.from_numpy(it["col"]).cuda(), torch.from_numpy(it["val"]).cuda(),
                  device_mem=True)
        jobs.append(j)
    y0s = [torch.from_numpy(it["y0"]).cuda() for it in inst]

    def reset():
        for j, y in zip(jobs, y0s):
            j.set_y(y, S.LAYOUT_POINT_MAJOR, True)
        torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # warm-up: graphs captured, caches primed
    reset()
    for j in jobs:
        j.run(16)
    batch = S.Batch(ctx, jobs, iters_per_launch)
    batch.run(iters_per_launch)
    torch.cuda.synchronize()
    # plain
    reset()
    e0.record(stream)
    for j in jobs:
        j.run(iters)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    # batched
    reset()
    e0.record(stream)
    batch.run(iters)
    e1.record(stream)
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1)
    errs = [j.info().error_flags for j in jobs]
    batch.close()
    for j in jobs:
        j.close()
    return {"plain_ms": plain_ms, "batched_ms": batch_ms,
            "error_flags": int(np.bitwise_or.reduce(errs))}


def plain_service_times(S, ctx, inst):
    """Each request alone through the public API from host buffers (job
    create, Y0 upload, iterations, centred result to the host): seconds."""
    out = []
    for it in inst:
        t0 = time.perf_counter()
        j = S.Job(ctx, job_params(S, it["d"], it["iters"], it["lambda"]), it["rp"], it["col"],
                  it["val"], device_mem=False)
        j.set_y(it["y0"], S.LAYOUT_POINT_MAJOR, False)
        j.run(it["iters"])
        y = np.empty_like(it["y0"])
        j.get_y(y, S.LAYOUT_POINT_MAJOR, False, 1)
        j.close()
        out.append(time.perf_counter() - t0)
    return np.array(out)


def fifo_latencies(arrivals, service):
    """Latencies of a single FIFO server running the requests one at a time
    (the plain form under the same arrival stream)."""
    fin = 0.0
    lat = np.empty(len(arrivals))
    for i, (a, s) in enumerate(zip(arrivals, service)):
        fin = max(fin, a) + s
        lat[i] = fin - a
    return lat


def serve_stream(S, inst, arrivals, device=0, **server_kw):
    """Open-loop stream: request i is submitted at arrivals[i] seconds after
    the start; returns (latencies, makespan, states)."""
    srv = S.Server(device, **server_kw)
    t0 = srv.now()
    ids = []
    done = 0
    i = 0
    while done < len(inst):
        now = srv.now() - t0
        while i < len(inst) and arrivals[i] <= now:
            it = inst[i]
            rid, _ = srv.submit(job_params(S, it["d"], it["iters"], it["lambda"]), it["rp"],
                                it["col"], it["val"], it["y0"])
            ids.append(rid)
            i += 1
        wait = 5.0 if i >= len(inst) else max(0.0, (arrivals[i] - (srv.now() - t0)) * 1e3)
        done += len(srv.poll(wait_ms=min(wait, 5.0)))
    infos = [srv.info(r) for r in ids]
    srv.close()
    # latency from the scheduled arrival (open loop), not from the submit call
    lat = np.array([inf.t_done - t0 - a for inf, a in zip(infos, arrivals)])
    makespan = max(inf.t_done for inf in infos) - t0
    states = [inf.state for inf in infos]
    return lat, makespan, states


def percentiles(lat):
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(np.mean(lat))}
