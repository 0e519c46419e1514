"""Benchmark: SG-t-SNE gradient iterations per second on one embedding of
n = 1.3M points in 2-D (the 1.3M-point configuration: 50-D 40-component
Zipf(1.1) Gaussian mixture, exact kNN k = 30, lambda = 10, symmetrised,
h = 0.7, cubic interpolation, 1000 iterations with exaggeration 12 for the
first 250, Y0 ~ N(0, 1e-4 I)).

A step is one full gradient iteration (attractive SpMV, FFT-interpolated
repulsion, Z, gains/momentum update) of the run from Y0: W untimed warm-up
iterations, then K timed ones (the defaults, W = 5 and K = 995, time the
whole 1000-iteration job).  The iteration graphs are instantiated before the
timed region, so it holds graph launches only.  P (>= 400 MB) and the
per-point arrays exceed the 126 MB L2, so no flush is needed between steps.
The expanded-state line (a fixed spread-out embedding whose grid is at its
largest, 512 points per axis) is reported beside it for the large-grid
regime.

Both arms time the same P.  The first arm to run on a machine stores its P
in the temporary directory and the other arm reads it back: the engine arm
builds P on the device (kNN, lambda bisection, symmetrisation), the
reference arm with torch matrix products for the kNN and the CPU
restatement for the rest.  The engine arm always builds its own P too (the
setup it reports) and states how it compares with the stored one.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  Each rank runs an independent
replica of the embedding (the single-embedding path is not sharded: replicas
only); value = N * K / max-over-ranks time.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

# more hardware work queues than the default 8, so the streams of the
# served jobs (and the branches of a batch graph) do not share queues;
# read when the CUDA context is created, so set before torch starts CUDA
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "gpu-sg-sne_b200", "python"))
sys.path.insert(0, REPO)

METRIC = "t-SNE iters/s at n=1.3M,d=2 (%HBM roofline); served embeds/s, p99 vs plain"
PUBLISHED_ITERS_PER_S = 4.4  # 1.3M points, d=2, GTX 1060 (README chart, ~225 s / 1000 it)
WORKLOAD = ("n=1,300,000 FP32 points in 50-D, 40-component Gaussian mixture with "
            "Zipf(1.1) sizes, centres N(0,25I), eigenvalues U(0.2,2) under random rotations; "
            "exact kNN k=30, lambda=10 bisection on squared distances, (P+P^T)/(2n); "
            "d=2, h=0.7, cubic Lagrange (np=3)")


# ---------------------------------------------------------------------------
# distributed plumbing (also exercised by tests/test_bench_dist.py on gloo)
# ---------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def dist_init(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return dist


def barrier(dist, device=None):
    if dist is not None:
        if device is not None:
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()


def max_over_ranks(dist, value, device="cpu"):
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
KNN_SECONDS = [None]  # wall time of the last build_knn search (upload included)


def build_knn(n, seed, device, ctx=None):
    """The 1.3M-point configuration's points and their exact 30 nearest
    neighbours: through the engine (sgt_knn) when a context is given, else
    with torch matrix products (the reference arm on a host without the
    engine's device)."""
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_zipf(n, dim=50, ncomp=40, zipf_a=1.1, centre_var=25.0, seed=seed)
    t0 = time.perf_counter()
    if ctx is not None:
        idx, d2 = W.knn_engine(ctx, X, 30, device)
    else:
        idx, d2 = W.knn_torch(X, 30, device=device, block=1024)
    if str(device).startswith("cuda"):
        import torch
        torch.cuda.synchronize()
    KNN_SECONDS[0] = time.perf_counter() - t0
    if str(device).startswith("cuda"):
        torch.cuda.empty_cache()
    return X, idx, d2


def expanded_state(X, d, spread, seed):
    """Fixed expanded embedding: random 2-D projection of X, per-axis std =
    spread, so the h-driven grid reaches its largest size (the large-grid
    regime; a real run at this n stays on grids of 16-25 points)."""
    rng = np.random.default_rng(seed + 1)
    R = rng.standard_normal((X.shape[1], d)).astype(np.float32)
    Y = X @ R
    Y = (Y - Y.mean(0)) / Y.std(0) * spread
    return np.ascontiguousarray(Y.astype(np.float32))


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(nnz, n):
    """Per-launch DRAM bytes of the attractive SpMV from the committed ncu
    summary, scaled from its capture size to this launch (traffic grows with
    nnz and n)."""
    path = os.path.join(REPO, "profiles", "attr_spmv_traffic.txt")
    try:
        kv = {}
        for line in open(path):
            if ":" in line:
                k, v = line.split(":", 1)
                kv[k.strip()] = v.strip()
        b = float(kv["dram_bytes_per_launch"])
        alg = float(kv["algorithmic_bytes_per_launch"])
        return b / alg  # ratio applied to this launch's algorithmic bytes
    except Exception:
        return None


def spmv_alg_bytes(n, nnz, d):
    """Algorithmic bytes of one attractive SpMV launch: P stream (8 B per
    nonzero + rowptr), Y read once, F_attr written once."""
    S = 4 if d == 3 else d
    return 8 * nnz + 4 * (n + 1) + 4 * n * S * 2


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def initial_state(n, d, seed):
    """Y0 ~ N(0, 1e-4 I) (standard deviation 1e-2), seeded."""
    rng = np.random.default_rng(seed + 7)
    return (rng.standard_normal((n, d)) * 1e-2).astype(np.float32)


def build_problem(args, dev, ctx):
    """kNN on the device, then lambda bisection and (P + P^T)/(2n)
    through the engine on the device; returns (X, srp, sc, sv) on the
    host and the seconds the device pipeline took."""
    import torch

    X, idx, d2 = build_knn(args.n, args.seed, dev, ctx)
    t0 = time.perf_counter()
    n, k = idx.shape
    rp_knn = torch.arange(0, (n + 1) * k, k, dtype=torch.int32, device=dev)
    vals = d2.reshape(-1).contiguous().clone()
    col = idx.reshape(-1).to(torch.int32).contiguous()
    torch.cuda.synchronize(dev)  # torch's writes complete before the engine reads
    ctx.lambda_bisect(n, rp_knn, vals, 10.0, 1)
    nnz = int(col.numel())
    srp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    sc = torch.empty(2 * nnz, dtype=torch.int32, device=dev)
    sv = torch.empty(2 * nnz, dtype=torch.float32, device=dev)
    m = ctx.symmetrize(n, nnz, rp_knn, col, vals, 1.0 / (2 * n), srp, sc, sv)
    out = (srp.cpu().numpy(), sc[:m].cpu().numpy(), sv[:m].cpu().numpy())
    prep_s = time.perf_counter() - t0
    return X, out, (idx, d2), prep_s


def p_cache_path(n, seed):
    return os.path.join(tempfile.gettempdir(), f"sgtsne_b200_bench_P_n{n}_seed{seed}.npz")


def load_p_cache(n, seed):
    """P stored by the arm that ran first on this machine, or None."""
    path = p_cache_path(n, seed)
    try:
        z = np.load(path)
        srp, sc, sv = z["rowptr"], z["col"], z["val"]
        if len(srp) != n + 1 or int(srp[-1]) != len(sc) or len(sc) != len(sv):
            return None
        return srp, sc, sv.astype(np.float32), str(z["source"])
    except Exception:
        return None


def save_p_cache(n, seed, srp, sc, sv, source):
    """Store P for the other arm (written under a temporary name, then
    renamed, so a reader never sees a partial file)."""
    path = p_cache_path(n, seed)
    tmp = f"{path}.{os.getpid()}.tmp.npz"
    try:
        np.savez(tmp, rowptr=srp, col=sc, val=sv.astype(np.float32), source=np.array(source))
        os.replace(tmp, path)
    except OSError:
        pass


def compare_p(a, b):
    """How the engine-built P compares with the stored one: identical
    pattern, largest relative value difference, rows whose pattern differs."""
    (ra, ca, va), (rb, cb, vb) = a, b
    same_rp = len(ra) == len(rb) and np.array_equal(ra, rb)
    out = {"nnz_engine": int(ra[-1]), "nnz_stored": int(rb[-1])}
    if same_rp and np.array_equal(ca, cb):
        va64, vb64 = va.astype(np.float64), vb.astype(np.float64)
        out.update(pattern_identical=True,
                   val_max_rel=float(np.max(np.abs(va64 - vb64) / np.maximum(np.abs(vb64), 1e-30))),
                   val_rel_l2=float(np.linalg.norm(va64 - vb64) / np.linalg.norm(vb64)))
    else:
        n = len(rb) - 1
        diff = 0
        if len(ra) == len(rb):
            la, lb = np.diff(ra), np.diff(rb)
            diff = int(np.sum(la != lb))
            eq = np.flatnonzero(la == lb)
            # rows of equal length whose columns differ
            for r in eq[:: max(1, len(eq) // 20000)]:
                if not np.array_equal(ca[ra[r]:ra[r + 1]], cb[rb[r]:rb[r + 1]]):
                    diff += 1
        else:
            diff = n
        out.update(pattern_identical=False, rows_differing_sampled=diff)
    return out


def run_params(S, args):
    p = S.default_params(d=2, format=S.FORMAT_CSR, max_iter=1000, early_iter=250, h=0.7)
    p.lambda_ = 10.0
    p.relayout_every = args.relayout
    p.locality_order = args.locality_order
    return p


def run_knn_compare(n, seed, ctx, dev):
    """Both kNN methods on a bounded sample of the configuration's points
    (the first n of a fresh draw): CUDA-synchronised wall times and whether
    indices and distance bits agree.  A failure is reported, not raised."""
    import torch

    import sgtsne_b200 as S
    from sgtsne_b200 import workloads as W
    try:
        X, _ = W.gmm_zipf(n, dim=50, ncomp=40, zipf_a=1.1, centre_var=25.0, seed=seed + 7)
        Xd = torch.as_tensor(np.ascontiguousarray(X, np.float32), device=dev)
        res = {}
        for name, m in (("tensor", S.KNN_TENSOR), ("simt", S.KNN_SIMT)):
            idx = torch.empty(n * 30, dtype=torch.int32, device=dev)
            d2 = torch.empty(n * 30, dtype=torch.float32, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            redo = ctx.knn(n, 50, Xd, 30, idx, d2, method=m)
            res[name] = (time.perf_counter() - t0, idx.cpu().numpy(), d2.cpu().numpy(), redo)
        del Xd
        torch.cuda.empty_cache()
        (tt, it, dt, redo), (ts, is_, ds, _) = res["tensor"], res["simt"]
        return {"points": n, "dim": 50, "k": 30, "tensor_s": round(tt, 4), "simt_s": round(ts, 4),
                "speedup": round(ts / tt, 2), "redone_by_simt": redo,
                "identical": bool(np.array_equal(it, is_) and
                                  np.array_equal(dt.view(np.uint32), ds.view(np.uint32)))}
    except Exception as e:  # the comparison is informative only
        return {"points": n, "error": f"{type(e).__name__}: {e}"}


def run_ours(args, rank, world, local, dist):
    import torch

    import sgtsne_b200 as S
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    n, d = args.n, 2
    t_setup = time.time()
    ctx = S.Context(local)
    # one non-default stream for the engine and the timing events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    X, p_engine, (knn_idx, knn_d2), prep_s = build_problem(args, dev, ctx)
    t_setup = time.time() - t_setup
    # the P both arms time: the stored one if the other arm ran first here
    cached = load_p_cache(n, args.seed)
    if cached is not None:
        srp, sc, sv, p_source = cached
        p_match = compare_p(p_engine, (srp, sc, sv))
    else:
        srp, sc, sv = p_engine
        p_source, p_match = "engine (device kNN, lambda bisection, symmetrisation)", None
        save_p_cache(n, args.seed, srp, sc, sv, p_source)
    nnz = int(srp[-1])
    p = run_params(S, args)
    Y0 = initial_state(n, d, args.seed)
    W, K = max(args.warmup, 3), args.steps

    # ---- value: the run from Y0, device-resident inputs ----
    d_rp, d_c, d_v = (torch.from_numpy(srp).to(dev), torch.from_numpy(sc).to(dev),
                      torch.from_numpy(sv).to(dev))
    torch.cuda.synchronize()
    job = S.Job(ctx, p, d_rp, d_c, d_v, device_mem=True)
    job.set_y(torch.from_numpy(Y0).to(dev), S.LAYOUT_POINT_MAJOR, True)
    job.run(W)
    job.prepare()  # both iteration graphs exist before the timed region
    torch.cuda.synchronize()
    grid_start = job.info().grid_points
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, local)
    torch.cuda.synchronize()
    e0.record(stream)
    job.run(K)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(dist, local)
    clk = clocks.stop()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), dev)
    info = job.info()
    # the forces at the state the timed region ended in, through the
    # operators, for the parity check against the CPU restatement
    Yend = torch.empty(n, d, dtype=torch.float32, device=dev)
    job.get_y(Yend, S.LAYOUT_POINT_MAJOR, True, 1)
    fa = torch.empty(n * d, dtype=torch.float32, device=dev)
    fr = torch.empty(n * d, dtype=torch.float32, device=dev)
    ctx.attractive(S.FORMAT_CSR, n, d, nnz, d_rp, None, d_c, d_v, Yend, S.LAYOUT_POINT_MAJOR, fa)
    z_e, grid_e, _ = ctx.repulsive(n, d, 0.7, 0, Yend, S.LAYOUT_POINT_MAJOR, fr)
    torch.cuda.synchronize()
    parity_state = {"y": Yend.cpu().numpy(), "f_attr": fa.cpu().numpy().reshape(n, d),
                    "f_rep": fr.cpu().numpy().reshape(n, d), "z": z_e, "grid": grid_e}
    del fa, fr
    # per-stage durations on the same stream, continuing the run
    prof_iters = 20
    stage = job.profile(prof_iters)
    spmv_ms = stage[6] / prof_iters
    stage_avg = (stage / prof_iters).tolist()
    job.close()

    # ---- the large-grid regime: a fixed expanded embedding ----
    expanded = None
    if args.expanded:
        Ye = expanded_state(X, d, args.spread, args.seed)
        jobe = S.Job(ctx, p, d_rp, d_c, d_v, device_mem=True)
        jobe.set_y(torch.from_numpy(Ye).to(dev), S.LAYOUT_POINT_MAJOR, True)
        jobe.run(3)
        jobe.prepare()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        jobe.run(50)
        f1.record(stream)
        torch.cuda.synchronize()
        ste = jobe.profile(prof_iters)
        expanded = {"state": f"random 2-D projection of X, std {args.spread}",
                    "grid_points": jobe.info().grid_points,
                    "iters_per_s": 50 / (f0.elapsed_time(f1) / 1e3),
                    "stage_ms": dict(zip(["bin", "s2g", "g2g", "g2s", "attr+combine",
                                          "total_serial", "attr_spmv", "combine"],
                                         [round(x / prof_iters, 4) for x in ste]))}
        jobe.close()
        del Ye
    del X, d_rp, d_c, d_v

    # ---- e2e: the library entry (sgt_embed, the drop-in for the
    # reference's sgtsneCUDA) from pinned host buffers: the kNN graph in,
    # lambda bisection, symmetrisation, job creation, the whole
    # 1000-iteration run, the embedding back on the host ----
    k = knn_idx.shape[1]
    e_rp = torch.arange(0, (n + 1) * k, k, dtype=torch.int32).pin_memory()
    e_c = knn_idx.reshape(-1).to(torch.int32).cpu().pin_memory()
    e_v = knn_d2.reshape(-1).cpu().pin_memory()
    del knn_idx, knn_d2
    y_in = torch.from_numpy(np.ascontiguousarray(Y0.T)).pin_memory()  # dim-major
    y_out = torch.empty(d, n, dtype=torch.float32).pin_memory()
    pe = run_params(S, args)
    pe.max_iter = 1000
    pe.lambda_dist = 1
    # warm-up: one small call pages in the kernels of the preparation path
    # (lambda bisection, symmetrisation, locality order) the run uses first
    nw = 70000
    pw = run_params(S, args)
    pw.max_iter = 2
    ctx.embed(e_rp.numpy()[:nw + 1], e_c.numpy()[:nw * k] % nw, e_v.numpy()[:nw * k], pw)
    # three whole calls; the line reports the median (one call is one
    # embedding, and its wall time varies with the host)
    walls = []
    for _ in range(3):
        barrier(dist, local)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.embed(e_rp.numpy(), e_c.numpy(), e_v.numpy(), pe, y_in=y_in.numpy(),
                  y_out=y_out.numpy())
        t1 = time.perf_counter()
        barrier(dist, local)
        walls.append(max_over_ranks(dist, t1 - t0, dev))
    e2e_s = sorted(walls)[1]
    h2d = (e_rp.numel() * 4 + e_c.numel() * 4 + e_v.numel() * 4 + y_in.numel() * 4) / pe.max_iter
    d2h = y_out.numel() * 4 / pe.max_iter
    e2e = {"value": world * pe.max_iter / e2e_s, "unit": "iters/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "includes": "sgt_embed (the library entry) from pinned host buffers: the kNN graph "
                       "(k = 30 squared distances) in, lambda = 10 bisection, (P+P^T)/(2n), job "
                       "creation, the whole 1000-iteration run, the embedding back on the host",
           "wall_s": e2e_s, "wall_s_calls": [round(w, 4) for w in walls]}
    del e_rp, e_c, e_v

    batched = served = knn_cmp = None
    if rank == 0 and args.knn_compare > 0:
        knn_cmp = run_knn_compare(args.knn_compare, args.seed, ctx, dev)
    if rank == 0 and args.batched:
        batched = run_batched_leg(args, ctx, stream, dev)
    if rank == 0 and args.served:
        served = run_served_leg(args, ctx, local)

    out = None
    if rank == 0:
        alg = spmv_alg_bytes(n, nnz, d)
        hbm, src = peaks()
        achieved = alg / (spmv_ms / 1e3) / 1e9
        ratio = read_traffic(nnz, n)
        # bin count (with the tile scan in its last block), bin scatter,
        # s2g (tile + cell), fft x3, g2s, SpMV, combine
        per_iter_kernels = 10
        # a relayout before every R-th iteration: cell keys, two 3-kernel
        # scans, key scatter, permutation prep, row relabel, 3 gathers
        R = args.relayout
        relayouts = 0 if R <= 0 else (W + K - 1) // R - (W - 1) // R
        launches = per_iter_kernels * K + 13 * relayouts
        value = world * K / (ms / 1e3)
        out = {
            "metric": METRIC, "value": value, "unit": "iters/s",
            "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_ITERS_PER_S,
            "dtype": "f32 (FP64 Z/KL/row-sum reductions)",
            "data": "synthetic (seeded generator with the configuration's shapes)",
            "config": {"workload": WORKLOAD, "n": n, "d": d, "nnz": nnz, "format": "csr",
                       "parallelism": f"replicas x{world}",
                       "timed_state": f"iterations {W + 1}..{W + K} of the run from "
                                      "Y0 ~ N(0, 1e-4 I)",
                       "p_source": p_source, "p_engine_vs_stored": p_match,
                       "grid_points_start": grid_start, "grid_points_end": info.grid_points,
                       "h_eff_end": round(info.h_eff, 5), "row_group": info.row_group,
                       "relayout_every": args.relayout,
                       "row_group_tune_ms": [round(x, 4) for x in info.tune_ms],
                       "l2": "inputs larger than L2 (P >= 400 MB), no flush",
                       "stage_ms": dict(zip(["bin", "s2g", "g2g", "g2s", "attr+combine",
                                             "total_serial", "attr_spmv", "combine"],
                                            [round(x, 4) for x in stage_avg])),
                       "stage_note": "stages run one after another on one stream; the "
                                     "timed iteration runs the SpMV beside the repulsion",
                       "setup_s": round(t_setup, 1), "p_prep_s": round(prep_s, 2),
                       "knn_s": None if KNN_SECONDS[0] is None else round(KNN_SECONDS[0], 2),
                       "knn": "sgt_knn, exact: the tcgen05 tensor-core filter (50-D, k = 30) "
                              "re-ranked with the SIMT arithmetic",
                       "expanded_state": expanded},
            "roofline": {"bound": "hbm", "kernel": "k_attr_rows (CSR attractive SpMV)",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_source": src,
                         "algorithmic_bytes_per_launch": alg,
                         "traffic": None if ratio is None else ratio * alg},
            "e2e": e2e,
            # the engine has one arithmetic form (FP32 SpMV, scatter, FFT and
            # gather; FP64 Z, KL and row sums), the precision form of the
            # north star without its optional split-BF16 DFT-GEMM convolution;
            # the convolution's share bounds what a faster convolution can give
            "precision": {
                "form": "FP32 SpMV/S2G/FFT/G2S with FP32 accumulation; FP64 Z, KL, row sums",
                "split_bf16_dft_gemm_convolution": "not built",
                "convolution_ms": round(stage_avg[2], 4),
                "convolution_share_of_serial_iteration": round(stage_avg[2] / stage_avg[5], 4),
                "iteration_speedup_if_convolution_were_free":
                    round(1.0 / (1.0 - stage_avg[2] / stage_avg[5]), 4)},
            "gpu_launches": launches,
            "clocks": clk,
            "knn_compare": knn_cmp,
            "batched": batched,
            "served": served,
        }
    ctx.close()
    return out, (srp, sc, sv, Y0, parity_state)


def run_batched_leg(args, ctx, stream, dev):
    """The batched configuration (a bounded sample of its 256 instances):
    plain = each job's iterations one job after another; batched = every
    job in one CUDA graph.  Embeddings/s = jobs / time of `iters`."""
    import sgtsne_b200 as S
    from sgtsne_b200 import multi as Mu
    t = time.time()
    inst = Mu.batched_instances(ctx, args.batch_jobs, args.seed, dev)
    setup = time.time() - t
    r = Mu.run_batched(S, ctx, inst, args.batch_iters, stream, iters_per_launch=8)
    njobs = len(inst)
    out = {"workload": "independent embeddings, n log-uniform in [2000, 200000], dim U{20..100}, "
                       "isotropic mixture (5-30 components, seed per instance), k=30, lambda=1, "
                       "half d=2 / half d=3",
           "jobs": njobs, "of_configured": 256, "iters": args.batch_iters,
           "total_points": int(sum(i["n"] for i in inst)),
           "plain_embeds_per_s": njobs / (r["plain_ms"] / 1e3),
           "batched_embeds_per_s": njobs / (r["batched_ms"] / 1e3),
           "speedup": r["plain_ms"] / r["batched_ms"], "iters_per_launch": 8,
           "error_flags": r["error_flags"], "setup_s": round(setup, 1),
           "timing": "CUDA events on the engine stream; device-resident P and Y0"}
    return out


def run_served_leg(args, ctx, local):
    """The served configuration (a bounded sample of its 2000 requests):
    plain = each request alone through the public API, one after another
    (service times measured, latencies of a FIFO single server under the
    same arrivals); served = the continuous-batching server under an
    open-loop Poisson stream at multiples of the plain capacity, and with
    every request arriving at once (saturation)."""
    import sgtsne_b200 as S
    from sgtsne_b200 import multi as Mu
    t = time.time()
    req = Mu.request_instances(ctx, args.serve_requests, args.seed + 1, f"cuda:{local}")
    setup = time.time() - t
    svc = Mu.plain_service_times(S, ctx, req)
    cap = 1.0 / float(np.mean(svc))
    nr = len(req)
    kw = {"max_active": args.serve_active, "iters_per_round": 16, "rounds_ahead": 2,
          "hbm_budget": 150 << 30}
    rows = []
    for mult in args.serve_rates:
        rate = mult * cap
        arr = np.cumsum(np.random.default_rng(args.seed + 3).exponential(1.0 / rate, nr))
        arr -= arr[0]
        lat, mk, states = Mu.serve_stream(S, req, arr, device=local, **kw)
        pl = Mu.fifo_latencies(arr, svc)
        rows.append({"rate_per_s": rate, "x_plain_capacity": mult,
                     "served_embeds_per_s": nr / mk,
                     "served": Mu.percentiles(lat), "plain": Mu.percentiles(pl),
                     "all_done": all(x == S.REQ_DONE for x in states)})
    arr = np.zeros(nr)
    lat, mk, states = Mu.serve_stream(S, req, arr, device=local, **kw)
    pl = Mu.fifo_latencies(arr, svc)
    sat = {"served_embeds_per_s": nr / mk, "plain_embeds_per_s": cap,
           "speedup": (nr / mk) / cap, "served": Mu.percentiles(lat),
           "plain": Mu.percentiles(pl), "all_done": all(x == S.REQ_DONE for x in states)}
    return {"workload": "requests with n log-uniform in [1000, 500000], d in {2,3}, "
                        "lambda in {1,10,30}, 500-1000 iterations, P from the 50-D 40-component "
                        "Zipf(1.1) mixture (seed per request), 150 GB HBM budget",
            "requests": nr, "of_configured": 2000,
            "total_points": int(sum(i["n"] for i in req)),
            "plain_service_s": {"mean": float(np.mean(svc)), "sum": float(np.sum(svc))},
            "server": kw, "open_loop": rows, "saturation": sat, "setup_s": round(setup, 1),
            "latency": "scheduled arrival to coordinates in the caller's host buffer"}


def cpu_sample(srp, sc, sv, Ystate, iters, threads):
    """The oracle (FP64 CPU path: CSR SpMV, FFT repulsion, update) on the
    same P and state; returns seconds per iteration and the state after."""
    from oracle import oracle as O
    Y = Ystate.astype(np.float64)
    t = time.perf_counter()
    Y = O.kl_minimization(srp, sc, sv.astype(np.float64), Y, iters, early_iter=250, alpha=12.0,
                          h=0.7, grid_mode=0, nthreads=threads)
    return (time.perf_counter() - t) / iters, Y


def parity_check(srp, sc, sv, st, threads):
    """The checker at full size: the oracle's FP64 attractive and
    interpolated repulsive forces at the coordinates the timed region ended
    in (same grid), against the engine's operators on the same state."""
    from oracle import oracle as O
    Y = st["y"].astype(np.float64)
    fa = O.attractive(srp, sc, sv.astype(np.float64), Y, nthreads=threads)
    fr, z, grid, _ = O.repulsive_interp(Y, 0.7, n1_force=st["grid"] - 2, nthreads=threads)

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return {"state": "centred coordinates after the timed region", "grid_points": int(st["grid"]),
            "grid_points_oracle": int(grid),
            "f_attr_rel_l2": rel(st["f_attr"].astype(np.float64), fa),
            "f_rep_rel_l2": rel(st["f_rep"].astype(np.float64), fr),
            "z_rel": abs(st["z"] - z) / abs(z),
            "bars": {"f_attr": 1e-5, "f_rep": 3e-4, "z": 5e-4},
            "checker": "FP64 CPU restatement of the reference (oracle/)"}


def run_reference(args, rank, world, local, dist):
    """The reference's CPU path, restated by the oracle (the reference's own
    CPU code needs Cilk Plus and FFTW, absent here), with all host threads,
    on the same P as the engine arm (stored by whichever arm ran first; built
    here with torch matrix products for the kNN and the oracle for lambda
    and symmetrisation when this arm runs first).  The engine library is not
    loaded."""
    if rank != 0:
        return None
    import torch
    from oracle import oracle as O
    n = args.n
    cached = load_p_cache(n, args.seed)
    if cached is not None:
        srp, sc, sv, p_source = cached
    else:
        from sgtsne_b200 import workloads as Wl  # pure Python: generator and torch kNN
        X, _ = Wl.gmm_zipf(n, dim=50, ncomp=40, zipf_a=1.1, centre_var=25.0, seed=args.seed)
        if torch.cuda.is_available():
            idx, d2 = Wl.knn_torch(X, 30, device=f"cuda:{local}", block=2048)
            idx, d2 = idx.cpu().numpy(), d2.cpu().numpy()
            torch.cuda.empty_cache()
        else:
            idx, d2 = Wl.knn_numpy(X, 30)
        del X
        k = idx.shape[1]
        rp = (np.arange(n + 1, dtype=np.int64) * k).astype(np.int32)
        col = idx.reshape(-1).astype(np.int32)
        v, _ = O.lambda_rescale(rp, d2.reshape(-1).astype(np.float64), 10.0, dist=True)
        srp, sc, sv = O.symmetrize(rp, col, v, 1.0 / (2 * n))
        sv = sv.astype(np.float32)
        p_source = "torch kNN (FP32 matrix products) + oracle lambda bisection and symmetrisation"
        save_p_cache(n, args.seed, srp, sc, sv, p_source)
    Ystate = initial_state(n, 2, args.seed)
    threads = os.cpu_count() or 1
    steps = args.steps if args.ref_steps is None else max(1, min(args.steps, args.ref_steps))
    warm = max(3, args.warmup)
    _, Yw = cpu_sample(srp, sc, sv, Ystate, warm, threads)
    spi, _ = cpu_sample(srp, sc, sv, Yw.astype(np.float32), steps, threads)
    val_ = 1.0 / spi
    return {
        "metric": METRIC, "impl": "reference", "value": val_, "unit": "iters/s", "n_gpus": world,
        "steps": steps, "warmup": warm, "ms_per_step": spi * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": val_ / PUBLISHED_ITERS_PER_S,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "d": 2, "nnz": int(srp[-1]), "format": "csr",
                   "p_source": p_source,
                   "timed_state": f"iterations {warm + 1}..{warm + steps} of the run from "
                                  "Y0 ~ N(0, 1e-4 I)"},
        "cpu_baseline": {"value": val_, "unit": "iters/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full iterations at n={n} after {warm} warm-up "
                                   "iterations from Y0"},
        "e2e": {"value": val_, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=995)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1300000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--spread", type=float, default=60.0)
    ap.add_argument("--cpu-iters", type=int, default=2)
    ap.add_argument("--ref-steps", type=int, default=None,
                    help="cap on the reference arm's timed iterations (default: --steps)")
    ap.add_argument("--relayout", type=int, default=200,
                    help="relabel points along the cell Morton order every R iterations (0 = off)")
    ap.add_argument("--no-expanded", dest="expanded", action="store_false",
                    help="skip the fixed expanded-state (largest grid) line")
    ap.add_argument("--no-cpu", dest="cpu", action="store_false")
    ap.add_argument("--locality-order", type=int, default=1, choices=[0, 1],
                    help="sgt_params.locality_order of every job (1: the engine default)")
    ap.add_argument("--knn-compare", type=int, default=200000,
                    help="points of the tensor-core vs SIMT kNN comparison (0 = skip)")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the batched-embeddings line")
    ap.add_argument("--batch-jobs", type=int, default=64)
    ap.add_argument("--batch-iters", type=int, default=1000)
    ap.add_argument("--no-served", dest="served", action="store_false",
                    help="skip the served request-stream line")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-active", type=int, default=32)
    ap.add_argument("--serve-rates", type=float, nargs="*", default=[2.0, 4.0])
    args = ap.parse_args()
    from sgtsne_b200 import multi as _multi
    _multi.LOCALITY_ORDER = args.locality_order
    rank, world, local = dist_env()
    import torch
    dist = dist_init(world, "nccl" if torch.cuda.is_available() else "gloo")
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world, local, dist)
        else:
            out, prob = run_ours(args, rank, world, local, dist)
            if rank == 0 and world == 1 and args.cpu and out is not None:
                srp, sc, sv, Y0, pstate = prob
                threads = os.cpu_count() or 1
                # the checker at full size, then the CPU baseline sample
                out["parity"] = parity_check(srp, sc, sv, pstate, threads)
                par = out["parity"] or {}
                out["precision"]["error_vs_fp64"] = {
                    k: par.get(k) for k in ("f_attr_rel_l2", "f_rep_rel_l2", "z_rel")}
                spi, _ = cpu_sample(srp, sc, sv, pstate["y"], args.cpu_iters, threads)
                out["cpu_baseline"] = {"value": 1.0 / spi, "unit": "iters/s", "cores": threads,
                                       "kind": "port",
                                       "sample": f"{args.cpu_iters} full iterations at n={args.n} "
                                                 "from the state the timed region ended in, "
                                                 "FP64 oracle"}
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
