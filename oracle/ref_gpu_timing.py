"""Times the reference's own GPU gradient-descent loop (kl_minimization of
code/cuda/SG-tSNE-CUDA/src/gradient_descend.cu:102-282, compiled for sm_100a
from the reference sources by oracle/build_ref.sh) beside this engine, on the
same P, Y0 and fixed grid, on one B200.

The reference loop runs on the fixed grid of its command line tool (-g ng,
default 50); both are timed there and on the grids a real 1.3M-point run
uses (16 and 25 points per axis).  The reference times its loop itself
(wall clock after its allocations and FFT plans; timeInfo[7000]); this
engine is timed with CUDA events around sgt_job_run.

  python oracle/ref_gpu_timing.py [--n 1300000] [--iters 30]

Measurement only (prints a markdown table); needs oracle/_ref/libref_cu.so.
"""
import argparse
import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "gpu-sg-sne_b200", "python"))


def load_ref():
    lib = C.CDLL(os.path.join(HERE, "_ref", "libref_cu.so"))
    f = lib.ref_cu_kl_minimization
    f.restype = C.c_double
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    return f


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1300000)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import torch

    import bench as B
    import sgtsne_b200 as S
    ref = load_ref()
    dev = "cuda:0"
    ctx = S.Context(0)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    t = time.time()
    X, srp, sc, sv = B.build_problem(args, dev, ctx)
    del X
    n, d, nnz = args.n, 2, int(srp[-1])
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(srp)).astype(np.int32)
    w = S.ell_width(srp)
    ec, ev, cr, cc, cv = S.csr_to_hybrid(srp, sc, sv, w)
    y0 = B.initial_state(n, d, args.seed)
    y0_dm = np.ascontiguousarray(y0.T)
    print(f"setup {time.time() - t:.1f}s  n={n} nnz={nnz} ell_width={w} coo_tail={len(cr)}",
          flush=True)

    def ref_rate(fmt, ng):
        y = y0_dm.copy()
        a = (srp if fmt == 0 else rows) if fmt != 3 else None
        call = lambda it, yy: ref(fmt, n, d, nnz, it, ng, ptr(a), ptr(sc if fmt != 3 else None),
                                  ptr(sv if fmt != 3 else None), w, ptr(ec), ptr(ev), len(cr),
                                  ptr(cr), ptr(cc), ptr(cv), ptr(yy))
        if call(3, y.copy()) < 0:
            return None
        ms = call(args.iters, y)
        return None if ms < 0 else args.iters / (ms / 1e3)

    def ours_rate(ng, fmt):
        p = S.default_params(d=d, format=fmt, max_iter=1000, early_iter=250, h=0.7)
        if ng > 0:
            p.grid_mode = S.GRID_FIXED
            p.ng = ng
        job = S.Job(ctx, p, torch.from_numpy(srp).to(dev), torch.from_numpy(sc).to(dev),
                    torch.from_numpy(sv).to(dev), device_mem=True)
        job.set_y(torch.from_numpy(y0).to(dev), S.LAYOUT_POINT_MAJOR, True)
        job.run(3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        job.run(args.iters)
        e1.record(stream)
        torch.cuda.synchronize()
        grid = job.info().grid_points
        job.close()
        return args.iters / (e0.elapsed_time(e1) / 1e3), grid

    print("| grid (points/axis) | reference CSR (fmt 0) | reference COO (fmt 2) | "
          "reference ELL+COO (fmt 3) | engine CSR | engine COO | engine ELL+COO | "
          "engine CSR / best reference |")
    print("|---|---|---|---|---|---|---|---|")
    for ng in (14, 23, 50):
        r = {f: ref_rate(f, ng) for f in (0, 2, 3)}
        o = {f: ours_rate(ng, f) for f in (0, 2, 3)}
        best = max(v for v in r.values() if v is not None)
        fmt = lambda v: "failed" if v is None else f"{v:.1f} it/s"
        print(f"| {o[0][1]} | {fmt(r[0])} | {fmt(r[2])} | {fmt(r[3])} | "
              f"{o[0][0]:.0f} it/s | {o[2][0]:.0f} it/s | {o[3][0]:.0f} it/s | "
              f"{o[0][0] / best:.0f}x |", flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
