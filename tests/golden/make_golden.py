"""Generate golden vectors from the reference's own CUDA kernels.

Run on a machine with a B200 after `bash oracle/build_ref.sh` (which compiles the
reference sources in place into oracle/_ref/):

    python tests/golden/make_golden.py OUTDIR

Writes ref_*.npz into OUTDIR (copy them to tests/golden/).  Inputs are
seeded; the reference functions called are
  ref_hyb_repulsive       HYB/cuda/Frep.cu:142-175 (FP64, h-driven grid)
  ref_cu_attractive_coo   CU/pq.cu:24-57 (FP32, COO format)
  ref_cu_repulsive_fixed  CU/Frep.cu:81-125 (FP32, fixed grid getBestGridSize(ng))
"""
import ctypes as C
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, os.path.join(REPO, "gpu-sg-sne_b200", "python"))


def main(out):
    os.makedirs(out, exist_ok=True)
    hyb = C.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_hyb.so"))
    cu = C.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_cu.so"))
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    hyb.ref_hyb_repulsive.restype = C.c_double
    hyb.ref_hyb_repulsive.argtypes = [C.c_int, C.c_int, C.c_double, dp, dp]
    cu.ref_cu_attractive_coo.restype = C.c_int
    cu.ref_cu_attractive_coo.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, fp, fp, fp]
    cu.ref_cu_repulsive_fixed.restype = C.c_float
    cu.ref_cu_repulsive_fixed.argtypes = [C.c_int, C.c_int, C.c_int, fp, fp, C.POINTER(C.c_int)]

    # 1. FP64 repulsion: the reference's installation-test inputs (U(0,1)^d,
    #    HYB/test_modules.cpp:122-156) plus a wide clustered 2-D case
    cases = []
    for d in (1, 2, 3):
        for h in (0.05, 0.13):
            rng = np.random.default_rng(100 * d + int(h * 100))
            cases.append((f"u{d}_{h}", rng.random((2000, d)), h))
    rng = np.random.default_rng(7)
    c = rng.standard_normal((6, 2)) * 15
    cases.append(("clusters2_0.7", c[rng.integers(0, 6, 5000)] + rng.standard_normal((5000, 2)), 0.7))
    for name, Y, h in cases:
        Y = np.ascontiguousarray(Y, np.float64)
        n, d = Y.shape
        F = np.zeros((n, d), np.float64)
        Z = hyb.ref_hyb_repulsive(n, d, h, Y, F)
        np.savez_compressed(os.path.join(out, f"ref_hyb_rep_{name}.npz"), y=Y, h=h, F=F, Z=Z)
        print("hyb", name, Z)

    # 2. FP32 attractive term, COO format
    from conftest import make_problem
    for d in (1, 2, 3):
        rp, col, val, _ = make_problem(n=3000, k=12, seed=30 + d)
        n = len(rp) - 1
        rows = np.repeat(np.arange(n), np.diff(rp)).astype(np.int32)
        Y = (np.random.default_rng(40 + d).standard_normal((n, d)) * 3).astype(np.float32)
        v32 = val.astype(np.float32)
        F = np.zeros(n * d, np.float32)
        e = cu.ref_cu_attractive_coo(n, d, int(rp[-1]), rows, col.astype(np.int32), v32,
                                     np.ascontiguousarray(Y.T.reshape(-1)), F)
        assert e == 0
        np.savez_compressed(os.path.join(out, f"ref_cu_attr_d{d}.npz"), rowptr=rp, col=col,
                            val=v32, y=Y, F=F.reshape(d, n).T.copy())
        print("cu attr", d)

    # 3. FP32 fixed-grid repulsion (ng = 50): d = 1 and d = 2
    for d in (1, 2):
        rng = np.random.default_rng(50 + d)
        Y = (rng.standard_normal((4000, d)) * 4).astype(np.float32)
        F = np.zeros(4000 * d, np.float32)
        g = C.c_int()
        Z = cu.ref_cu_repulsive_fixed(4000, d, 50, np.ascontiguousarray(Y.T.reshape(-1)), F,
                                      C.byref(g))
        np.savez_compressed(os.path.join(out, f"ref_cu_rep_fixed_d{d}.npz"), y=Y, ng=50,
                            F=F.reshape(d, 4000).T.copy(), Z=Z, grid=g.value)
        print("cu rep fixed", d, Z, g.value)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py OUTDIR")
    main(sys.argv[1])
