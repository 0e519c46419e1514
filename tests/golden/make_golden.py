"""Generate golden vectors from the reference's own CUDA kernels.

Run on a machine with a B200 after `bash oracle/build_ref.sh` (which compiles the
reference sources in place into oracle/_ref/):

    python tests/golden/make_golden.py OUTDIR

Writes ref_*.npz into OUTDIR (copy them to tests/golden/).  Inputs are
seeded; the reference functions called are
  ref_hyb_repulsive       HYB/cuda/Frep.cu:142-175 (FP64, h-driven grid)
  ref_cu_attractive_coo   CU/pq.cu:24-57 (FP32, COO format)
  ref_cu_repulsive_fixed  CU/Frep.cu:81-125 (FP32, fixed grid getBestGridSize(ng))
  ref_cu_kl_minimization  CU/gradient_descend.cu:102-282 (FP32, the whole loop on
                          the fixed grid; d = 1, which the d >= 2 layout defect of
                          CU/gridding.cu does not touch)
  ref_cu_tsne_cost_f32/64 CU/pq.cu:104-125 (tsneCost, float and double)
  ref_cu_perplexity       CU/perplexity_search.cu:113-208 (perplexityEqualization)
  ref_cu_lambda_rescale   CU/graph_rescaling.cu:11-107 (bisectionSearchKernel)
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

    # 4. the reference's whole loop: d = 1, fixed grid ng = 50, CSR, from one
    #    Y0; separate runs of 10, 50 and 300 iterations (alpha = 12 for the
    #    first 251, momentum 0.5 -> 0.8 after iteration 250), each ending
    #    with the reference's mean centring
    kl = cu.ref_cu_kl_minimization
    kl.restype = C.c_double
    kl.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    rp, col, val, _ = make_problem(n=2000, k=15, seed=61)
    n = len(rp) - 1
    v32 = val.astype(np.float32)
    c32 = col.astype(np.int32)
    y0 = (np.random.default_rng(62).standard_normal(n) * 1e-4).astype(np.float32)
    traj = {}
    for it in (10, 50, 300):
        y = y0.copy()
        ms = kl(0, n, 1, int(rp[-1]), it, 50, rp.ctypes.data, c32.ctypes.data, v32.ctypes.data,
                0, None, None, 0, None, None, None, y.ctypes.data)
        assert ms >= 0, ms
        traj[f"y{it}"] = y
        print("cu kl_minimization", it, float(np.abs(y).max()))
    np.savez_compressed(os.path.join(out, "ref_cu_kl_traj_d1.npz"), rowptr=rp, col=c32, val=v32,
                        y0=y0, ng=50, **traj)

    # 5. tsneCost (COO, dim-major Y), float and double, exaggerated and not
    cu.ref_cu_tsne_cost_f32.restype = C.c_float
    cu.ref_cu_tsne_cost_f32.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, fp, fp, C.c_float,
                                        C.c_float]
    cu.ref_cu_tsne_cost_f64.restype = C.c_double
    cu.ref_cu_tsne_cost_f64.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, dp, dp, C.c_double,
                                        C.c_double]
    from oracle import oracle as O
    for d in (1, 2, 3):
        rp, col, val, _ = make_problem(n=3000, k=12, seed=70 + d)
        n = len(rp) - 1
        rows = np.repeat(np.arange(n), np.diff(rp)).astype(np.int32)
        c32 = col.astype(np.int32)
        v32 = val.astype(np.float32)
        Y = (np.random.default_rng(80 + d).standard_normal((n, d)) * 3).astype(np.float32)
        _, Z, _, _ = O.repulsive_interp(Y.astype(np.float64), 0.7)
        ydm32 = np.ascontiguousarray(Y.T.reshape(-1))
        ydm64 = ydm32.astype(np.float64)
        res = {}
        for alpha in (1.0, 12.0):
            res[f"c32_a{int(alpha)}"] = cu.ref_cu_tsne_cost_f32(n, d, int(rp[-1]), rows, c32, v32,
                                                                ydm32, alpha, float(Z))
            res[f"c64_a{int(alpha)}"] = cu.ref_cu_tsne_cost_f64(n, d, int(rp[-1]), rows, c32,
                                                                v32.astype(np.float64), ydm64,
                                                                alpha, float(Z))
        np.savez_compressed(os.path.join(out, f"ref_cu_cost_d{d}.npz"), rowptr=rp, col=c32,
                            val=v32, y=Y, zeta=np.float32(Z), **res)
        print("cu cost", d, res)

    # 6. perplexityEqualization: kNN lists with the point itself first (at
    #    distance 0) and squared distances divided by their maximum
    from sgtsne_b200 import workloads as W
    cu.ref_cu_perplexity.restype = C.c_int
    cu.ref_cu_perplexity.argtypes = [C.c_int, C.c_int, ip, fp, C.c_float, ip, ip, fp]
    for (n, dim, nn, u, seed) in ((2000, 20, 60, 20.0, 90), (1500, 50, 90, 30.0, 91)):
        X, _ = W.gmm_isotropic(n, dim, 8, 16.0, seed)
        idx, d2 = W.knn_numpy(X, nn)
        I = np.concatenate([np.arange(n)[:, None], idx], 1).astype(np.int32)
        D = np.concatenate([np.zeros((n, 1)), d2], 1)
        D = (D / D.max()).astype(np.float32)
        orow = np.empty(n + 1, np.int32)
        ocol = np.empty(n * nn, np.int32)
        oval = np.empty(n * nn, np.float32)
        e = cu.ref_cu_perplexity(n, nn, np.ascontiguousarray(I), np.ascontiguousarray(D),
                                 u, orow, ocol, oval)
        assert e == 0
        np.savez_compressed(os.path.join(out, f"ref_cu_perplexity_n{n}_k{nn}.npz"), I=I, D=D,
                            u=np.float32(u), rowptr=orow, col=ocol, val=oval)
        print("cu perplexity", n, nn)

    # 7. the lambda bisection on raw values (the distances), with rows of
    #    uneven length, single-entry rows, and with / without dropping leaves
    rs = C.CDLL(os.path.join(REPO, "oracle", "_ref", "libref_rescale.so"))
    rs.ref_cu_lambda_rescale.restype = C.c_int
    rs.ref_cu_lambda_rescale.argtypes = [C.c_int, ip, fp, C.c_float, C.c_int]
    X, _ = W.gmm_isotropic(3000, 16, 6, 16.0, 95)
    idx, d2 = W.knn_numpy(X, 14)
    rng = np.random.default_rng(96)
    lens = rng.integers(1, 15, size=3000)
    lens[::50] = 1
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([idx[i, :lens[i]] for i in range(3000)]).astype(np.int32)
    dist = np.concatenate([d2[i, :lens[i]] for i in range(3000)]).astype(np.float32)
    for lam, drop in ((10.0, 0), (3.0, 1), (1.0, 0)):
        v = dist.copy()
        e = rs.ref_cu_lambda_rescale(3000, rp, v, lam, drop)
        assert e == 0
        np.savez_compressed(os.path.join(out, f"ref_cu_lambda_{int(lam)}_drop{drop}.npz"),
                            rowptr=rp, col=col, dist=dist, lam=np.float32(lam), drop=drop, val=v)
        print("cu lambda", lam, drop)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py OUTDIR")
    main(sys.argv[1])
