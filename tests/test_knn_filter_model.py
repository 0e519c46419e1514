"""A CPU model of the tensor-core kNN filter (k_knn_tc in
gpu-sg-sne_b200/csrc/sgt_knn.cu): its error bound and its settling rule.

1. Error of the approximate distance.  The augmented rows (q, 1, -|q|^2/2)
   and (c, -|c|^2/2, 1) are split into TF32 hi + lo parts (round to nearest,
   ties away, 10 explicit mantissa bits, as cvt.rna.tf32.f32).  The three
   products hi.hi + hi.lo + lo.hi are summed in FP32, eight products per MMA
   step, steps accumulated in K order.  The largest error of -2 D relative to
   |q|^2 + |c|^2 stays below a quarter of the kernel's bound EPS = 1e-4.
   The inputs are the 50-D generator of the 1.3M-point configuration,
   integer lattice points, and a small cloud far from the origin.  The
   hardware's summation order inside an MMA is not modelled bit for bit; the
   factor four is the margin for it.
2. The settling rule.  Each query keeps the 64 smallest approximate
   distances, then re-ranks them with exact distances.  It is settled when
   the list's largest approximate distance minus the bound exceeds the k-th
   exact distance.  With errors within the bound, every settled query has
   the exact k nearest.  With errors fifty times the bound, the same rule
   settles some queries wrongly, so the bound is what makes the rule exact.
"""
import numpy as np
import pytest

EPS = 1e-4
CAP = 64


def tf32(x):
    """cvt.rna.tf32.f32: keep 10 explicit mantissa bits, ties away from 0."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).astype(np.uint32)
    return r.view(np.float32)


def augmented(X, role):
    n, dim = X.shape
    nrm = np.zeros(n, np.float32)
    for kk in range(dim):  # FP32 norms in dimension order, as k_knn_norms
        nrm = (nrm + X[:, kk] * X[:, kk]).astype(np.float32)
    kp = ((dim + 2 + 7) // 8) * 8
    R = np.zeros((n, kp), np.float32)
    R[:, :dim] = X
    half = (np.float32(-0.5) * nrm).astype(np.float32)
    if role == "query":
        R[:, dim], R[:, dim + 1] = 1.0, half
    else:
        R[:, dim], R[:, dim + 1] = half, 1.0
    return R, nrm


def approx_d2(X):
    """-2 D of every pair under the model above (FP32 throughout)."""
    A, nrm = augmented(X, "query")
    B, _ = augmented(X, "cand")
    ah = tf32(A)
    al = tf32((A - ah).astype(np.float32))
    bh = tf32(B)
    bl = tf32((B - bh).astype(np.float32))
    n, kp = A.shape
    acc = np.zeros((n, n), np.float32)
    for ks in range(0, kp, 8):
        for (a, b) in ((ah, bh), (ah, bl), (al, bh)):
            part = np.zeros((n, n), np.float32)
            for kk in range(ks, ks + 8):
                # products of TF32 values are exact in FP32
                part = (part + np.outer(a[:, kk], b[:, kk]).astype(np.float32)).astype(np.float32)
            acc = (acc + part).astype(np.float32)
    return (np.float32(-2.0) * acc).astype(np.float32), nrm


def exact_d2(X):
    """FP64 sums of squared differences (no cancellation)."""
    X64 = X.astype(np.float64)
    D = np.empty((len(X64), len(X64)))
    for i in range(len(X64)):
        D[i] = ((X64[i] - X64) ** 2).sum(1)
    return D


@pytest.mark.parametrize("kind", ["zipf", "lattice", "offset"])
def test_error_within_bound(kind):
    rng = np.random.default_rng(11)
    if kind == "zipf":
        from sgtsne_b200 import workloads as W
        X, _ = W.gmm_zipf(700, dim=50, ncomp=40, zipf_a=1.1, centre_var=25.0, seed=5)
    elif kind == "lattice":
        X = rng.integers(0, 40, (700, 7))
    else:
        X = 1000.0 + 0.1 * rng.standard_normal((500, 16))
    X = np.ascontiguousarray(X, np.float32)
    Da, nrm = approx_d2(X)
    D = exact_d2(X)
    scale = nrm.astype(np.float64)[:, None] + nrm.astype(np.float64)[None, :]
    rel = np.abs(Da.astype(np.float64) - D) / np.maximum(scale, 1e-30)
    worst = float(rel.max())
    print(f"\n{kind}: largest |d~ - d| / (|q|^2 + |c|^2) = {worst:.2e} (bound {EPS:.0e})")
    assert worst <= EPS / 4


def settle(D, Dap, bound, k):
    """The kernel's list, re-rank and settling rule for every query.
    Returns (settled mask, indices of the k nearest per settled query)."""
    n = len(D)
    Dap = Dap.copy()
    np.fill_diagonal(Dap, np.inf)  # the kernel drops the query at the re-rank
    settled = np.zeros(n, bool)
    out = np.full((n, k), -1)
    for q in range(n):
        lst = np.argpartition(Dap[q], CAP)[:CAP]
        tail = Dap[q, lst].max()
        order = lst[np.lexsort((lst, D[q, lst]))]
        dk = D[q, order[k - 1]]
        if tail - bound[q] > dk:
            settled[q] = True
            out[q] = order[:k]
    return settled, out


def truth(D, k):
    n = len(D)
    Dx = D.copy()
    np.fill_diagonal(Dx, np.inf)
    idx = np.arange(n)
    return np.array([np.lexsort((idx, Dx[q]))[:k] for q in range(n)])


def test_settling_rule_exact_within_bound_and_wrong_beyond():
    rng = np.random.default_rng(3)
    n, dim, k = 1500, 6, 10
    c = rng.standard_normal((6, dim)) * 3
    X = (c[rng.integers(0, 6, n)] + rng.standard_normal((n, dim))).astype(np.float64)
    D = exact_d2(X)
    T = truth(D, k)
    # a bound that matters at this scale: a fraction of the typical k-th gap
    bound = np.full(n, 0.05)
    noise = rng.uniform(-1.0, 1.0, D.shape)
    ok_settled, ok_out = settle(D, D + bound[:, None] * noise, bound, k)
    assert ok_settled.mean() > 0.9
    assert np.array_equal(ok_out[ok_settled], T[ok_settled])
    # errors fifty times the bound the rule assumes: some settle wrongly
    bad_settled, bad_out = settle(D, D + 50 * bound[:, None] * noise, bound, k)
    wrong = (bad_out != T).any(1) & bad_settled
    assert wrong.sum() > 0
