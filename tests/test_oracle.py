"""CPU tests of the oracle (the checker) -- pinned against the reference's own
known-answer tests and against independent numpy/scipy computations."""
import numpy as np
import pytest

from conftest import make_problem


def test_grid_size_table(oracle):
    # CU/utils.cu:194-215: smallest table size >= ng + 2, minus 2; saturates at 510
    assert oracle.best_grid_size(14) == 14
    assert oracle.best_grid_size(50) == 50
    assert oracle.best_grid_size(51) == 52
    assert oracle.best_grid_size(299) == 306
    assert oracle.best_grid_size(600) == 510
    assert oracle.best_grid_size(0) == 6
    # h-driven rule max(ceil(maxy/h),14) (HYB/qq.cpp:165-166)
    assert oracle.grid_points_h(1e-3, 0.7) == 16
    assert oracle.grid_points_h(100.0, 0.7) == oracle.best_grid_size(143) + 2


@pytest.mark.parametrize("L", [8, 12, 13, 52, 77, 91, 117, 273, 455, 512, 1024])
def test_fft_matches_numpy(oracle, L):
    rng = np.random.default_rng(L)
    x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    ref = np.fft.fft(x)
    assert np.abs(oracle.fft(x) - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(oracle.fft(x, +1) - np.fft.ifft(x) * L).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("d,N", [(1, 30), (2, 16), (2, 25), (3, 10)])
def test_even_odd_conv_equals_direct(oracle, d, N):
    # the 2^d half-shift FFT terms (HYB/non_periodic_conv.cpp) sum to the
    # exact aperiodic convolution
    rng = np.random.default_rng(d * 100 + N)
    V = rng.standard_normal((d + 1,) + (N,) * d)
    a = oracle.g2g(V, 0.37, 0)
    b = oracle.g2g(V, 0.37, 1)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_direct_conv_matches_scipy(oracle):
    from scipy.signal import fftconvolve
    rng = np.random.default_rng(5)
    N, h = 18, 0.5
    V = rng.standard_normal((3, N, N))
    r = np.arange(-(N - 1), N)
    K = (1 + h * h * (r[:, None] ** 2 + r[None, :] ** 2)) ** -2.0
    ref = np.stack([fftconvolve(V[c], K, mode="full")[N - 1:2 * N - 1, N - 1:2 * N - 1]
                    for c in range(3)])
    assert np.abs(oracle.g2g(V, h, 1) - ref).max() <= 1e-10


@pytest.mark.parametrize("n", [1000, 2000, 3000])
@pytest.mark.parametrize("d", [1, 2, 3])
def test_repulsive_interp_vs_exact_reference_tolerance(oracle, n, d):
    # HYB/test_modules.cpp:122-156: y ~ U(0,1)^d, h in {0.05, 0.08, 0.13};
    # max |F_interp - F_exact| <= 1e-7 and |Z - Z_exact|/Z_exact <= 1e-4
    rng = np.random.default_rng(1000 * d + n)
    Y = rng.random((n, d))
    Fe, Ze = oracle.repulsive_exact(Y)
    for h in (0.05, 0.08, 0.13):
        F, Z, N, he = oracle.repulsive_interp(Y, h)
        assert np.abs(F - Fe).max() <= 1e-7
        assert abs(Z - Ze) / Ze <= 1e-4


def test_repulsive_exact_matches_numpy(oracle):
    rng = np.random.default_rng(3)
    Y = rng.standard_normal((300, 2))
    D = ((Y[:, None, :] - Y[None, :, :]) ** 2).sum(-1)
    Q = 1.0 / (1.0 + D)
    np.fill_diagonal(Q, 0.0)
    Z = Q.sum()
    F = ((Q ** 2)[:, :, None] * (Y[:, None, :] - Y[None, :, :])).sum(1) / Z
    F2, Z2 = oracle.repulsive_exact(Y)
    assert abs(Z2 - Z) / Z < 1e-13
    assert np.abs(F2 - F).max() < 1e-13 * np.abs(F).max() + 1e-18


def test_attractive_matches_dense(oracle):
    rp, col, val, _ = make_problem(n=500, k=10)
    rng = np.random.default_rng(2)
    Y = rng.standard_normal((500, 2))
    P = np.zeros((500, 500))
    for i in range(500):
        P[i, col[rp[i]:rp[i + 1]]] = val[rp[i]:rp[i + 1]]
    D = ((Y[:, None, :] - Y[None, :, :]) ** 2).sum(-1)
    W = P / (1 + D)
    F = (W[:, :, None] * (Y[:, None, :] - Y[None, :, :])).sum(1)
    assert np.abs(oracle.attractive(rp, col, val, Y) - F).max() < 1e-15


def test_csr_to_coo_and_hybrid(oracle):
    rp, col, val, _ = make_problem(n=800, k=12)
    rows = oracle.csr_to_coo(rp)
    assert np.array_equal(rows, np.repeat(np.arange(800), np.diff(rp)))
    # empty rows are skipped by the binary search
    rp2 = np.array([0, 2, 2, 2, 5, 6], np.int32)
    assert list(oracle.csr_to_coo(rp2)) == [0, 0, 3, 3, 3, 4]
    W = oracle.ell_width_cusp(rp)
    lens = np.diff(rp)
    assert (lens > W).sum() < max(800 / 3, 1) or (lens > W).sum() < 4096
    ec, ev, cr, cc, cv = oracle.csr_to_hybrid(rp, col, val.astype(np.float32), W)
    # ELL + COO is a partition of the CSR entries
    tot = np.zeros((800, 800))
    for r in range(800):
        for k in range(W):
            tot[r, ec[k * 800 + r]] += ev[k * 800 + r]
    np.add.at(tot, (cr, cc), cv)
    dense = np.zeros((800, 800))
    for i in range(800):
        dense[i, col[rp[i]:rp[i + 1]]] += val[rp[i]:rp[i + 1]].astype(np.float32)
    assert np.allclose(tot, dense, rtol=0, atol=1e-9)
    assert len(cr) == int(np.maximum(lens - W, 0).sum())


def test_symmetrize(oracle):
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_isotropic(600, 10, 4, 16.0, 1)
    idx, d2 = W.knn_numpy(X, 8)
    rp, col, val = W.knn_csr(idx, d2)
    srp, sc, sv = oracle.symmetrize(rp, col, val, 0.5)
    n = 600
    A = np.zeros((n, n))
    for i in range(n):
        A[i, col[rp[i]:rp[i + 1]]] += val[rp[i]:rp[i + 1]]
    S = np.zeros((n, n))
    for i in range(n):
        seg = sc[srp[i]:srp[i + 1]]
        assert np.all(np.diff(seg) > 0)  # sorted, no duplicates
        S[i, seg] = sv[srp[i]:srp[i + 1]]
    assert np.allclose(S, 0.5 * (A + A.T), atol=1e-14)
    assert int(srp[-1]) == int(((A + A.T) != 0).sum())


def test_lambda_rescale(oracle):
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_isotropic(400, 10, 4, 16.0, 2)
    idx, d2 = W.knn_numpy(X, 12)
    rp, col, val = W.knn_csr(idx, d2)
    for lam in (1.0, 10.0):
        v, sig = oracle.lambda_rescale(rp, val, lam, dist=True)
        # converged: sum_j exp(-sigma d_j) == lambda within the tolerance
        s = np.array([np.exp(-val[rp[i]:rp[i + 1]] * sig[i]).sum() for i in range(400)])
        assert np.abs(s - lam).max() <= 1e-5
        assert np.allclose(np.add.reduceat(v, rp[:-1]), 1.0)


def test_perplexity(oracle):
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_isotropic(300, 10, 3, 16.0, 3)
    idx, d2 = W.knn_numpy(X, 30)
    D = np.concatenate([np.zeros((300, 1)), d2], 1)
    P = oracle.perplexity(D, 10.0)
    assert np.allclose(P.sum(1), 1.0)
    H = -(P * np.log(np.maximum(P, 1e-300))).sum(1)
    assert np.abs(H - np.log(10.0)).max() < 1e-4


def test_bins_f32_emulation(oracle):
    # FP32 CUDA binning restated op by op; compare with numpy float32 math
    rng = np.random.default_rng(4)
    Y = (rng.standard_normal((5000, 2)) * 7).astype(np.float32)
    bins, sc, sh, N, mx = oracle.bins_f32(Y, 0.7)
    mn = np.minimum(np.float32(100.0), Y.min(0))
    s = (Y - mn).astype(np.float32)
    assert np.array_equal(s, sh)
    maxy = np.float32(s.max())
    assert maxy == np.float32(mx)
    ng = max(int(np.ceil(np.float32(maxy / np.float32(0.7)))), 14)
    assert N == oracle.best_grid_size(ng) + 2
    v = (s / maxy).astype(np.float32)
    v[v >= 1] = np.float32(1 - np.finfo(np.float32).eps)
    t = (v * np.float32(N - 3)).astype(np.float32)
    assert np.array_equal(np.floor(t).astype(np.uint32), bins)
    assert bins.max() <= N - 4


def test_kl_and_descent(oracle):
    rp, col, val, lab = make_problem(n=600, k=10)
    rng = np.random.default_rng(7)
    Y0 = rng.standard_normal((600, 2)) * 1e-2
    Y, z = oracle.kl_minimization(rp, col, val, Y0, 300, return_zeta=True)
    F, Z, _, _ = oracle.repulsive_interp(Y, 0.7)
    kl_end = oracle.kl(rp, col, val, Y, 1.0, Z)
    F0, Z0, _, _ = oracle.repulsive_interp(Y0, 0.7)
    kl_start = oracle.kl(rp, col, val, Y0, 1.0, Z0)
    assert kl_end < 0.5 * kl_start
    assert np.abs(Y.mean(0)).max() < 1e-9  # mean-centred every iteration
