"""Error of the engine's arithmetic (FP32 SpMV, scatter/gather and FFT with
FP32 accumulation; FP64 only for Z, KL and the bisection row sums) against
the FP64 oracle, on the 60,000-point digits-like configuration (784-D, 10
clusters of 150 active coordinates, uint8 quantised, k = 90, perplexity 30),
for d = 2 and d = 3.

Each force is compared at one state Y (the engine's embedding after 300
iterations from Y0): F_attr, F_rep and Z against the oracle at the same
grid, F_rep also against the exact O(n^2) sum (the interpolation error
itself), and the full gradient F_attr - F_rep (alpha = 1 after the early
exaggeration; both forces as the update uses them, F_rep divided by Z).  KL is compared after
500 iterations of both from the same Y0.  The measured values are printed
(pytest -s / -rP) and each is held to its bar:

  F_attr           rel-L2 <= 1e-5      F_rep (same grid)   rel-L2 <= 3e-4
  Z                rel    <= 5e-4      gradient            rel-L2 <= 1e-3
  KL after 500     within 1 %
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 60000


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def digits_p(oracle):
    import torch

    from sgtsne_b200 import workloads as W
    X = W.digits_like(n=N, dim=784, ncomp=10, active=150, keep=0.9, noise=20.0, seed=0)[0]
    idx, d2 = W.knn_torch(X, 90, device="cuda", block=2048)
    torch.cuda.synchronize()
    idx = idx.cpu().numpy()
    d2 = d2.cpu().numpy().astype(np.float64)
    D = np.concatenate([np.zeros((N, 1)), d2 / d2.max()], 1)
    Pk = oracle.perplexity(D, 30.0)
    rp = (np.arange(N + 1, dtype=np.int64) * 90).astype(np.int32)
    srp, sc, sv = oracle.symmetrize(rp, idx.reshape(-1).astype(np.int32), Pk.reshape(-1),
                                    1.0 / (2 * N))
    return srp, sc, sv


@pytest.mark.parametrize("d", [2, 3])
def test_errors_against_fp64(digits_p, oracle, d):
    import torch

    import sgtsne_b200 as S
    srp, sc, sv = digits_p
    v32 = sv.astype(np.float32)
    h = 0.7 if d == 2 else 1.2
    ctx = S.Context(0)
    p = S.default_params(d=d, format=S.FORMAT_CSR, max_iter=1000, early_iter=250, h=h)
    y0 = (np.random.default_rng(5).standard_normal((N, d)) * 1e-2).astype(np.float32)
    job = S.Job(ctx, p, srp, sc, v32, device_mem=False)
    job.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
    job.run(300)
    Y = np.empty((N, d), np.float32)
    job.get_y(Y, S.LAYOUT_POINT_MAJOR, False, 1)
    job.close()
    Yd = torch.from_numpy(Y).cuda()
    nnz = int(srp[-1])
    # attractive
    fa = torch.empty(N * d, dtype=torch.float32, device="cuda")
    ctx.attractive(S.FORMAT_CSR, N, d, nnz, torch.from_numpy(srp).cuda(), None,
                   torch.from_numpy(sc).cuda(), torch.from_numpy(v32).cuda(), Yd,
                   S.LAYOUT_POINT_MAJOR, fa)
    Fa = fa.cpu().numpy().reshape(N, d)
    Fa_o = oracle.attractive(srp, sc, sv, Y.astype(np.float64))
    e_attr = rel(Fa, Fa_o)
    # repulsive, same grid, and exact
    fr = torch.empty(N * d, dtype=torch.float32, device="cuda")
    Z, grid, he = ctx.repulsive(N, d, h, 0, Yd, S.LAYOUT_POINT_MAJOR, fr)
    Fr = fr.cpu().numpy().reshape(N, d)
    Fr_o, Z_o, grid_o, _ = oracle.repulsive_interp(Y.astype(np.float64), h, n1_force=grid - 2)
    Fr_x, Z_x = oracle.repulsive_exact(Y.astype(np.float64))
    e_rep, e_z = rel(Fr, Fr_o), abs(Z - Z_o) / abs(Z_o)
    e_rep_exact = rel(Fr, Fr_x)
    e_interp = rel(Fr_o, Fr_x)
    # full gradient as the update uses it (alpha = 1 after early exaggeration)
    g = Fa - Fr
    g_o = Fa_o - Fr_o
    e_grad = rel(g, g_o)
    # KL after 500 iterations of both from the same Y0
    job = S.Job(ctx, p, srp, sc, v32, device_mem=False)
    job.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
    job.run(500)
    Ye = np.empty((N, d), np.float32)
    job.get_y(Ye, S.LAYOUT_POINT_MAJOR, False, 1)
    job.close()
    ctx.close()
    Yo = oracle.kl_minimization(srp, sc, sv, y0.astype(np.float64), 500, early_iter=250,
                                alpha=12.0, h=h, grid_mode=0)
    _, Ze, _, _ = oracle.repulsive_interp(Ye.astype(np.float64), h)
    _, Zo, _, _ = oracle.repulsive_interp(Yo, h)
    kl_e = oracle.kl(srp, sc, sv, Ye.astype(np.float64), 1.0, Ze)
    kl_o = oracle.kl(srp, sc, sv, Yo, 1.0, Zo)
    e_kl = abs(kl_e - kl_o) / kl_o
    print(f"\nprecision d={d} n={N} nnz={nnz} grid={grid}: F_attr {e_attr:.2e} | "
          f"F_rep(same grid) {e_rep:.2e} | Z {e_z:.2e} | gradient {e_grad:.2e} | "
          f"F_rep vs exact {e_rep_exact:.2e} (oracle's own interpolation {e_interp:.2e}) | "
          f"KL@500 {kl_e:.5f} vs {kl_o:.5f} ({e_kl:.2e})")
    assert grid == grid_o
    assert e_attr <= 1e-5
    assert e_rep <= 3e-4
    assert e_z <= 5e-4
    assert e_grad <= 1e-3
    assert e_kl <= 0.01
