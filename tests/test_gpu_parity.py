"""GPU parity tests: the CUDA engine, called through the C ABI, against the
oracle on the same seeded inputs.

Tolerances (FP32 engine vs FP64 oracle):
  integer work (bins, grid sizes, CSR->COO, formats)      bit-exact
  attractive forces                                       rel L2 <= 1e-5
  S2G grid / G2G grid at a fixed Y                        rel L2 <= 1e-4
  repulsive forces at a fixed Y                           rel L2 <= 3e-4 (FP32
      scatter/FFT/gather against FP64; the FP32 atomics make the value vary
      by ~2e-5 from run to run; 5e-4 for 1-D at the fixed 40-interval grid)
  Z at a fixed Y                                          rel <= 5e-4 (the
      reference's Z = sum (1+2|y|^2)Phi0 - 2 y.Phi - n cancels; its FP32
      potentials carry ~1e-7 relative error amplified by |y|^2)
  KL                                                      rel <= 1e-5
  lambda / perplexity values                              rel <= 1e-4
  iterations (same P, Y0): KL after the run               within 1 %
"""
import os

import numpy as np
import pytest

from conftest import make_problem

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def ctx():
    import sgtsne_b200 as S
    c = S.Context(0)
    yield c
    c.close()


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def coords(kind, n, d, seed):
    rng = np.random.default_rng(seed)
    if kind == "gauss":
        Y = rng.standard_normal((n, d)) * 5
    elif kind == "uniform":
        Y = rng.random((n, d))
    elif kind == "clusters":
        c = rng.standard_normal((8, d)) * 20
        Y = c[rng.integers(0, 8, n)] + rng.standard_normal((n, d))
    elif kind == "tiny":
        Y = rng.standard_normal((n, d)) * 1e-4
    elif kind == "offset":  # every coordinate above 100: the 100.0 min-init quirk
        Y = 150 + rng.random((n, d)) * 30
    else:
        raise ValueError(kind)
    return Y.astype(np.float32)


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("kind", ["gauss", "uniform", "clusters", "tiny", "offset"])
@pytest.mark.parametrize("ng", [0, 50])
def test_bins_and_grid_bit_exact(torch, ctx, oracle, d, kind, ng):
    import sgtsne_b200 as S
    n = 20000
    Y = coords(kind, n, d, seed=d * 7 + len(kind))
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    out = torch.empty(n * d, dtype=torch.int32, device="cuda")
    N = ctx.bins(n, d, h, ng, dev(torch, Y), S.LAYOUT_POINT_MAJOR, out)
    b_ref, _, _, N_ref, _ = oracle.bins_f32(Y, h, oracle.best_grid_size(ng) if ng else 0)
    assert N == N_ref
    assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(n, d), b_ref)


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("kind", ["gauss", "clusters", "uniform"])
def test_repulsive_vs_oracle(torch, ctx, oracle, d, kind):
    import sgtsne_b200 as S
    n = 8000 if d < 3 else 4000
    Y = coords(kind, n, d, seed=11 + d)
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    Z, N, he = ctx.repulsive(n, d, h, 0, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    F = f.cpu().numpy().reshape(n, d)
    Fo, Zo, No, heo = oracle.repulsive_interp(Y.astype(np.float64), h, n1_force=N - 2)
    assert N == No
    assert abs(he - heo) <= 1e-6 * heo
    assert abs(Z - Zo) <= 5e-4 * abs(Zo)
    assert rel(F, Fo) <= 3e-4


@pytest.mark.parametrize("d", [1, 2, 3])
def test_grids_vs_oracle(torch, ctx, oracle, d):
    """S2G and G2G stage by stage: the engine's charge grid against the
    oracle's S2G of the same FP32-scaled coordinates, and its potential grid
    against the oracle's G2G of the engine's own charge grid."""
    import sgtsne_b200 as S
    n = 6000
    Y = coords("clusters", n, d, seed=3 + d)
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    Z, N, he = ctx.repulsive(n, d, h, 0, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    V, Phi = ctx.last_grids(d, N)
    _, sc, sh, N2, mx = oracle.bins_f32(Y, h)
    assert N2 == N
    # the engine takes the charges about the grid middle (y - maxy/2)
    hc = np.float32(0.5) * np.float32(mx)
    q = np.concatenate([np.ones((n, 1)), (sh - hc).astype(np.float64)], 1)
    Vo = oracle.s2g(sc.astype(np.float64), q, N)
    assert rel(V, Vo) <= 1e-5
    Phio = oracle.g2g(V.astype(np.float64), float(he), 0)
    assert rel(Phi, Phio) <= 1e-4


def cell_mode(n, d, N):
    """The engine's binning rule: one tile per cell when the (N-3)^d cells fit
    4096 tiles and hold at least 64 points each on average."""
    cells = (N - 3) ** d
    return cells <= 4096 and n >= 64 * cells


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("kind", ["compact", "clusters"])
def test_cell_mode_vs_oracle(torch, ctx, oracle, d, kind):
    """Many points on a small grid (the regime of a real run at 1.3M points):
    the binning keys are cells and S2G sums each cell's points in registers.
    Charge grid, forces and Z against the oracle at the tolerances above."""
    import sgtsne_b200 as S
    n = {1: 20000, 2: 40000, 3: 200000}[d]
    rng = np.random.default_rng(40 + d)
    if kind == "compact":
        Y = (rng.standard_normal((n, d)) * 1.5).astype(np.float32)
    else:
        c = rng.standard_normal((6, d)) * 3
        Y = (c[rng.integers(0, 6, n)] + rng.standard_normal((n, d)) * 0.3).astype(np.float32)
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    Z, N, he = ctx.repulsive(n, d, h, 0, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    assert cell_mode(n, d, N), (n, d, N)
    V, Phi = ctx.last_grids(d, N)
    _, sc, sh, N2, mx = oracle.bins_f32(Y, h)
    assert N2 == N
    hc = np.float32(0.5) * np.float32(mx)
    q = np.concatenate([np.ones((n, 1)), (sh - hc).astype(np.float64)], 1)
    Vo = oracle.s2g(sc.astype(np.float64), q, N)
    assert rel(V, Vo) <= 1e-5
    F = f.cpu().numpy().reshape(n, d)
    Fo, Zo, No, heo = oracle.repulsive_interp(Y.astype(np.float64), h, n1_force=N - 2)
    assert N == No
    assert abs(Z - Zo) <= 5e-4 * abs(Zo)
    assert rel(F, Fo) <= 3e-4


@pytest.mark.parametrize("kind", ["clusters", "compact", "ordered"])
@pytest.mark.parametrize("ng", [58, 66])
def test_direct_and_sorted_modes_2d(torch, ctx, oracle, kind, ng):
    """2-D grids too sparse for cell mode, on either side of the direct-mode
    limit (64 points per axis): fixed grid 58 -> N = 60 takes the direct mode
    (S2G in shared memory over the points in their own order), 66 -> N = 70
    the tile sort.  Points in
    clusters, compact, and sorted along a space-filling order (the warp
    reduction of the direct S2G); charge grid, forces and Z against the
    oracle."""
    import sgtsne_b200 as S
    n, d, h = 40000, 2, 0.7
    rng = np.random.default_rng(77 + ng)
    if kind == "compact":
        Y = (rng.standard_normal((n, d)) * 1.5).astype(np.float32)
    else:
        c = rng.standard_normal((6, d)) * 3
        Y = (c[rng.integers(0, 6, n)] + rng.standard_normal((n, d)) * 0.3).astype(np.float32)
    if kind == "ordered":  # runs of points in one cell, as after a relabelling
        q = np.floor((Y - Y.min(0)) / 0.25).astype(np.int64)
        Y = Y[np.lexsort((q[:, 0], q[:, 1]))]
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    Z, N, he = ctx.repulsive(n, d, h, ng, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    assert N == oracle.best_grid_size(ng) + 2
    V, Phi = ctx.last_grids(d, N)
    _, sc, sh, N2, mx = oracle.bins_f32(Y, h, oracle.best_grid_size(ng))
    assert N2 == N
    hc = np.float32(0.5) * np.float32(mx)
    q = np.concatenate([np.ones((n, 1)), (sh - hc).astype(np.float64)], 1)
    Vo = oracle.s2g(sc.astype(np.float64), q, N)
    assert rel(V, Vo) <= 1e-5
    F = f.cpu().numpy().reshape(n, d)
    Fo, Zo, No, heo = oracle.repulsive_interp(Y.astype(np.float64), h, n1_force=N - 2)
    assert No == N
    assert abs(Z - Zo) <= 5e-4 * abs(Zo)
    assert rel(F, Fo) <= 3e-4


@pytest.mark.parametrize("ng", [20, 40])
def test_dense_job_modes_2d(torch, ctx, oracle, ng):
    """A 2-D job with enough points (2.6M) that its grids up to 64 points per
    axis are all dense never takes the direct mode: fixed grids 20 -> N = 25
    and 40 -> N = 42 run in cell mode, with many chunks per cell.  Charge
    grid, forces and Z against the oracle."""
    import sgtsne_b200 as S
    n, d, h = 2600000, 2, 0.7
    rng = np.random.default_rng(90 + ng)
    c = rng.standard_normal((6, d)) * 3
    Y = (c[rng.integers(0, 6, n)] + rng.standard_normal((n, d)) * 0.5).astype(np.float32)
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    Z, N, he = ctx.repulsive(n, d, h, ng, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    assert N == oracle.best_grid_size(ng) + 2
    V, Phi = ctx.last_grids(d, N)
    _, sc, sh, N2, mx = oracle.bins_f32(Y, h, oracle.best_grid_size(ng))
    assert N2 == N
    hc = np.float32(0.5) * np.float32(mx)
    q = np.concatenate([np.ones((n, 1)), (sh - hc).astype(np.float64)], 1)
    Vo = oracle.s2g(sc.astype(np.float64), q, N)
    assert rel(V, Vo) <= 1e-5
    F = f.cpu().numpy().reshape(n, d)
    Fo, Zo, No, heo = oracle.repulsive_interp(Y.astype(np.float64), h, n1_force=N - 2)
    assert No == N
    assert abs(Z - Zo) <= 5e-4 * abs(Zo)
    assert rel(F, Fo) <= 3e-4


@pytest.mark.parametrize("fmt", [0, 2, 3])
@pytest.mark.parametrize("d", [1, 2, 3])
def test_attractive_formats(torch, ctx, oracle, fmt, d):
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=3000, k=12, seed=d)
    n = len(rp) - 1
    rng = np.random.default_rng(5)
    Y = (rng.standard_normal((n, d)) * 3).astype(np.float32)
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    rows = dev(torch, np.repeat(np.arange(n), np.diff(rp)).astype(np.int32))
    ctx.attractive(fmt, n, d, int(rp[-1]), dev(torch, rp), rows, dev(torch, col),
                   dev(torch, val.astype(np.float32)), dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    Fo = oracle.attractive(rp, col, val.astype(np.float32).astype(np.float64), Y.astype(np.float64))
    assert rel(f.cpu().numpy().reshape(n, d), Fo) <= 1e-5


def test_dim_major_layout(torch, ctx, oracle):
    import sgtsne_b200 as S
    n, d = 5000, 2
    Y = coords("gauss", n, d, 9)
    f1 = torch.empty(n * d, dtype=torch.float32, device="cuda")
    f2 = torch.empty(n * d, dtype=torch.float32, device="cuda")
    z1, _, _ = ctx.repulsive(n, d, 0.7, 0, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f1)
    z2, _, _ = ctx.repulsive(n, d, 0.7, 0, dev(torch, Y.T.copy()), S.LAYOUT_DIM_MAJOR, f2)
    # identical inputs; the difference is the order of FP32 atomics in S2G
    assert rel(f2.cpu().numpy().reshape(d, n).T, f1.cpu().numpy().reshape(n, d)) <= 2e-5
    assert abs(z1 - z2) <= 2e-5 * abs(z1)


def test_csr_to_coo_bit_exact(torch, ctx, oracle):
    rp, col, val, _ = make_problem(n=2500, k=9)
    rp2 = rp.copy()
    n = len(rp2) - 1
    rows = torch.empty(int(rp2[-1]), dtype=torch.int32, device="cuda")
    ctx.csr_to_coo(n, int(rp2[-1]), dev(torch, rp2), rows)
    assert np.array_equal(rows.cpu().numpy(), oracle.csr_to_coo(rp2))


def test_kl(torch, ctx, oracle):
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=2000, k=10)
    n = len(rp) - 1
    Y = coords("gauss", n, 2, 2)
    v32 = val.astype(np.float32)
    kl = ctx.kl(n, 2, int(rp[-1]), dev(torch, rp), dev(torch, col), dev(torch, v32),
                dev(torch, Y), S.LAYOUT_POINT_MAJOR, 12.0, 1234.5)
    ko = oracle.kl(rp, col, v32.astype(np.float64), Y.astype(np.float64), 12.0, 1234.5)
    assert abs(kl - ko) <= 1e-5 * abs(ko)


@pytest.mark.parametrize("lam", [1.0, 10.0])
def test_lambda_bisect(torch, ctx, oracle, lam):
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_isotropic(3000, 20, 5, 16.0, 6)
    idx, d2 = W.knn_numpy(X, 20)
    rp, col, val = W.knn_csr(idx, d2)
    v = dev(torch, val.astype(np.float32))
    sig = torch.empty(3000, dtype=torch.float32, device="cuda")
    ctx.lambda_bisect(3000, dev(torch, rp), v, lam, 1, sig)
    vo, so = oracle.lambda_rescale(rp, val.astype(np.float32).astype(np.float64), lam, dist=True)
    assert rel(v.cpu().numpy(), vo) <= 1e-4
    assert rel(sig.cpu().numpy(), so) <= 1e-4


def test_perplexity(torch, ctx, oracle):
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_isotropic(3000, 20, 5, 16.0, 8)
    idx, d2 = W.knn_numpy(X, 90)
    d2 = d2 / d2.max()
    p = torch.empty(3000 * 90, dtype=torch.float32, device="cuda")
    ctx.perplexity(3000, 90, dev(torch, d2.astype(np.float32)), 30.0, p)
    D = np.concatenate([np.zeros((3000, 1)), d2.astype(np.float32).astype(np.float64)], 1)
    Po = oracle.perplexity(D, 30.0)
    assert rel(p.cpu().numpy().reshape(3000, 90), Po) <= 1e-4


@pytest.mark.parametrize("d", [1, 2, 3])
def test_iterations_vs_oracle(torch, ctx, oracle, d):
    """The graph-captured iteration loop against the oracle's gradient
    descent (h-driven grid, per-iteration centring) on the same P and Y0."""
    import sgtsne_b200 as S
    rp, col, val, lab = make_problem(n=2000, k=12, seed=20 + d)
    n = len(rp) - 1
    rng = np.random.default_rng(1)
    Y0 = (rng.standard_normal((n, d)) * 1e-2).astype(np.float32)
    v32 = val.astype(np.float32)
    p = S.default_params(d=d, format=S.FORMAT_CSR, max_iter=400, early_iter=100)
    job = S.Job(ctx, p, rp, col, v32, device_mem=False)
    job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
    job.run(400)
    Y = job.get_y(np.empty((n, d), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
    info = job.info()
    assert info.iter == 400 and info.error_flags == 0
    Yo = oracle.kl_minimization(rp, col, v32.astype(np.float64), Y0.astype(np.float64), 400,
                                early_iter=100, alpha=12.0, h=p.h if p.h > 0 else
                                {1: 0.5, 2: 0.7, 3: 1.2}[d], grid_mode=0)
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    _, Zg, _, _ = oracle.repulsive_interp(Y.astype(np.float64), h)
    _, Zo, _, _ = oracle.repulsive_interp(Yo, h)
    klg = oracle.kl(rp, col, v32.astype(np.float64), Y.astype(np.float64), 1.0, Zg)
    klo = oracle.kl(rp, col, v32.astype(np.float64), Yo, 1.0, Zo)
    assert abs(klg - klo) <= 0.01 * klo
    job.close()


def test_formats_same_trajectory(torch, ctx):
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=3000, k=12, seed=4)
    n = len(rp) - 1
    Y0 = (np.random.default_rng(2).standard_normal((n, 2)) * 1e-2).astype(np.float32)
    out = {}
    for fmt in (0, 2, 3):
        p = S.default_params(d=2, format=fmt)
        job = S.Job(ctx, p, rp, col, val.astype(np.float32), device_mem=False)
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(30)
        out[fmt] = job.get_y(np.empty((n, 2), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
        job.close()
    assert rel(out[2], out[0]) <= 1e-3
    assert rel(out[3], out[0]) <= 1e-3


def test_embed_dropin(torch, ctx, oracle):
    """sgt_embed (the sgtsneCUDA flow: lambda rescaling, symmetrisation,
    iterations, centring) against the oracle pipeline."""
    import sgtsne_b200 as S
    from sgtsne_b200 import workloads as W
    n, k = 2500, 15
    X, _ = W.gmm_isotropic(n, 20, 6, 16.0, 12)
    idx, d2 = W.knn_numpy(X, k)
    rp, col, val = W.knn_csr(idx, d2)
    val = (val / val.max()).astype(np.float32)
    Y0 = (np.random.default_rng(3).standard_normal((n, 2)) * 1e-2).astype(np.float32)
    p = S.default_params(d=2, lambda_=1.0, max_iter=300, early_iter=100, format=S.FORMAT_CSR)
    p.lambda_ = 10.0
    Y, ti = ctx.embed(rp, col, val, p, y_in=Y0.T.copy(), time_info=np.zeros(7003))
    assert np.abs(Y.mean(0)).max() < 1e-3
    # per-iteration stage times in the reference's timeInfo layout: every
    # slot of the 300 iterations filled, nothing beyond them
    st = ti[:7000].reshape(1000, 7)
    assert (st[:300] > 0).all() and (st[300:] == 0).all()
    # slot 5 (S2G..G2S) spans slots 1-3
    assert (st[:300, 5] >= 0.99 * st[:300, 1:4].sum(1)).all()
    vo, _ = oracle.lambda_rescale(rp, val.astype(np.float64), 10.0, dist=True)
    srp, sc, sv = oracle.symmetrize(rp, col, vo, 1.0 / (2 * n))
    Yo = oracle.kl_minimization(srp, sc, sv, Y0.astype(np.float64), 300, early_iter=100,
                                alpha=12.0, h=0.7, grid_mode=0)
    _, Zg, _, _ = oracle.repulsive_interp(Y.astype(np.float64), 0.7)
    _, Zo, _, _ = oracle.repulsive_interp(Yo, 0.7)
    klg = oracle.kl(srp, sc, sv, Y.astype(np.float64), 1.0, Zg)
    klo = oracle.kl(srp, sc, sv, Yo, 1.0, Zo)
    assert abs(klg - klo) <= 0.01 * klo
    assert ti[7000] > 0


def test_invalid_csr_rejected(torch, ctx):
    import sgtsne_b200 as S
    rp = np.array([0, 2, 1, 3], np.int32)  # not monotone
    col = np.array([1, 2, 0], np.int32)
    p = S.default_params(d=2, format=S.FORMAT_CSR)
    with pytest.raises(S.SgtError) as e:
        S.Job(ctx, p, rp, col, np.ones(3, np.float32), device_mem=False)
    assert e.value.status == 1
    # sgt_embed: a column out of range is caught on the device, before the
    # iterations; a non-monotone rowptr on the host
    rp2 = np.array([0, 2, 3, 4], np.int32)
    p.lambda_ = 3.0
    for r, c in ((rp2, np.array([1, 2, 5, 0], np.int32)), (rp, col)):
        with pytest.raises(S.SgtError) as e:
            ctx.embed(r, c, np.ones(len(c), np.float32), p)
        assert e.value.status == 1


def test_relayout_is_transparent(torch, ctx):
    """Locality relabelling every 10 iterations against none: the caller sees
    the same embedding in the same point order (per-row sums are
    bit-identical; only the order of the FP32 scatter atomics differs)."""
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=4000, k=12, seed=9)
    n = len(rp) - 1
    Y0 = (np.random.default_rng(4).standard_normal((n, 2)) * 5).astype(np.float32)
    out = {}
    for every in (0, 10):
        p = S.default_params(d=2, format=S.FORMAT_CSR)
        p.relayout_every = every
        job = S.Job(ctx, p, rp, col, val.astype(np.float32), device_mem=False)
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(35)
        out[every] = job.get_y(np.empty((n, 2), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
        # a second run from the same start after relabelling still maps back
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(35)
        again = job.get_y(np.empty((n, 2), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
        assert rel(again, out[every]) <= 1e-4
        job.close()
    assert rel(out[10], out[0]) <= 1e-4


@pytest.mark.parametrize("d", [2, 3])
def test_locality_order_is_transparent(torch, ctx, oracle, d):
    """A job of at least 65,536 points starts from the diffusion locality
    order of its P (locality_order = 1, the default); the caller sees the
    embedding of locality_order = 0 in its own point order (rel-L2 <= 1e-5
    after 2 iterations: only the order of FP32 atomics differs)."""
    import sgtsne_b200 as S
    n, k = 70000, 10
    rng = np.random.default_rng(21)
    col = rng.integers(0, n - 1, (n, k))
    col += col >= np.arange(n)[:, None]  # no self loops
    rp = (np.arange(n + 1) * k).astype(np.int32)
    v = rng.random(n * k) + 0.1
    srp, sc, sv = oracle.symmetrize(rp, col.reshape(-1).astype(np.int32), v, 1.0 / (2 * n))
    Y0 = (rng.standard_normal((n, d)) * 1e-2).astype(np.float32)
    out = {}
    for order in (0, 1):
        p = S.default_params(d=d, format=S.FORMAT_CSR)
        p.locality_order = order
        job = S.Job(ctx, p, srp, sc, sv.astype(np.float32), device_mem=False)
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(2)
        out[order] = job.get_y(np.empty((n, d), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
        job.close()
    assert rel(out[1], out[0]) <= 1e-5


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("n", [3000, 150000])
def test_csr_spmv_kernels_agree_with_coo(torch, ctx, oracle, d, n):
    """The CSR row kernel (with the lane count the autotuner picks, and the
    locality order for the large case) against the COO path: two
    iterations agree (rel-L2 <= 1e-5)."""
    import sgtsne_b200 as S
    k = 10
    rng = np.random.default_rng(n + d)
    col = rng.integers(0, n - 1, (n, k))
    col += col >= np.arange(n)[:, None]
    rp = (np.arange(n + 1) * k).astype(np.int32)
    srp, sc, sv = oracle.symmetrize(rp, col.reshape(-1).astype(np.int32), rng.random(n * k) + 0.1,
                                    1.0 / (2 * n))
    Y0 = (rng.standard_normal((n, d)) * 1e-2).astype(np.float32)
    out = {}
    for fmt in (S.FORMAT_CSR, S.FORMAT_COO):
        job = S.Job(ctx, S.default_params(d=d, format=fmt), srp, sc, sv.astype(np.float32),
                    device_mem=False)
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(2)
        out[fmt] = job.get_y(np.empty((n, d), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
        job.close()
    assert rel(out[S.FORMAT_CSR], out[S.FORMAT_COO]) <= 1e-5


@pytest.mark.parametrize("d", [1, 2, 3])
def test_repulsive_error_probe(torch, ctx, oracle, d):
    """sgt_job_repulsive_error (the -f probe of CU/compute_error.cu:80-99):
    after one iteration from Y0 the job's repulsive force was computed at the
    centred Y0, so the probe must equal rel-L2(F_interp(Y0), F_exact(Y0)),
    F_exact from the oracle's FP64 direct sum, within 2 % of its value."""
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=3000, k=12, seed=30 + d)
    n = len(rp) - 1
    Y0 = coords("clusters", n, d, seed=31 + d) * np.float32(0.2)
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    p = S.default_params(d=d, format=S.FORMAT_CSR, h=h)
    job = S.Job(ctx, p, rp, col, val.astype(np.float32), device_mem=False)
    job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
    job.run(1)
    e_job = job.repulsive_error()
    job.close()
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    ctx.repulsive(n, d, h, 0, dev(torch, Y0), S.LAYOUT_POINT_MAJOR, f)
    Fx, _ = oracle.repulsive_exact(Y0.astype(np.float64))
    e_ref = rel(f.cpu().numpy().reshape(n, d), Fx)
    assert 0 < e_job < 0.5  # the interpolation error itself is ~1e-2..1e-1 here
    assert abs(e_job - e_ref) <= 0.02 * e_ref


def test_embed_compute_error_writes_error_info(torch, ctx, tmp_path, monkeypatch):
    """sgt_embed with compute_error = 1 appends one line of max_iter/10
    errors to errorInfo.txt, as the reference's -f option does."""
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=1500, k=10, seed=44)
    monkeypatch.chdir(tmp_path)
    p = S.default_params(d=2, max_iter=35, early_iter=20, format=S.FORMAT_CSR)
    p.compute_error = 1
    ctx.embed(rp, col, val.astype(np.float32), p)
    ctx.embed(rp, col, val.astype(np.float32), p)
    lines = (tmp_path / "errorInfo.txt").read_text().splitlines()
    assert len(lines) == 2
    errs = [float(x) for x in lines[0].split()]
    assert len(errs) == 4  # iterations 0, 10, 20, 30
    assert all(0 < e < 0.5 for e in errs)


@pytest.mark.parametrize("case", ["knn", "ragged"])
def test_symmetrize_device_bit_exact(torch, ctx, case):
    """sgt_symmetrize_device against the host sgt_symmetrize: same rowptr,
    columns and value bits.  'knn': rows of 15 neighbours in distance order
    (unsorted columns); 'ragged': empty rows, single-entry rows and repeated
    columns inside a row."""
    import sgtsne_b200 as S
    rng = np.random.default_rng(71)
    if case == "knn":
        from sgtsne_b200 import workloads as W
        X, _ = W.gmm_isotropic(5000, 20, 6, 16.0, 9)
        idx, d2 = W.knn_numpy(X, 15)
        rp, col, val = W.knn_csr(idx, d2)
        val = (val / val.max()).astype(np.float32)
    else:
        n = 3000
        lens = rng.integers(0, 9, n)
        lens[rng.integers(0, n, 300)] = 0
        lens[rng.integers(0, n, 300)] = 1
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        col = rng.integers(0, n, int(rp[-1])).astype(np.int32)
        dup = rng.integers(0, int(rp[-1]) - 1, 400)
        col[dup + 1] = col[dup]  # repeats (some cross a row end: harmless)
        val = rng.random(int(rp[-1])).astype(np.float32)
    n = len(rp) - 1
    nnz = int(rp[-1])
    hrp, hc, hv = S.symmetrize(rp, col, val, 1.0 / (2 * n))
    orp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    oc = torch.empty(2 * nnz, dtype=torch.int32, device="cuda")
    ov = torch.empty(2 * nnz, dtype=torch.float32, device="cuda")
    m = ctx.symmetrize(n, nnz, dev(torch, rp), dev(torch, col), dev(torch, val), 1.0 / (2 * n),
                       orp, oc, ov)
    assert m == len(hc)
    assert np.array_equal(orp.cpu().numpy(), hrp)
    assert np.array_equal(oc[:m].cpu().numpy(), hc)
    assert np.array_equal(ov[:m].cpu().numpy().view(np.uint32), hv.view(np.uint32))


def test_symmetrize_device_rejects_bad_column(torch, ctx):
    import sgtsne_b200 as S
    rp = np.array([0, 2, 3], np.int32)
    col = np.array([1, 5, 0], np.int32)  # 5 >= n
    val = np.ones(3, np.float32)
    orp = torch.empty(3, dtype=torch.int32, device="cuda")
    oc = torch.empty(6, dtype=torch.int32, device="cuda")
    ov = torch.empty(6, dtype=torch.float32, device="cuda")
    with pytest.raises(S.SgtError) as e:
        ctx.symmetrize(2, 3, dev(torch, rp), dev(torch, col), dev(torch, val), 0.25, orp, oc, ov)
    assert e.value.status == 1


@pytest.mark.parametrize("case", ["knn", "ragged"])
def test_csr_to_hybrid_device_bit_exact(torch, ctx, case):
    """sgt_csr_to_hybrid_device against the host sgt_csr_to_hybrid at the
    reference's width rule and at widths 0 and 1: the same ELL slots, padding
    and COO tail, bit for bit.  Then a hybrid job made from device arrays
    (split on the device) against one made from host arrays: the same Y
    after two iterations."""
    import sgtsne_b200 as S
    rng = np.random.default_rng(73)
    if case == "knn":
        rp, col, val, _ = make_problem(n=6000, dim=20, ncomp=5, k=12, seed=8)
        val = val.astype(np.float32)
    else:
        n = 4000
        lens = rng.integers(0, 40, n)
        lens[rng.integers(0, n, 400)] = 0
        lens[rng.integers(0, n, 20)] = 300
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        col = rng.integers(0, n, int(rp[-1])).astype(np.int32)
        val = rng.random(int(rp[-1])).astype(np.float32)
    n = len(rp) - 1
    nnz = int(rp[-1])
    for width in (S.ell_width(rp), 0, 1):
        ec, ev, cr, cc, cv = S.csr_to_hybrid(rp, col, val, width)
        dec = torch.zeros(max(n * width, 1), dtype=torch.int32, device="cuda")
        dev_ = torch.zeros(max(n * width, 1), dtype=torch.float32, device="cuda")
        dcr = torch.zeros(max(nnz, 1), dtype=torch.int32, device="cuda")
        dcc = torch.zeros(max(nnz, 1), dtype=torch.int32, device="cuda")
        dcv = torch.zeros(max(nnz, 1), dtype=torch.float32, device="cuda")
        m = ctx.csr_to_hybrid(n, dev(torch, rp), dev(torch, col), dev(torch, val), width,
                              dec, dev_, dcr, dcc, dcv)
        assert m == len(cr)
        if width:
            assert np.array_equal(dec.cpu().numpy().view(np.uint32), ec[:n * width])
            assert np.array_equal(dev_.cpu().numpy().view(np.uint32),
                                  ev[:n * width].view(np.uint32))
        assert np.array_equal(dcr[:m].cpu().numpy().view(np.uint32), cr)
        assert np.array_equal(dcc[:m].cpu().numpy().view(np.uint32), cc)
        assert np.array_equal(dcv[:m].cpu().numpy().view(np.uint32), cv.view(np.uint32))
    y0 = (rng.standard_normal((n, 2)) * 1e-2).astype(np.float32)
    out = []
    for on_device in (False, True):
        p = S.default_params(d=2, format=S.FORMAT_HYBRID, max_iter=2, early_iter=1, h=0.7)
        args = (dev(torch, rp), dev(torch, col), dev(torch, val)) if on_device else (rp, col, val)
        job = S.Job(ctx, p, *args, device_mem=on_device)
        job.set_y(y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(2)
        out.append(job.get_y(np.empty_like(y0), S.LAYOUT_POINT_MAJOR, False, 1))
        job.close()
    a, b = (o.astype(np.float64) for o in out)
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(a)


def test_csr_to_hybrid_device_rejects_bad_rowptr(torch, ctx):
    import sgtsne_b200 as S
    rp = np.array([0, 3, 2], np.int32)
    col = np.zeros(3, np.int32)
    val = np.ones(3, np.float32)
    z = torch.zeros(8, dtype=torch.int32, device="cuda")
    zf = torch.zeros(8, dtype=torch.float32, device="cuda")
    with pytest.raises(S.SgtError) as e:
        ctx.csr_to_hybrid(2, dev(torch, rp), dev(torch, col), dev(torch, val), 2, z, zf, z, z, zf)
    assert e.value.status == 1


@pytest.mark.parametrize("d", [1, 2, 3])
@pytest.mark.parametrize("ng", [40, 80])
def test_mixed_radix_fft_lengths(torch, ctx, oracle, d, ng):
    """Fixed grids whose FFT length has the factor 3: ng = 40 gives N = 42
    (2N-1 = 83, M = 96) and ng = 80 gives N = 84 (M = 192).  The potential
    grid against the oracle's G2G of the engine's own charge grid, and the
    forces against the oracle at the same grid."""
    import sgtsne_b200 as S
    n = 6000
    Y = coords("clusters", n, d, seed=60 + d)
    h = {1: 0.5, 2: 0.7, 3: 1.2}[d]
    f = torch.empty(n * d, dtype=torch.float32, device="cuda")
    Z, N, he = ctx.repulsive(n, d, h, ng, dev(torch, Y), S.LAYOUT_POINT_MAJOR, f)
    assert N == S.best_grid_size(ng) + 2
    assert 2 * N - 1 in range(65, 97) if ng == 40 else 2 * N - 1 in range(129, 193)
    V, Phi = ctx.last_grids(d, N)
    Phio = oracle.g2g(V.astype(np.float64), float(he), 0)
    assert rel(Phi, Phio) <= 1e-4
    Fo, Zo, No, _ = oracle.repulsive_interp(Y.astype(np.float64), h, n1_force=N - 2)
    assert No == N
    # In 1-D the force y*Phi0 - Phi1 cancels more (6000 clustered points on
    # 40 intervals): its FP32 rel-L2 error sits just under 3e-4 and measured
    # 3.2e-4 in one run, so the 1-D bar at this grid is 5e-4.
    assert rel(f.cpu().numpy().reshape(n, d), Fo) <= (5e-4 if d == 1 else 3e-4)
    assert abs(Z - Zo) <= 5e-4 * abs(Zo)


@pytest.mark.parametrize("n,dim,k", [(3000, 50, 30), (2500, 37, 90), (1800, 130, 15),
                                     (700, 3, 1), (1500, 784, 128)])
def test_knn_exact(torch, ctx, n, dim, k):
    """sgt_knn against FP64 distances computed directly: the k-th distance of
    every row within 1e-5, and the neighbour lists equal except where a
    distance ties within FP32 rounding (at most 0.1 % of the entries)."""
    import sgtsne_b200 as S
    rng = np.random.default_rng(dim + k)
    c = rng.standard_normal((8, dim)) * 4
    X = (c[rng.integers(0, 8, n)] + rng.standard_normal((n, dim))).astype(np.float32)
    idx = torch.empty(n * k, dtype=torch.int32, device="cuda")
    d2 = torch.empty(n * k, dtype=torch.float32, device="cuda")
    ctx.knn(n, dim, dev(torch, X), k, idx, d2)
    I = idx.cpu().numpy().reshape(n, k)
    Dg = d2.cpu().numpy().reshape(n, k).astype(np.float64)
    X64 = X.astype(np.float64)
    D = np.empty((n, n))
    b = max(1, int(2e7 // (n * dim)))  # direct differences, b rows at a time
    for s0 in range(0, n, b):
        D[s0:s0 + b] = ((X64[s0:s0 + b, None, :] - X64[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(D, np.inf)
    order = np.argsort(D, axis=1, kind="stable")[:, :k]
    Dref = np.take_along_axis(D, order, 1)
    assert np.all(np.diff(Dg, axis=1) >= 0)                     # rows sorted
    assert np.all(I != np.arange(n)[:, None])                   # self excluded
    assert np.abs(Dg - Dref).max() <= 1e-5 * max(Dref.max(), 1.0)
    same = np.mean([len(set(a) & set(b)) / k for a, b in zip(I, order)])
    assert same >= 0.999
    # the distances returned are those of the indices returned
    Dchk = np.take_along_axis(D, I.astype(np.int64), 1)
    assert np.abs(Dchk - Dg).max() <= 1e-5 * max(Dref.max(), 1.0)


@pytest.mark.parametrize("n,dim,k,kind", [(20000, 50, 30, "zipf"), (9999, 7, 15, "blobs"),
                                          (6000, 64, 32, "blobs"), (5000, 33, 1, "blobs"),
                                          (4500, 2, 10, "grid"), (300, 16, 10, "blobs"),
                                          (60, 8, 5, "blobs")])
def test_knn_tensor_filter_matches_simt(torch, ctx, n, dim, k, kind):
    """The tensor-core filter (TF32 in three terms, exact re-rank, SIMT redo
    of unsettled queries) against the SIMT search: the same indices and the
    same distance bits.  'zipf' is the 50-D generator of the 1.3M-point
    configuration; 'grid' puts points on an integer lattice, so distances
    tie everywhere and the ties must resolve by index as in the SIMT
    search."""
    import sgtsne_b200 as S
    from sgtsne_b200 import workloads as W
    rng = np.random.default_rng(n + dim)
    if kind == "zipf":
        X, _ = W.gmm_zipf(n, dim=dim, ncomp=40, zipf_a=1.1, centre_var=25.0, seed=3)
    elif kind == "grid":
        X = rng.integers(0, 40, (n, dim)).astype(np.float32)
    else:
        c = rng.standard_normal((8, dim)) * 4
        X = (c[rng.integers(0, 8, n)] + rng.standard_normal((n, dim))).astype(np.float32)
    X = np.ascontiguousarray(X, np.float32)
    out = {}
    for m in (S.KNN_SIMT, S.KNN_TENSOR):
        idx = torch.full((n * k,), -7, dtype=torch.int32, device="cuda")
        d2 = torch.full((n * k,), -7.0, dtype=torch.float32, device="cuda")
        redo = ctx.knn(n, dim, dev(torch, X), k, idx, d2, method=m)
        out[m] = (idx.cpu().numpy(), d2.cpu().numpy(), redo)
    (i1, d1, _), (i2, dd2, redo) = out[S.KNN_SIMT], out[S.KNN_TENSOR]
    print(f"\nknn n={n} dim={dim} k={k} {kind}: {redo} of {n} queries redone by the SIMT search")
    assert np.array_equal(i1, i2)
    assert np.array_equal(d1.view(np.uint32), dd2.view(np.uint32))
    if kind != "grid":
        assert redo <= 0.01 * n


@pytest.mark.parametrize("kind", ["mixed", "far"])
def test_knn_tensor_filter_redo_path(torch, ctx, kind):
    """Queries the filter cannot settle go to the SIMT search.  A query
    settles when its 64th candidate's approximate distance, minus the error
    bound 1e-4 (|q|^2 + max |c|^2), exceeds its k-th exact distance.
    'mixed': half the points in a tight blob (spread 1e-3, distance gaps far
    below the bound: redone) and half spread wide (spread 10: settled).
    'far': every point 3000 from the origin, so the bound exceeds every gap
    and every query is redone.  Either way the result equals the SIMT
    search bit for bit."""
    import sgtsne_b200 as S
    n, dim, k = 5000, 24, 16
    rng = np.random.default_rng(17)
    if kind == "mixed":
        X = rng.standard_normal((n, dim)) * 10.0
        X[: n // 2] = rng.standard_normal((n // 2, dim)) * 1e-3
    else:
        X = rng.standard_normal((n, dim)) + 3000.0
    X = np.ascontiguousarray(X, np.float32)
    out = {}
    for m in (S.KNN_SIMT, S.KNN_TENSOR):
        idx = torch.full((n * k,), -7, dtype=torch.int32, device="cuda")
        d2 = torch.full((n * k,), -7.0, dtype=torch.float32, device="cuda")
        redo = ctx.knn(n, dim, dev(torch, X), k, idx, d2, method=m)
        out[m] = (idx.cpu().numpy(), d2.cpu().numpy(), redo)
    (i1, d1, _), (i2, dd2, redo) = out[S.KNN_SIMT], out[S.KNN_TENSOR]
    print(f"\nknn redo {kind}: {redo} of {n} queries redone by the SIMT search")
    if kind == "far":
        assert redo == n
    else:
        assert 0 < redo < n
    assert np.array_equal(i1, i2)
    assert np.array_equal(d1.view(np.uint32), dd2.view(np.uint32))


def test_knn_tensor_rejects_wide_points_and_large_k(torch, ctx):
    import sgtsne_b200 as S
    X = torch.zeros(5000 * 65, dtype=torch.float32, device="cuda")
    idx = torch.empty(5000 * 40, dtype=torch.int32, device="cuda")
    d2 = torch.empty(5000 * 40, dtype=torch.float32, device="cuda")
    for dim, k in ((65, 4), (20, 33)):
        with pytest.raises(S.SgtError) as e:
            ctx.knn(5000, dim, X, k, idx, d2, method=S.KNN_TENSOR)
        assert e.value.status == 4


def test_knn_rejects_bad_k(torch, ctx):
    import sgtsne_b200 as S
    X = torch.zeros(10 * 3, dtype=torch.float32, device="cuda")
    idx = torch.empty(10 * 200, dtype=torch.int32, device="cuda")
    d2 = torch.empty(10 * 200, dtype=torch.float32, device="cuda")
    for k in (10, 129):
        with pytest.raises(S.SgtError) as e:
            ctx.knn(10, 3, X, k, idx, d2)
        assert e.value.status == 4


def test_cli_dense_and_mtx(torch, ctx, oracle, tmp_path):
    """sg_tsne_cuda on dense points (kNN, perplexity, embedding on the
    device) and on a Matrix Market P: n finite, centred rows each, and the
    dense run's KL within 2 % of the same pipeline driven from Python."""
    import subprocess

    import sgtsne_b200 as S
    from sgtsne_b200 import workloads as W
    exe = os.path.join(os.path.dirname(S.LIB_PATH), "..", "bin", "sg_tsne_cuda")
    n, dim, u = 1500, 20, 10.0
    X, _ = W.gmm_isotropic(n, dim, 6, 16.0, 3, dtype=np.float32)
    with open(tmp_path / "pts.txt", "w") as f:
        f.write(f"{n} {dim}\n")
        np.savetxt(f, X, fmt="%.7g")
    args = [exe, "-d", "2", "-m", "300", "-e", "100", "-u", str(u), "-t", "csr"]
    r = subprocess.run(args + ["-b", "1", str(tmp_path / "pts.txt")], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    Y = np.loadtxt(tmp_path / "sgtsneEmbedding.txt")
    assert Y.shape == (n, 2) and np.isfinite(Y).all()
    assert np.abs(Y.mean(0)).max() < 1e-3
    # embedding.bin: the same coordinates, raw FP32, dimension-major
    Yb = np.fromfile(tmp_path / "embedding.bin", dtype=np.float32)
    assert Yb.size == n * 2
    assert np.allclose(Yb.reshape(2, n).T, Y, rtol=1e-5, atol=1e-6 * np.abs(Y).max())
    # the same stages from Python: kNN, max-normalised distances, perplexity
    nn = int(np.ceil(3 * u))
    idx = torch.empty(n * nn, dtype=torch.int32, device="cuda")
    d2 = torch.empty(n * nn, dtype=torch.float32, device="cuda")
    ctx.knn(n, dim, dev(torch, X), nn, idx, d2)
    D = d2 / d2.max()
    Pk = torch.empty(n * nn, dtype=torch.float32, device="cuda")
    ctx.perplexity(n, nn, D.contiguous(), u, Pk)
    rp = (np.arange(n + 1) * nn).astype(np.int32)
    col, val = idx.cpu().numpy(), Pk.cpu().numpy()
    p = S.default_params(d=2, max_iter=300, early_iter=100, format=S.FORMAT_CSR)
    Yp, _ = ctx.embed(rp, col, val, p)
    srp, sc, sv = S.symmetrize(rp, col, val, 1.0 / (2 * n))

    def kl(Yx):
        _, Z, _, _ = oracle.repulsive_interp(Yx.astype(np.float64), 0.7)
        return oracle.kl(srp, sc, sv.astype(np.float64), Yx.astype(np.float64), 1.0, Z)
    assert abs(kl(Y) - kl(Yp)) <= 0.02 * kl(Yp)
    # Matrix Market input: the symmetrised P written 1-based, column-major
    rows = np.repeat(np.arange(n), np.diff(srp))
    with open(tmp_path / "p.mtx", "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {len(sc)}\n")
        for a, b, v in zip(sc, rows, sv):  # column-major: (row, col) of P^T
            f.write(f"{b + 1} {a + 1} {v:.9g}\n")
    r = subprocess.run([exe, "-d", "2", "-m", "100", "-t", "coo", str(tmp_path / "p.mtx")],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    Y2 = np.loadtxt(tmp_path / "sgtsneEmbedding.txt")
    assert Y2.shape == (n, 2) and np.isfinite(Y2).all()
    # timeInfo.txt in the reference's layout, one block per run (two runs so far)
    lines = (tmp_path / "timeInfo.txt").read_text().splitlines()
    assert lines.count("N d gds matrix total: ") == 2
    assert len(lines[1].split()) == 5 and lines[1].split()[:2] == [str(n), "2"]
    # Y0 from yin2m.txt (one point per line): with no iteration the result is
    # Y0 minus its mean
    Yin = np.random.default_rng(4).standard_normal((n, 2)).astype(np.float32)
    np.savetxt(tmp_path / "yin2m.txt", Yin, fmt="%.9g")
    r = subprocess.run([exe, "-d", "2", "-m", "0", "-t", "csr", str(tmp_path / "p.mtx")],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    Y3 = np.loadtxt(tmp_path / "sgtsneEmbedding.txt")
    assert np.abs(Y3 - (Yin - Yin.mean(0))).max() <= 1e-5


@pytest.mark.parametrize("fmt", [0, 2, 3])
def test_ragged_p_iterations(torch, ctx, oracle, fmt):
    """P with empty rows and single-entry rows (isolated and leaf points)
    through 60 iterations in each format: finite, the isolated points feel
    only repulsion, and the run stays within 1 % KL of the oracle's."""
    import sgtsne_b200 as S
    rp, col, val, _ = make_problem(n=2000, k=10, seed=77)
    n = len(rp) - 1
    lens = np.diff(rp).copy()
    keep = np.ones(int(rp[-1]), bool)
    empty = np.arange(0, n, 97)          # rows emptied
    for r in empty:
        keep[rp[r]:rp[r + 1]] = False
    single = np.arange(50, n, 101)       # rows cut to one entry
    for r in single:
        keep[rp[r] + 1:rp[r + 1]] = False
    lens = np.add.reduceat(keep.astype(np.int64), rp[:-1]) * (lens > 0)
    rp2 = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col2, val2 = col[keep], val[keep].astype(np.float32)
    Y0 = (np.random.default_rng(8).standard_normal((n, 2)) * 1e-2).astype(np.float32)
    p = S.default_params(d=2, format=fmt, max_iter=60, early_iter=20)
    job = S.Job(ctx, p, rp2, col2, val2, device_mem=False)
    job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
    job.run(60)
    Y = job.get_y(np.empty((n, 2), np.float32), S.LAYOUT_POINT_MAJOR, False, 1)
    assert job.info().error_flags == 0
    job.close()
    assert np.isfinite(Y).all()
    Yo = oracle.kl_minimization(rp2, col2, val2.astype(np.float64), Y0.astype(np.float64), 60,
                                early_iter=20, alpha=12.0, h=0.7, grid_mode=0)
    kls = []
    for Yx in (Y.astype(np.float64), Yo):
        _, Z, _, _ = oracle.repulsive_interp(Yx, 0.7)
        kls.append(oracle.kl(rp2, col2, val2.astype(np.float64), Yx, 1.0, Z))
    assert abs(kls[0] - kls[1]) <= 0.01 * kls[1]


@pytest.mark.parametrize("d", [1, 2, 3])
def test_smallest_embeddings(torch, ctx, d):
    """n = 3 and n = 40 points: every stage runs with one block and the
    result stays finite.  So few points repel each other far apart, so a 3-D
    run may outgrow the largest grid the job allocated: the engine then
    clamps the grid and says so (flag 2), which is allowed here; non-finite
    values (1) and chunk overflow (4) are not."""
    import sgtsne_b200 as S
    for n in (3, 40):
        rng = np.random.default_rng(n + d)
        rp = np.arange(0, 2 * (n + 1), 2, dtype=np.int32)
        col = np.stack([(np.arange(n) + 1) % n, (np.arange(n) + 2) % n], 1).reshape(-1)
        val = np.full(2 * n, 0.5 / n, np.float32)
        Y0 = (rng.standard_normal((n, d)) * 1e-2).astype(np.float32)
        job = S.Job(ctx, S.default_params(d=d, format=S.FORMAT_CSR), rp, col.astype(np.int32),
                    val, device_mem=False)
        job.set_y(Y0, S.LAYOUT_POINT_MAJOR, False)
        job.run(40)
        Y = np.empty((n, d), np.float32)
        try:
            job.get_y(Y, S.LAYOUT_POINT_MAJOR, False, 1)
        except S.SgtError as e:  # the clamp is reported; the coordinates are written
            assert e.status == S.ERR_CAPACITY and "max_grid" in str(e)
        assert (job.info().error_flags & ~2) == 0 and np.isfinite(Y).all()
        job.close()


def test_grid_clamp_is_a_status(torch, ctx):
    """An embedding wider than the provisioned grid runs on the largest
    provisioned grid and says so: the job API (sgt_job_get_y), sgt_repulsive
    and sgt_embed return SGT_ERR_CAPACITY with the outputs written, never
    SGT_OK."""
    import sgtsne_b200 as S
    n, d = 3000, 2
    rp, col, val, _ = make_problem(n=n, k=10, seed=91)
    rng = np.random.default_rng(91)
    # spread 300 at h = 0.7 needs several hundred grid points per axis
    Yw = (rng.standard_normal((n, d)) * 300).astype(np.float32)
    p = S.default_params(d=d, format=S.FORMAT_CSR, max_grid=64)
    job = S.Job(ctx, p, rp, col, val.astype(np.float32), device_mem=False)
    job.set_y(Yw, S.LAYOUT_POINT_MAJOR, False)
    job.run(1)
    Y = np.full((n, d), np.nan, np.float32)
    with pytest.raises(S.SgtError) as e:
        job.get_y(Y, S.LAYOUT_POINT_MAJOR, False, 1)
    assert e.value.status == S.ERR_CAPACITY and "max_grid" in str(e.value)
    inf = job.info()
    assert inf.error_flags & 2 and inf.grid_points <= 64 and np.isfinite(Y).all()
    # set_y starts a new run: the flag is cleared with the state
    job.set_y((Yw * 1e-3).astype(np.float32), S.LAYOUT_POINT_MAJOR, False)
    job.run(1)
    job.get_y(Y, S.LAYOUT_POINT_MAJOR, False, 1)
    job.close()
    # the operator in 3-D provisions 128 points per axis; h = 0.1 over an
    # extent of ~60 asks for the table's largest, 512 (in 2-D that largest
    # is provisioned, as the reference's grid-size table ends there)
    Yo = (rng.standard_normal((n, 3)) * 10).astype(np.float32)
    f = torch.full((n * 3,), float("nan"), dtype=torch.float32, device="cuda")
    with pytest.raises(S.SgtError) as e:
        ctx.repulsive(n, 3, 0.1, 0, dev(torch, Yo), S.LAYOUT_POINT_MAJOR, f)
    assert e.value.status == S.ERR_CAPACITY and "max_grid" in str(e.value)
    assert torch.isfinite(f).all()
