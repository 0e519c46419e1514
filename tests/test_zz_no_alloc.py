"""sgt_repulsive_noalloc against sgt_repulsive, through the C ABI.

The no-allocation entry point is for callers that cannot allocate device
memory (their own pool owns the GPU, or a cudaMalloc/cudaFree pair would
stall a latency-sensitive loop).  Its scratch is one fixed array inside the
library that every call reuses, so this test makes two calls in a row on
different inputs and checks each against the allocating entry point with the
parity tolerances of tests/test_gpu_parity.py (forces rel L2 <= 3e-4,
Z rel <= 5e-4; the two paths differ only in the order of FP32 atomics).
This file is collected last; it passes alone in a fresh process and after
the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_allocating_entry_two_calls():
    import torch

    import sgtsne_b200 as S
    ctx = S.Context(0)
    try:
        for call, (n, d, seed) in enumerate([(20000, 2, 1), (12000, 1, 2)]):
            rng = np.random.default_rng(seed)
            Y = (rng.standard_normal((n, d)) * 6).astype(np.float32)
            yd = torch.as_tensor(Y).cuda()
            fa = torch.empty(n * d, dtype=torch.float32, device="cuda")
            fb = torch.empty(n * d, dtype=torch.float32, device="cuda")
            za, na, ha = ctx.repulsive(n, d, 0.7, 0, yd, S.LAYOUT_POINT_MAJOR, fa)
            zb, nb, hb = ctx.repulsive_noalloc(n, d, 0.7, 0, yd, S.LAYOUT_POINT_MAJOR, fb)
            assert nb == na and hb == ha, (call, na, nb, ha, hb)
            assert abs(zb - za) <= 5e-4 * abs(za), (call, za, zb)
            assert _rel(fb.cpu().numpy(), fa.cpu().numpy()) <= 3e-4, call
    finally:
        ctx.close()


def test_noalloc_fixed_grid_dim_major():
    """The fixed-grid path (ng_fixed > 0) and dim-major input and output,
    against the allocating entry point, on two calls in a row."""
    import torch

    import sgtsne_b200 as S
    ctx = S.Context(0)
    try:
        for call, (n, d, ng, seed) in enumerate([(16000, 2, 50, 4), (9000, 1, 200, 5)]):
            rng = np.random.default_rng(seed)
            Y = (rng.standard_normal((n, d)) * 5).astype(np.float32)
            ydm = torch.as_tensor(np.ascontiguousarray(Y.T)).cuda()  # y[i + k n]
            fa = torch.empty(n * d, dtype=torch.float32, device="cuda")
            fb = torch.empty(n * d, dtype=torch.float32, device="cuda")
            za, na, ha = ctx.repulsive(n, d, 0.7, ng, ydm, S.LAYOUT_DIM_MAJOR, fa)
            zb, nb, hb = ctx.repulsive_noalloc(n, d, 0.7, ng, ydm, S.LAYOUT_DIM_MAJOR, fb)
            assert na == S.best_grid_size(ng) + 2
            assert nb == na and hb == ha, (call, na, nb, ha, hb)
            assert abs(zb - za) <= 5e-4 * abs(za), (call, za, zb)
            assert _rel(fb.cpu().numpy(), fa.cpu().numpy()) <= 3e-4, call
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    import torch

    import sgtsne_b200 as S
    ctx = S.Context(0)
    try:
        y = torch.zeros(40000 * 2, dtype=torch.float32, device="cuda")
        f = torch.empty_like(y)
        with pytest.raises(S.SgtError) as e:
            ctx.repulsive_noalloc(40000, 2, 0.7, 0, y, S.LAYOUT_POINT_MAJOR, f)
        assert e.value.status == 1 and "32768" in str(e.value)
        # a 2-D embedding too wide for the 128-point grid is refused too
        Y = (np.random.default_rng(3).standard_normal((5000, 2)) * 200).astype(np.float32)
        yd = torch.as_tensor(Y).cuda()
        f2 = torch.empty(5000 * 2, dtype=torch.float32, device="cuda")
        with pytest.raises(S.SgtError) as e:
            ctx.repulsive_noalloc(5000, 2, 0.7, 0, yd, S.LAYOUT_POINT_MAJOR, f2)
        assert e.value.status == 1 and "128" in str(e.value)
        # a fixed 2-D grid above 128 points per axis is refused before any work
        f3 = torch.full((5000 * 2,), 7.0, dtype=torch.float32, device="cuda")
        with pytest.raises(S.SgtError) as e:
            ctx.repulsive_noalloc(5000, 2, 0.7, 127, yd, S.LAYOUT_POINT_MAJOR, f3)
        assert e.value.status == 1 and "128" in str(e.value)
        assert bool((f3 == 7.0).all())
    finally:
        ctx.close()
