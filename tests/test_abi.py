"""CPU tests of the C-ABI library: it loads, exports every symbol the header
declares, and its host-side routines agree bit-exactly with the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO, make_problem


@pytest.fixture(scope="module")
def S():
    import sgtsne_b200 as S
    if not os.path.exists(S.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "gpu-sg-sne_b200")], check=True)
    S.load()
    return S


def header_functions():
    src = open(os.path.join(REPO, "include", "sgtsne_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sgt_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(S):
    import ctypes
    names = header_functions()
    assert len(names) >= 25
    lib = ctypes.CDLL(S.LIB_PATH)
    for nm in names:
        assert hasattr(lib, nm), nm
    assert set(names) == set(S.SIGNATURES), set(names) ^ set(S.SIGNATURES)
    assert S.load().sgt_abi_version() == 1


def header_arg_counts():
    """Parameter count of every function prototype in the header."""
    src = open(os.path.join(REPO, "include", "sgtsne_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(sgt_[a-z0-9_]+)\s*\(([^()]*)\)\s*;", src):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_binding_argument_counts_match_header(S):
    """Every ctypes signature takes as many arguments as the C prototype."""
    counts = header_arg_counts()
    assert len(counts) >= 25
    for nm, (_, args) in S.SIGNATURES.items():
        assert nm in counts, nm
        assert len(args) == counts[nm], (nm, len(args), counts[nm])


def test_no_device_is_reported_not_faked(S):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    import ctypes
    h = ctypes.c_void_p()
    assert S.load().sgt_create(0, ctypes.byref(h)) == 6  # SGT_ERR_NO_DEVICE


def test_best_grid_size_matches_oracle(S, oracle):
    for ng in range(0, 620):
        assert S.best_grid_size(ng) == oracle.best_grid_size(ng)


def test_ell_width_and_hybrid_bit_exact(S, oracle):
    rp, col, val, _ = make_problem(n=1500, k=12)
    v32 = val.astype(np.float32)
    assert S.ell_width(rp) == oracle.ell_width_cusp(rp)
    for W in (0, 3, S.ell_width(rp), 40):
        a = S.csr_to_hybrid(rp, col, v32, W)
        b = oracle.csr_to_hybrid(rp, col, v32, W)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_symmetrize_pattern_bit_exact(S, oracle):
    from sgtsne_b200 import workloads as W
    X, _ = W.gmm_isotropic(1200, 12, 5, 16.0, 4)
    idx, d2 = W.knn_numpy(X, 10)
    rp, col, val = W.knn_csr(idx, d2)
    v = (np.exp(-d2 / d2.max())).reshape(-1).astype(np.float32)
    a_rp, a_c, a_v = S.symmetrize(rp, col, v, 1.0 / 2400)
    b_rp, b_c, b_v = oracle.symmetrize(rp, col, v.astype(np.float64), 1.0 / 2400)
    assert np.array_equal(a_rp, b_rp) and np.array_equal(a_c, b_c)
    assert np.allclose(a_v, b_v, rtol=2e-7, atol=0)


def test_symmetrize_rejects_bad_columns(S):
    rp = np.array([0, 1, 2], np.int32)
    col = np.array([1, 5], np.int32)
    with pytest.raises(S.SgtError):
        S.symmetrize(rp, col, np.ones(2, np.float32), 1.0)


def test_job_footprint_host_rule(S):
    """Admission footprint: host arithmetic only (no device), monotone in n
    and nnz, larger for d = 3 (FFT planes of M^3), zero for bad input."""
    p2 = S.default_params(d=2, format=S.FORMAT_CSR)
    p3 = S.default_params(d=3, format=S.FORMAT_CSR)
    a = S.job_footprint(p2, 10000, 300000)
    assert a > 8 * 300000
    assert S.job_footprint(p2, 20000, 300000) > a
    assert S.job_footprint(p2, 10000, 600000) > a
    assert S.job_footprint(p3, 10000, 300000) > a
    assert S.job_footprint(S.default_params(d=4), 10000, 10) == 0
    small = S.default_params(d=3, format=S.FORMAT_CSR, max_grid=64)
    assert S.job_footprint(small, 10000, 300000) < S.job_footprint(p3, 10000, 300000)
