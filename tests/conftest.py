import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "gpu-sg-sne_b200", "python"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    # GPU tests run only where a CUDA device exists; elsewhere they are
    # skipped (select them with -m gpu on a machine with a B200).
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def make_problem(n=2000, dim=20, ncomp=6, k=15, lam=1.0, seed=0):
    """Symmetric stochastic P from a seeded mixture, built with the oracle:
    exact kNN -> lambda bisection on squared distances -> (P + P^T)/(2n)."""
    from oracle import oracle as O
    from sgtsne_b200 import workloads as W
    X, lab = W.gmm_isotropic(n, dim, ncomp, 16.0, seed)
    idx, d2 = W.knn_numpy(X, k)
    rp, col, val = W.knn_csr(idx, d2)
    v, _ = O.lambda_rescale(rp, val, lam, dist=True)
    srp, sc, sv = O.symmetrize(rp, col, v, 1.0 / (2 * n))
    return srp, sc, sv, lab


@pytest.fixture(scope="session")
def problem():
    return make_problem()
