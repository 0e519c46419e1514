"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference's published runs use datasets that are not available here
(10x Genomics 1.3M, MNIST); these generators stand in for them with the
sizes, dimensions and cluster structure the configurations name:

  gmm_isotropic   n points in D dims from a c-component isotropic mixture,
                  centres ~ N(0, s2 I), unit variance, equal weights
  digits_like     n uint8-quantised 784-D vectors in 10 clusters (150 active
                  coordinates per template ~ U(0,255), kept with p = 0.9,
                  N(0, 20^2) noise, clipped to [0,255])
  gmm_zipf        n points in D dims, Zipf(a) component sizes, centres
                  ~ N(0, s2 I), covariance eigenvalues ~ U(0.2, 2) under
                  random rotations

P is built as the reference pipeline does: exact kNN (squared Euclidean,
self excluded), lambda or perplexity rescaling, symmetrisation
(P + P^T)/(2n).  kNN runs on the GPU through torch matrix products when a
device is given (setup only, outside every timed region), else with numpy.
"""
from __future__ import annotations

import numpy as np


def gmm_isotropic(n, dim=50, ncomp=10, centre_var=16.0, seed=0, dtype=np.float64):
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, np.sqrt(centre_var), size=(ncomp, dim))
    lab = rng.integers(0, ncomp, size=n)
    X = centres[lab] + rng.normal(0.0, 1.0, size=(n, dim))
    return X.astype(dtype), lab


def digits_like(n=60000, dim=784, ncomp=10, active=150, keep=0.9, noise=20.0, seed=0):
    rng = np.random.default_rng(seed)
    templates = np.zeros((ncomp, dim), np.float32)
    for c in range(ncomp):
        idx = rng.choice(dim, size=active, replace=False)
        templates[c, idx] = rng.uniform(0, 255, size=active)
    lab = rng.integers(0, ncomp, size=n)
    X = np.empty((n, dim), np.float32)
    for s in range(0, n, 8192):
        e = min(n, s + 8192)
        t = templates[lab[s:e]]
        mask = (t > 0) & (rng.random(t.shape) < keep)
        x = np.where(mask, t, 0.0) + rng.normal(0.0, noise, size=t.shape)
        X[s:e] = np.clip(x, 0, 255).astype(np.uint8).astype(np.float32)
    return X, lab


def gmm_zipf(n, dim=50, ncomp=40, zipf_a=1.1, centre_var=25.0, seed=0, dtype=np.float32):
    rng = np.random.default_rng(seed)
    w = 1.0 / np.arange(1, ncomp + 1) ** zipf_a
    w /= w.sum()
    sizes = rng.multinomial(n, w)
    X = np.empty((n, dim), dtype)
    lab = np.empty(n, np.int32)
    pos = 0
    for c in range(ncomp):
        m = int(sizes[c])
        if m == 0:
            continue
        q, _ = np.linalg.qr(rng.normal(size=(dim, dim)))
        ev = rng.uniform(0.2, 2.0, size=dim)
        A = q * np.sqrt(ev)  # cov = q diag(ev) q^T
        mu = rng.normal(0.0, np.sqrt(centre_var), size=dim)
        X[pos:pos + m] = (mu + rng.normal(size=(m, dim)) @ A.T).astype(dtype)
        lab[pos:pos + m] = c
        pos += m
    perm = rng.permutation(n)  # datasets arrive in no particular order
    return X[perm], lab[perm]


def knn_numpy(X, k, block=2048):
    """Exact kNN (squared Euclidean), self excluded; returns (idx, d2) n*k."""
    X = np.asarray(X, np.float64)
    n = X.shape[0]
    sq = (X * X).sum(1)
    idx = np.empty((n, k), np.int32)
    d2 = np.empty((n, k), np.float64)
    for s in range(0, n, block):
        e = min(n, s + block)
        D = sq[s:e, None] + sq[None, :] - 2.0 * X[s:e] @ X.T
        D[np.arange(e - s), np.arange(s, e)] = np.inf
        part = np.argpartition(D, k, axis=1)[:, :k]
        pd = np.take_along_axis(D, part, 1)
        o = np.argsort(pd, axis=1, kind="stable")
        idx[s:e] = np.take_along_axis(part, o, 1)
        d2[s:e] = np.maximum(np.take_along_axis(pd, o, 1), 0.0)
    return idx, d2


def knn_engine(ctx, X, k, device="cuda"):
    """Exact kNN through the engine (sgt_knn): returns device tensors
    idx (n, k) int32 and d2 (n, k) float32, rows sorted, self excluded."""
    import torch
    Xd = torch.as_tensor(np.ascontiguousarray(X, np.float32), device=device)
    n, dim = Xd.shape
    idx = torch.empty((n, k), dtype=torch.int32, device=device)
    d2 = torch.empty((n, k), dtype=torch.float32, device=device)
    torch.cuda.synchronize(device)  # X written by torch before the engine reads it
    ctx.knn(n, dim, Xd, k, idx, d2)
    return idx, d2


def knn_torch(X, k, device="cuda", block=4096):
    """Exact kNN on the GPU with fp32 matrix products (setup only)."""
    import torch
    Xt = torch.as_tensor(np.asarray(X, np.float32), device=device)
    n = Xt.shape[0]
    sq = (Xt * Xt).sum(1)
    idx = torch.empty((n, k), dtype=torch.int32, device=device)
    d2 = torch.empty((n, k), dtype=torch.float32, device=device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for s in range(0, n, block):
            e = min(n, s + block)
            D = sq[s:e, None] + sq[None, :] - 2.0 * (Xt[s:e] @ Xt.T)
            D[torch.arange(e - s, device=device), torch.arange(s, e, device=device)] = float("inf")
            v, i = torch.topk(D, k, dim=1, largest=False, sorted=True)
            idx[s:e] = i.to(torch.int32)
            d2[s:e] = v.clamp_min(0.0)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return idx, d2


def knn_csr(idx, vals):
    """Row-wise kNN lists to CSR (rows of k entries)."""
    n, k = idx.shape
    rowptr = (np.arange(n + 1, dtype=np.int64) * k).astype(np.int32)
    return rowptr, np.ascontiguousarray(idx.reshape(-1), np.int32), \
        np.ascontiguousarray(vals.reshape(-1))
