"""ctypes view of liboracle.so -- the CPU restatement of the SG-t-SNE path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py, never by the engine.  Each
wrapper names the C function (oracle/sgt_oracle.c) it calls; the C file cites
the reference source each one restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile oracle/liboracle.so with make (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "sgt_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        build()
    L = C.CDLL(path)
    sig = {
        "orc_best_grid_size": (C.c_int, [C.c_int]),
        "orc_grid_points_h": (C.c_int, [C.c_double, C.c_double]),
        "orc_csr_to_coo": (None, [C.c_int, C.c_int, _i32p, _i32p]),
        "orc_ell_width_cusp": (C.c_int, [C.c_int, _i32p]),
        "orc_csr_to_hybrid": (C.c_int, [C.c_int, _i32p, _i32p, _f32p, C.c_int,
                                         _u32p, _f32p, _u32p, _u32p, _f32p]),
        "orc_symmetrize": (C.c_int, [C.c_int, _i32p, _i32p, _f64p, C.c_double,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
        "orc_attractive": (None, [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                   _f64p, C.c_int]),
        "orc_repulsive_exact": (C.c_double, [C.c_int, C.c_int, _f64p, _f64p, C.c_int]),
        "orc_repulsive_interp": (C.c_double, [C.c_int, C.c_int, C.c_double, C.c_int,
                                               _f64p, _f64p, C.POINTER(C.c_int),
                                               C.POINTER(C.c_double), C.c_int, C.c_int]),
        "orc_s2g": (None, [C.c_int, C.c_int, C.c_int, _f64p, _f64p, _f64p]),
        "orc_g2g": (None, [C.c_int, C.c_int, C.c_int, C.c_double, _f64p, _f64p,
                            C.c_int, C.c_int]),
        "orc_g2s": (None, [C.c_int, C.c_int, C.c_int, _f64p, _f64p, _f64p]),
        "orc_bins_f32": (C.c_int, [C.c_int, C.c_int, C.c_float, C.c_int, _f32p,
                                    _u32p, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_float)]),
        "orc_fft": (None, [C.c_int, _f64p, _f64p, C.c_int]),
        "orc_update": (None, [C.c_int, C.c_int, _f64p, _f64p, _f64p, _f64p,
                               C.c_double, C.c_double, C.c_int]),
        "orc_kl_minimization": (None, [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                        C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_int, C.c_int, C.c_void_p, C.c_int]),
        "orc_kl": (C.c_double, [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                 C.c_double, C.c_double]),
        "orc_lambda_rescale_f32": (None, [C.c_int, _i32p, _f32p, C.c_float, C.c_void_p]),
        "orc_lambda_rescale": (None, [C.c_int, _i32p, _f64p, C.c_double, C.c_int,
                                       C.c_void_p]),
        "orc_perplexity": (None, [C.c_int, C.c_int, _f64p, C.c_double, _f64p, C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def best_grid_size(ng: int) -> int:
    return lib().orc_best_grid_size(int(ng))


def grid_points_h(maxy: float, h: float) -> int:
    return lib().orc_grid_points_h(float(maxy), float(h))


def csr_to_coo(rowptr):
    rowptr = _c(rowptr, np.int32)
    n = rowptr.size - 1
    nnz = int(rowptr[-1])
    rows = np.empty(nnz, np.int32)
    lib().orc_csr_to_coo(n, nnz, rowptr, rows)
    return rows


def ell_width_cusp(rowptr) -> int:
    rowptr = _c(rowptr, np.int32)
    return lib().orc_ell_width_cusp(rowptr.size - 1, rowptr)


def csr_to_hybrid(rowptr, col, val, width):
    rowptr = _c(rowptr, np.int32)
    col = _c(col, np.int32)
    val = _c(val, np.float32)
    n = rowptr.size - 1
    nnz = int(rowptr[-1])
    ec = np.empty(n * width, np.uint32)
    ev = np.empty(n * width, np.float32)
    cr = np.empty(max(nnz, 1), np.uint32)
    cc = np.empty(max(nnz, 1), np.uint32)
    cv = np.empty(max(nnz, 1), np.float32)
    k = lib().orc_csr_to_hybrid(n, rowptr, col, val, int(width), ec, ev, cr, cc, cv)
    return ec, ev, cr[:k].copy(), cc[:k].copy(), cv[:k].copy()


def symmetrize(rowptr, col, val, scale):
    rowptr = _c(rowptr, np.int32)
    col = _c(col, np.int32)
    val = _c(val, np.float64)
    n = rowptr.size - 1
    L = lib()
    nnz = L.orc_symmetrize(n, rowptr, col, val, float(scale), None, None, None)
    orp = np.empty(n + 1, np.int32)
    oc = np.empty(nnz, np.int32)
    ov = np.empty(nnz, np.float64)
    L.orc_symmetrize(n, rowptr, col, val, float(scale), orp.ctypes.data,
                     oc.ctypes.data, ov.ctypes.data)
    return orp, oc, ov


def attractive(rowptr, col, val, Y, nthreads=0):
    Y = _c(Y, np.float64)
    n, d = Y.shape
    F = np.empty_like(Y)
    lib().orc_attractive(n, d, _c(rowptr, np.int32), _c(col, np.int32),
                         _c(val, np.float64), Y, F, int(nthreads))
    return F


def repulsive_exact(Y, nthreads=0):
    Y = _c(Y, np.float64)
    n, d = Y.shape
    F = np.zeros_like(Y)
    Z = lib().orc_repulsive_exact(n, d, Y, F, int(nthreads))
    return F, Z


def repulsive_interp(Y, h, n1_force=0, conv_mode=0, nthreads=0):
    """Returns (F, Z, grid_points, h_eff)."""
    Y = _c(Y, np.float64)
    n, d = Y.shape
    F = np.empty_like(Y)
    gp = C.c_int(0)
    he = C.c_double(0)
    Z = lib().orc_repulsive_interp(n, d, float(h), int(n1_force), Y, F,
                                   C.byref(gp), C.byref(he), int(conv_mode),
                                   int(nthreads))
    return F, Z, gp.value, he.value


def s2g(ys, q, N):
    ys = _c(ys, np.float64)
    n, d = ys.shape
    V = np.empty((d + 1,) + (N,) * d, np.float64)
    lib().orc_s2g(n, d, int(N), ys, _c(q, np.float64), V.reshape(-1))
    return V


def g2g(V, h_eff, conv_mode=0, nthreads=0):
    V = _c(V, np.float64)
    m = V.shape[0]
    d = V.ndim - 1
    N = V.shape[1]
    Phi = np.empty_like(V)
    lib().orc_g2g(d, N, m, float(h_eff), V.reshape(-1), Phi.reshape(-1),
                  int(conv_mode), int(nthreads))
    return Phi


def g2s(ys, PhiGrid):
    ys = _c(ys, np.float64)
    n, d = ys.shape
    N = PhiGrid.shape[1]
    out = np.empty((n, d + 1), np.float64)
    lib().orc_g2s(n, d, int(N), ys, _c(PhiGrid, np.float64).reshape(-1), out)
    return out


def bins_f32(Y, h, n1_force=0):
    """FP32 CUDA-path binning; returns (bins uint32 n*d, scaled, shifted, N, maxy)."""
    Y = _c(Y, np.float32)
    n, d = Y.shape
    bins = np.empty((n, d), np.uint32)
    sc = np.empty((n, d), np.float32)
    sh = np.empty((n, d), np.float32)
    mx = C.c_float(0)
    N = lib().orc_bins_f32(n, d, float(h), int(n1_force), Y, bins,
                           sc.ctypes.data, sh.ctypes.data, C.byref(mx))
    return bins, sc, sh, N, mx.value


def fft(x, sign=-1):
    x = np.asarray(x, np.complex128)
    re = np.ascontiguousarray(x.real)
    im = np.ascontiguousarray(x.imag)
    lib().orc_fft(x.size, re, im, int(sign))
    return re + 1j * im


def kl_minimization(rowptr, col, val, Y0, max_iter, early_iter=250, alpha=12.0,
                    h=0.7, grid_mode=0, ng=50, nthreads=0, return_zeta=False):
    Y = _c(Y0, np.float64).copy()
    n, d = Y.shape
    z = np.zeros(max(max_iter, 1), np.float64)
    lib().orc_kl_minimization(n, d, _c(rowptr, np.int32), _c(col, np.int32),
                              _c(val, np.float64), Y, int(max_iter), int(early_iter),
                              float(alpha), float(h), int(grid_mode), int(ng),
                              z.ctypes.data, int(nthreads))
    return (Y, z[:max_iter]) if return_zeta else Y


def kl(rowptr, col, val, Y, alpha, zeta):
    Y = _c(Y, np.float64)
    n, d = Y.shape
    return lib().orc_kl(n, d, _c(rowptr, np.int32), _c(col, np.int32),
                        _c(val, np.float64), Y, float(alpha), float(zeta))


def lambda_rescale_f32(rowptr, val, lam):
    v = _c(val, np.float32).copy()
    rowptr = _c(rowptr, np.int32)
    sig = np.empty(rowptr.size - 1, np.float32)
    lib().orc_lambda_rescale_f32(rowptr.size - 1, rowptr, v, float(lam), sig.ctypes.data)
    return v, sig


def lambda_rescale(rowptr, val, lam, dist=True):
    v = _c(val, np.float64).copy()
    rowptr = _c(rowptr, np.int32)
    sig = np.empty(rowptr.size - 1, np.float64)
    lib().orc_lambda_rescale(rowptr.size - 1, rowptr, v, float(lam), int(bool(dist)),
                             sig.ctypes.data)
    return v, sig


def perplexity(D, perp, nthreads=0):
    D = _c(D, np.float64)
    n, k1 = D.shape
    P = np.empty((n, k1 - 1), np.float64)
    lib().orc_perplexity(n, k1 - 1, D, float(perp), P, int(nthreads))
    return P
