"""ctypes binding of libsgtsne_b200.so (include/sgtsne_b200.h).

The engine is CUDA + C++ behind a C ABI; this module only marshals
arguments.  Device buffers are passed as torch CUDA tensors (used purely as
device memory), host buffers as numpy arrays.  There is no fallback: if the
shared library is missing, load() raises.

Ordering: the engine queues its work on the context's stream (its own
non-blocking stream unless Context.set_stream names another).  Tensors that
torch writes on a different stream must be complete (synchronise, or share
the stream with set_stream) before an engine call reads them, and engine
results must be complete before torch reads them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.abspath(os.path.join(_HERE, "..", ".."))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libsgtsne_b200.so")
REPO = os.path.abspath(os.path.join(PKG_DIR, ".."))
HEADER = os.path.join(REPO, "include", "sgtsne_b200.h")

FORMAT_CSR, FORMAT_COO, FORMAT_HYBRID = 0, 2, 3
KNN_AUTO, KNN_SIMT, KNN_TENSOR = 0, 1, 2
LAYOUT_DIM_MAJOR, LAYOUT_POINT_MAJOR = 0, 1
GRID_H, GRID_FIXED = 0, 1
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
          4: "unsupported", 5: "non-finite values", 6: "no CUDA device",
          7: "device capacity reached"}
ERR_CAPACITY = 7


class SgtError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


class Params(C.Structure):
    """Mirror of sgt_params (field order of tsneparams, CU/types.hpp:55-72)."""
    _fields_ = [("d", C.c_int), ("lambda_", C.c_float), ("alpha", C.c_float),
                ("max_iter", C.c_int), ("early_iter", C.c_int), ("n", C.c_int),
                ("h", C.c_float), ("drop_leaf", C.c_int), ("np", C.c_int),
                ("format", C.c_int), ("bs", C.c_int), ("compute_error", C.c_int),
                ("ng", C.c_int), ("sim", C.c_int), ("grid_mode", C.c_int),
                ("lambda_dist", C.c_int), ("max_grid", C.c_int), ("kl_every", C.c_int),
                ("seed", C.c_uint64), ("relayout_every", C.c_int),
                ("locality_order", C.c_int)]


class JobInfo(C.Structure):
    _fields_ = [("iter", C.c_int), ("grid_points", C.c_int), ("h_eff", C.c_float),
                ("zeta", C.c_double), ("kl", C.c_double), ("error_flags", C.c_int),
                ("nnz", C.c_long), ("row_group", C.c_int), ("tune_ms", C.c_float * 4)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_active", C.c_int),
                ("iters_per_round", C.c_int), ("rounds_ahead", C.c_int)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("status", C.c_int), ("n", C.c_int), ("d", C.c_int),
                ("iters", C.c_int), ("footprint", C.c_size_t), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double)]


REQ_WAITING, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

# every symbol the header declares, with (restype, argtypes)
_vp, _i, _l, _f, _d = C.c_void_p, C.c_int, C.c_long, C.c_float, C.c_double
SIGNATURES = {
    "sgt_params_default": (None, [C.POINTER(Params)]),
    "sgt_abi_version": (_i, []),
    "sgt_status_string": (C.c_char_p, [_i]),
    "sgt_create": (_i, [_i, C.POINTER(_vp)]),
    "sgt_destroy": (None, [_vp]),
    "sgt_set_stream": (_i, [_vp, _vp]),
    "sgt_last_error": (C.c_char_p, [_vp]),
    "sgt_embed": (_i, [_vp, _i, _vp, _vp, _vp, C.POINTER(Params), _vp, _vp, _vp]),
    "sgt_job_create": (_i, [_vp, C.POINTER(Params), _i, _vp, _vp, _vp, _i, C.POINTER(_vp)]),
    "sgt_job_destroy": (None, [_vp]),
    "sgt_job_set_y": (_i, [_vp, _vp, _i, _i]),
    "sgt_job_run": (_i, [_vp, _i]),
    "sgt_job_prepare": (_i, [_vp]),
    "sgt_job_run_timed": (_i, [_vp, _i, _vp]),
    "sgt_job_get_y": (_i, [_vp, _vp, _i, _i, _i]),
    "sgt_job_get_info": (_i, [_vp, C.POINTER(JobInfo)]),
    "sgt_job_kl": (_i, [_vp, _d, C.POINTER(_d)]),
    "sgt_job_profile": (_i, [_vp, _i, _vp]),
    "sgt_job_repulsive_error": (_i, [_vp, C.POINTER(_d)]),
    "sgt_batch_create": (_i, [_vp, _i, C.POINTER(_vp), _i, C.POINTER(_vp)]),
    "sgt_batch_run": (_i, [_vp, _i]),
    "sgt_batch_destroy": (None, [_vp]),
    "sgt_batch_step": (_i, [_vp, _i, C.POINTER(_vp), _i]),
    "sgt_job_footprint": (C.c_size_t, [C.POINTER(Params), _i, _l]),
    "sgt_server_config_default": (None, [C.POINTER(ServerConfig)]),
    "sgt_server_create": (_i, [_i, C.POINTER(ServerConfig), C.POINTER(_vp)]),
    "sgt_server_destroy": (None, [_vp]),
    "sgt_server_submit": (_i, [_vp, C.POINTER(Params), _i, _vp, _vp, _vp, _vp, _vp,
                               C.POINTER(C.c_longlong)]),
    "sgt_server_poll": (_i, [_vp, _d, C.POINTER(C.c_longlong), _i, C.POINTER(_i)]),
    "sgt_server_request_info": (_i, [_vp, C.c_longlong, C.POINTER(RequestInfo)]),
    "sgt_server_now": (_d, [_vp]),
    "sgt_attractive": (_i, [_vp, _i, _i, _i, _l, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "sgt_repulsive": (_i, [_vp, _i, _i, _f, _i, _vp, _i, _vp, C.POINTER(_d),
                           C.POINTER(_i), C.POINTER(_f)]),
    "sgt_repulsive_noalloc": (_i, [_vp, _i, _i, _f, _i, _vp, _i, _vp, C.POINTER(_d),
                                   C.POINTER(_i), C.POINTER(_f)]),
    "sgt_bins": (_i, [_vp, _i, _i, _f, _i, _vp, _i, _vp, C.POINTER(_i)]),
    "sgt_last_grids": (_i, [_vp, _vp, _vp]),
    "sgt_best_grid_size": (_i, [_i]),
    "sgt_kl": (_i, [_vp, _i, _i, _l, _vp, _vp, _vp, _vp, _i, _d, _d, C.POINTER(_d)]),
    "sgt_lambda_bisect": (_i, [_vp, _i, _vp, _vp, _f, _i, _vp]),
    "sgt_perplexity": (_i, [_vp, _i, _i, _vp, _f, _vp, _vp]),
    "sgt_csr_to_coo": (_i, [_vp, _i, _l, _vp, _vp]),
    "sgt_ell_width": (_i, [_i, _vp]),
    "sgt_csr_to_hybrid": (_i, [_i, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, C.POINTER(_l)]),
    "sgt_symmetrize": (_i, [_i, _vp, _vp, _vp, _f, _vp, _vp, _vp, C.POINTER(_l)]),
    "sgt_symmetrize_device": (_i, [_vp, _i, _l, _vp, _vp, _vp, _f, _vp, _vp, _vp, C.POINTER(_l)]),
    "sgt_knn": (_i, [_vp, _i, _i, _vp, _i, _vp, _vp]),
    "sgt_knn_ex": (_i, [_vp, _i, _i, _vp, _i, _vp, _vp, _i, C.POINTER(_i)]),
    "sgt_csr_to_hybrid_device": (_i, [_vp, _i, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp,
                                      C.POINTER(_l)]),
    "sgt_shard_grid_floats": (C.c_size_t, [C.POINTER(Params)]),
    "sgt_shard_create": (_i, [_vp, C.POINTER(Params), _i, _i, _i, _vp, _vp, _vp, _i, _vp, _vp,
                              C.c_size_t, _vp, C.POINTER(_vp)]),
    "sgt_shard_destroy": (None, [_vp]),
    "sgt_shard_set_y": (_i, [_vp, _vp, _i, _i]),
    "sgt_shard_scatter": (_i, [_vp]),
    "sgt_shard_gather": (_i, [_vp]),
    "sgt_shard_update": (_i, [_vp]),
    "sgt_shard_get_y": (_i, [_vp, _vp, _i, _i, _i]),
    "sgt_shard_get_info": (_i, [_vp, C.POINTER(JobInfo)]),
}

_LIB = None


def load(path: str | None = None):
    """Load the engine library (raises if it is missing -- no fallback)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} not built; run `make -C gpu-sg-sne_b200`")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def default_params(**kw) -> Params:
    p = Params()
    load().sgt_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, "lambda_" if k == "lambda" else k, v)
    return p


def _ptr(x):
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return C.c_void_p(x.data_ptr())
    if isinstance(x, np.ndarray):
        assert x.flags["C_CONTIGUOUS"]
        return C.c_void_p(x.ctypes.data)
    return x


class Context:
    """One engine context on one device (sgt_create)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        st = self.lib.sgt_create(int(device), C.byref(h))
        if st != 0:
            raise SgtError(st, "sgt_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.sgt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st, what=""):
        if st != 0:
            raise SgtError(st, f"{what}: {self.lib.sgt_last_error(self.h).decode()}")

    def set_stream(self, stream_ptr):
        self.check(self.lib.sgt_set_stream(self.h, C.c_void_p(stream_ptr)), "set_stream")

    # ---- operators (device tensors) ----
    def attractive(self, fmt, n, d, nnz, rowptr, coo_rows, col, val, y, layout, f):
        self.check(self.lib.sgt_attractive(self.h, fmt, n, d, nnz, _ptr(rowptr), _ptr(coo_rows),
                                           _ptr(col), _ptr(val), _ptr(y), layout, _ptr(f)),
                   "attractive")

    def repulsive(self, n, d, h, ng_fixed, y, layout, f):
        z = C.c_double()
        gp = C.c_int()
        he = C.c_float()
        self.check(self.lib.sgt_repulsive(self.h, n, d, float(h), int(ng_fixed), _ptr(y), layout,
                                          _ptr(f), C.byref(z), C.byref(gp), C.byref(he)),
                   "repulsive")
        return z.value, gp.value, he.value

    def repulsive_noalloc(self, n, d, h, ng_fixed, y, layout, f):
        """sgt_repulsive_noalloc: the repulsion with no device allocation."""
        z = C.c_double()
        gp = C.c_int()
        he = C.c_float()
        self.check(self.lib.sgt_repulsive_noalloc(self.h, n, d, float(h), int(ng_fixed), _ptr(y),
                                                  layout, _ptr(f), C.byref(z), C.byref(gp),
                                                  C.byref(he)), "repulsive_noalloc")
        return z.value, gp.value, he.value

    def bins(self, n, d, h, ng_fixed, y, layout, out):
        gp = C.c_int()
        self.check(self.lib.sgt_bins(self.h, n, d, float(h), int(ng_fixed), _ptr(y), layout,
                                     _ptr(out), C.byref(gp)), "bins")
        return gp.value

    def last_grids(self, d, N):
        v = np.empty((d + 1,) + (N,) * d, np.float32)
        p = np.empty_like(v)
        self.check(self.lib.sgt_last_grids(self.h, _ptr(v), _ptr(p)), "last_grids")
        return v, p

    def kl(self, n, d, nnz, rowptr, col, val, y, layout, alpha, zeta):
        out = C.c_double()
        self.check(self.lib.sgt_kl(self.h, n, d, nnz, _ptr(rowptr), _ptr(col), _ptr(val), _ptr(y),
                                   layout, float(alpha), float(zeta), C.byref(out)), "kl")
        return out.value

    def lambda_bisect(self, n, rowptr, val, lam, dist=1, sigma=None):
        self.check(self.lib.sgt_lambda_bisect(self.h, n, _ptr(rowptr), _ptr(val), float(lam),
                                              int(dist), _ptr(sigma)), "lambda_bisect")

    def perplexity(self, n, k, dist, perp, p, beta=None):
        self.check(self.lib.sgt_perplexity(self.h, n, k, _ptr(dist), float(perp), _ptr(p),
                                           _ptr(beta)), "perplexity")

    def knn(self, n, dim, X, k, idx, d2, method=None):
        """Exact kNN (squared distances, self excluded) of device X (n*dim)
        into device idx/d2 (n*k).  method: None (sgt_knn) or KNN_AUTO /
        KNN_SIMT / KNN_TENSOR (sgt_knn_ex); with a method, returns the number
        of queries the tensor-core filter handed to the SIMT search."""
        if method is None:
            self.check(self.lib.sgt_knn(self.h, int(n), int(dim), _ptr(X), int(k), _ptr(idx),
                                        _ptr(d2)), "knn")
            return None
        redo = C.c_int()
        self.check(self.lib.sgt_knn_ex(self.h, int(n), int(dim), _ptr(X), int(k), _ptr(idx),
                                       _ptr(d2), int(method), C.byref(redo)), "knn_ex")
        return redo.value

    def csr_to_hybrid(self, n, rowptr, col, val, width, ell_cols, ell_vals, coo_rows,
                      coo_cols, coo_vals):
        """CSR -> ELL + COO on the device; returns the COO tail length."""
        k = C.c_long()
        self.check(self.lib.sgt_csr_to_hybrid_device(
            self.h, int(n), _ptr(rowptr), _ptr(col), _ptr(val), int(width), _ptr(ell_cols),
            _ptr(ell_vals), _ptr(coo_rows), _ptr(coo_cols), _ptr(coo_vals), C.byref(k)),
            "csr_to_hybrid_device")
        return k.value

    def symmetrize(self, n, nnz, rowptr, col, val, scale, out_rowptr, out_col, out_val):
        """(P + P^T) * scale on the device; out_col/out_val hold 2 nnz.
        Returns the output nnz."""
        out = C.c_long()
        self.check(self.lib.sgt_symmetrize_device(self.h, int(n), int(nnz), _ptr(rowptr),
                                                  _ptr(col), _ptr(val), float(scale),
                                                  _ptr(out_rowptr), _ptr(out_col), _ptr(out_val),
                                                  C.byref(out)), "symmetrize_device")
        return out.value

    def csr_to_coo(self, n, nnz, rowptr, rows):
        self.check(self.lib.sgt_csr_to_coo(self.h, n, nnz, _ptr(rowptr), _ptr(rows)), "csr_to_coo")

    # ---- library entry (host numpy arrays) ----
    def embed(self, rowptr, col, val, params: Params, y_in=None, y_out=None, time_info=None):
        """sgt_embed on host arrays.  y_in / y_out: dim-major n*d (y_out, if
        given, must be a C-contiguous float32 array of n*d values, e.g. a
        view of pinned memory); time_info: None (no stage times; the
        captured graphs run) or a float64 array of >= 7003 values.
        Returns (Y point-major (n, d), time_info)."""
        n = len(rowptr) - 1
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.float32)
        yin = None if y_in is None else np.ascontiguousarray(y_in, np.float32)
        if y_out is None:
            y = np.empty(n * params.d, np.float32)
        else:
            y = y_out
            assert y.dtype == np.float32 and y.flags["C_CONTIGUOUS"] and y.size == n * params.d
        ti = time_info  # None: NULL (the captured graphs, no stage times)
        self.check(self.lib.sgt_embed(self.h, n, _ptr(rowptr), _ptr(col), _ptr(val),
                                      C.byref(params), _ptr(yin), _ptr(y), _ptr(ti)), "embed")
        return y.reshape(params.d, n).T.copy(), ti


class Job:
    """Device-resident embedding (sgt_job_*)."""

    def __init__(self, ctx: Context, params: Params, rowptr, col, val, device_mem: bool):
        self.ctx = ctx
        self.lib = ctx.lib
        self.n = (rowptr.numel() if hasattr(rowptr, "numel") else len(rowptr)) - 1
        self.d = params.d
        self.params = params
        h = C.c_void_p()
        ctx.check(self.lib.sgt_job_create(ctx.h, C.byref(params), self.n, _ptr(rowptr), _ptr(col),
                                          _ptr(val), int(device_mem), C.byref(h)), "job_create")
        self.h = h

    def close(self):
        if self.h:
            self.lib.sgt_job_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_y(self, y, layout, device_mem):
        self.ctx.check(self.lib.sgt_job_set_y(self.h, _ptr(y), layout, int(device_mem)), "set_y")

    def run(self, iters):
        self.ctx.check(self.lib.sgt_job_run(self.h, int(iters)), "run")

    def run_timed(self, iters, time_info=None):
        """Iterations stage by stage; per-iteration stage ms in the
        reference's timeInfo layout (time_info[7 i + j], i < 1000)."""
        ti = time_info if time_info is not None else np.zeros(7003, np.float64)
        self.ctx.check(self.lib.sgt_job_run_timed(self.h, int(iters), _ptr(ti)), "run_timed")
        return ti

    def prepare(self):
        """Instantiate the iteration graphs now (sgt_job_prepare)."""
        self.ctx.check(self.lib.sgt_job_prepare(self.h), "prepare")

    def get_y(self, out, layout, device_mem, centre=1):
        self.ctx.check(self.lib.sgt_job_get_y(self.h, _ptr(out), layout, int(device_mem),
                                              int(centre)), "get_y")
        return out

    def info(self) -> JobInfo:
        inf = JobInfo()
        self.ctx.check(self.lib.sgt_job_get_info(self.h, C.byref(inf)), "info")
        return inf

    def kl(self, alpha=-1.0):
        out = C.c_double()
        self.ctx.check(self.lib.sgt_job_kl(self.h, float(alpha), C.byref(out)), "kl")
        return out.value

    def repulsive_error(self):
        out = C.c_double()
        self.ctx.check(self.lib.sgt_job_repulsive_error(self.h, C.byref(out)), "repulsive_error")
        return out.value

    def profile(self, iters):
        ms = np.zeros(8, np.float64)
        self.ctx.check(self.lib.sgt_job_profile(self.h, int(iters), _ptr(ms)), "profile")
        return ms


class Batch:
    """Jobs of one context advanced together through one CUDA graph
    (sgt_batch_*).  The jobs must stay open while the batch is used."""

    def __init__(self, ctx: Context, jobs, iters_per_launch=8):
        self.ctx = ctx
        self.lib = ctx.lib
        self.jobs = list(jobs)
        arr = (C.c_void_p * len(self.jobs))(*[j.h for j in self.jobs])
        h = C.c_void_p()
        ctx.check(self.lib.sgt_batch_create(ctx.h, len(self.jobs), arr, int(iters_per_launch),
                                            C.byref(h)), "batch_create")
        self.h = h

    def run(self, iters):
        self.ctx.check(self.lib.sgt_batch_run(self.h, int(iters)), "batch_run")

    def close(self):
        if self.h:
            self.lib.sgt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_step(ctx: Context, jobs, iters: int):
    """sgt_batch_step: `iters` fused iterations of `jobs` on ctx's stream."""
    arr = (C.c_void_p * len(jobs))(*[j.h for j in jobs])
    ctx.check(ctx.lib.sgt_batch_step(ctx.h, len(jobs), arr, int(iters)), "batch_step")


def job_footprint(params: Params, n: int, nnz: int) -> int:
    return int(load().sgt_job_footprint(C.byref(params), int(n), int(nnz)))


class Server:
    """Continuous-batching request server (sgt_server_*).  Host numpy
    buffers of a request are kept referenced here until it finishes."""

    def __init__(self, device=0, hbm_budget=None, max_active=None, iters_per_round=None,
                 rounds_ahead=None):
        self.lib = load()
        cfg = ServerConfig()
        self.lib.sgt_server_config_default(C.byref(cfg))
        if hbm_budget is not None:
            cfg.hbm_budget = int(hbm_budget)
        if max_active is not None:
            cfg.max_active = int(max_active)
        if iters_per_round is not None:
            cfg.iters_per_round = int(iters_per_round)
        if rounds_ahead is not None:
            cfg.rounds_ahead = int(rounds_ahead)
        self.cfg = cfg
        h = C.c_void_p()
        st = self.lib.sgt_server_create(int(device), C.byref(cfg), C.byref(h))
        if st != 0:
            raise SgtError(st, "server_create")
        self.h = h
        self._keep = {}

    def submit(self, params: Params, rowptr, col, val, y0):
        """Returns (request id, output array filled when the request is done)."""
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.float32)
        y0 = np.ascontiguousarray(y0, np.float32)
        n = len(rowptr) - 1
        out = np.empty((n, params.d), np.float32)
        rid = C.c_longlong()
        st = self.lib.sgt_server_submit(self.h, C.byref(params), n, _ptr(rowptr), _ptr(col),
                                        _ptr(val), _ptr(y0), _ptr(out), C.byref(rid))
        if st != 0:
            raise SgtError(st, "server_submit")
        self._keep[rid.value] = (rowptr, col, val, y0, out)
        return rid.value, out

    def poll(self, wait_ms=0.0, cap=256):
        ids = (C.c_longlong * cap)()
        cnt = C.c_int()
        st = self.lib.sgt_server_poll(self.h, float(wait_ms), ids, cap, C.byref(cnt))
        if st != 0:
            raise SgtError(st, "server_poll")
        done = [ids[k] for k in range(cnt.value)]
        for r in done:
            self._keep.pop(r, None)
        return done

    def info(self, rid) -> RequestInfo:
        inf = RequestInfo()
        st = self.lib.sgt_server_request_info(self.h, int(rid), C.byref(inf))
        if st != 0:
            raise SgtError(st, "server_request_info")
        return inf

    def now(self):
        return self.lib.sgt_server_now(self.h)

    def close(self):
        if self.h:
            self.lib.sgt_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- host-side helpers (no device) ----
def best_grid_size(ng: int) -> int:
    return load().sgt_best_grid_size(int(ng))


def ell_width(rowptr) -> int:
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    return load().sgt_ell_width(len(rowptr) - 1, _ptr(rowptr))


def csr_to_hybrid(rowptr, col, val, width):
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    n = len(rowptr) - 1
    nnz = int(rowptr[-1])
    ec = np.empty(max(n * width, 1), np.uint32)
    ev = np.empty(max(n * width, 1), np.float32)
    cr = np.empty(max(nnz, 1), np.uint32)
    cc = np.empty(max(nnz, 1), np.uint32)
    cv = np.empty(max(nnz, 1), np.float32)
    k = C.c_long()
    st = load().sgt_csr_to_hybrid(n, _ptr(rowptr), _ptr(col), _ptr(val), int(width), _ptr(ec),
                                  _ptr(ev), _ptr(cr), _ptr(cc), _ptr(cv), C.byref(k))
    if st != 0:
        raise SgtError(st, "csr_to_hybrid")
    k = k.value
    return ec[:n * width], ev[:n * width], cr[:k].copy(), cc[:k].copy(), cv[:k].copy()


def symmetrize(rowptr, col, val, scale):
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    n = len(rowptr) - 1
    L = load()
    nnz = C.c_long()
    st = L.sgt_symmetrize(n, _ptr(rowptr), _ptr(col), _ptr(val), float(scale), None, None, None,
                          C.byref(nnz))
    if st != 0:
        raise SgtError(st, "symmetrize")
    orp = np.empty(n + 1, np.int32)
    oc = np.empty(nnz.value, np.int32)
    ov = np.empty(nnz.value, np.float32)
    st = L.sgt_symmetrize(n, _ptr(rowptr), _ptr(col), _ptr(val), float(scale), _ptr(orp), _ptr(oc),
                          _ptr(ov), C.byref(nnz))
    if st != 0:
        raise SgtError(st, "symmetrize")
    return orp, oc, ov
