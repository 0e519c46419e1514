"""One embedding split by rows over the ranks of a torch.distributed process
group, one GPU per rank (sgt_shard_* of include/sgtsne_b200.h).

Rank r of R holds the stretch of rows [r c, min((r + 1) c, n)), c =
ceil(n / R): P's rows of those points (global column indices) and the
points' momentum, gains and forces.  Every rank keeps all n coordinates.
One iteration, in the same order on every rank:

  scatter          grid decision from all coordinates, S2G of the own
                   points into the charge grid, the own rows' attractive
                   SpMV (on a side stream)
  all-reduce grid  the sum of the ranks' charge grids
  gather           G2G of the summed grid, G2S of the own points, their Z
  all-reduce Z     the sum over ranks
  update           forces, gains, momentum and coordinates of the own rows
  all-gather Y     every rank's own rows into every rank's coordinates

The grid, Z and the exaggeration/momentum schedule are global, so every
rank runs the iteration of the whole embedding.  ShardedEmbedding drives any
backend with this phase interface: EngineShard (the C ABI on one GPU per
rank, NCCL between them), or a CPU restatement in the tests (gloo).
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def stretch(n: int, world: int, rank: int):
    """Rows [lo, hi) of `rank` and the common stretch length c (the last
    rank's stretch may be shorter; buffers hold world * c rows)."""
    c = -(-n // world)
    lo = min(rank * c, n)
    hi = min(lo + c, n)
    return lo, hi, c


def local_rows(rowptr, col, val, lo, hi):
    """P's rows [lo, hi) as a CSR of their own (rowptr from 0, global
    column indices)."""
    rowptr = np.asarray(rowptr)
    a, b = int(rowptr[lo]), int(rowptr[hi])
    rp = (rowptr[lo:hi + 1] - rowptr[lo]).astype(np.int32)
    return rp, np.ascontiguousarray(col[a:b], np.int32), np.ascontiguousarray(val[a:b], np.float32)


class ShardedEmbedding:
    """Runs iterations of one embedding split over the ranks of `group`
    (None: the default group).  `backend` holds the rank's shard: its
    buffers `grid`, `zsum`, `y_all` (world * c rows) and `y_own` (this
    rank's c rows of y_all) are torch tensors, and scatter(), gather(),
    update() queue the phases."""

    def __init__(self, backend, group=None):
        import torch.distributed as dist
        self.b = backend
        self.group = group
        self.dist = dist
        self.world = dist.get_world_size(group)
        self._into_tensor = dist.get_backend(group) == "nccl"

    def step(self):
        b, dist, g = self.b, self.dist, self.group
        b.scatter()
        dist.all_reduce(b.grid, op=dist.ReduceOp.SUM, group=g)
        b.gather()
        dist.all_reduce(b.zsum, op=dist.ReduceOp.SUM, group=g)
        b.update()
        if self._into_tensor:
            dist.all_gather_into_tensor(b.y_all, b.y_own, group=g)
        else:
            dist.all_gather(list(b.y_all.chunk(self.world)), b.y_own.clone(), group=g)

    def run(self, iters: int):
        for _ in range(int(iters)):
            self.step()


class EngineShard:
    """This rank's shard through the C ABI (sgt_shard_*): rows [lo, hi) of
    the global CSR P on `device`, the buffers the collectives exchange as
    torch CUDA tensors.  The context's stream must be torch's current
    stream (Context.set_stream), so that the collectives torch queues are
    ordered with the phases."""

    def __init__(self, ctx, params, n, rank, world, rowptr, col, val, device):
        import torch

        from . import SgtError, _ptr
        self.ctx, self.lib, self.n, self.d = ctx, ctx.lib, int(n), int(params.d)
        self.lo, self.hi, self.c = stretch(self.n, world, rank)
        if self.hi - self.lo < 1:
            raise SgtError(1, "every rank needs at least one row (n >= world)")
        S = 4 if self.d == 3 else self.d
        self.S = S
        self.y_all = torch.zeros(world * self.c * S, dtype=torch.float32, device=device)
        self.y_own = self.y_all[rank * self.c * S:(rank + 1) * self.c * S]
        gf = int(self.lib.sgt_shard_grid_floats(C.byref(params)))
        self.grid = torch.zeros(gf, dtype=torch.float32, device=device)
        self.zsum = torch.zeros(1, dtype=torch.float64, device=device)
        rp, cl, vl = local_rows(rowptr, col, val, self.lo, self.hi)
        self._host = (rp, cl, vl)
        torch.cuda.synchronize(device)  # the buffers above exist before the engine uses them
        h = C.c_void_p()
        ctx.check(self.lib.sgt_shard_create(ctx.h, C.byref(params), self.n, self.lo,
                                            self.hi - self.lo, _ptr(rp), _ptr(cl), _ptr(vl), 0,
                                            _ptr(self.y_all), _ptr(self.grid), gf,
                                            _ptr(self.zsum), C.byref(h)), "shard_create")
        self.h = h

    def set_y(self, Y):
        """All n points' coordinates (host array n x d, point-major)."""
        from . import LAYOUT_POINT_MAJOR, _ptr
        Y = np.ascontiguousarray(Y, np.float32)
        self.ctx.check(self.lib.sgt_shard_set_y(self.h, _ptr(Y), LAYOUT_POINT_MAJOR, 0), "set_y")

    def scatter(self):
        self.ctx.check(self.lib.sgt_shard_scatter(self.h), "shard_scatter")

    def gather(self):
        self.ctx.check(self.lib.sgt_shard_gather(self.h), "shard_gather")

    def update(self):
        self.ctx.check(self.lib.sgt_shard_update(self.h), "shard_update")

    def get_y(self, centre=1):
        """All n coordinates (host, n x d), centred by default."""
        from . import LAYOUT_POINT_MAJOR, _ptr
        out = np.empty((self.n, self.d), np.float32)
        self.ctx.check(self.lib.sgt_shard_get_y(self.h, _ptr(out), LAYOUT_POINT_MAJOR, 0,
                                                int(centre)), "shard_get_y")
        return out

    def info(self):
        from . import JobInfo
        inf = JobInfo()
        self.ctx.check(self.lib.sgt_shard_get_info(self.h, C.byref(inf)), "shard_info")
        return inf

    def close(self):
        if self.h:
            self.lib.sgt_shard_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
