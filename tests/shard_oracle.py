"""The phases of one row-split shard restated on the CPU in FP64 with the
oracle's stage functions (test infrastructure: the backend the gloo tests
drive through sgtsne_b200.sharded.ShardedEmbedding).

It follows the oracle's iteration (HYB/qq.cpp:25-244, HYB/nuconv.cpp:22-153,
HYB/gradient_descendHYB.cpp:29-78) with the sums split by rows:
  scatter  centre all coordinates (every rank alike), min shift and grid
           size from all of them, S2G of the own points' charges [1, y],
           the own rows' attractive term
  gather   G2G of the summed grid, G2S of the own points,
           Z_own = sum_own (1 + 2|y|^2) Phi0 - 2 y.Phi, minus the own count
  update   F_rep = (y Phi0 - Phi_{1..d}) / Z, dY = alpha F_attr - F_rep,
           gains / momentum / coordinates of the own rows
"""
import numpy as np
import torch

from oracle import oracle as O
from sgtsne_b200.sharded import stretch


class OracleShard:
    def __init__(self, rowptr, col, val, n, d, rank, world, h=0.7, early_iter=250,
                 alpha=12.0):
        self.n, self.d, self.h = n, d, h
        self.lo, self.hi, self.c = stretch(n, world, rank)
        self.rp = np.asarray(rowptr, np.int64)
        self.col = np.asarray(col, np.int64)
        self.val = np.asarray(val, np.float64)
        self.early_iter, self.alpha0 = early_iter, alpha
        self.y_all = torch.zeros(world * self.c * d, dtype=torch.float64)
        self.y_own = self.y_all[rank * self.c * d:(rank + 1) * self.c * d]
        self.grid = torch.zeros(1, dtype=torch.float64)
        self.zsum = torch.zeros(1, dtype=torch.float64)
        m = self.hi - self.lo
        self.uY = np.zeros((m, d))
        self.gains = np.ones((m, d))
        self.iter = 0

    def set_y(self, Y):
        self.y_all[:self.n * self.d] = torch.as_tensor(np.asarray(Y, np.float64).reshape(-1))
        self.uY[:] = 0
        self.gains[:] = 1
        self.iter = 0

    def Y(self):
        return self.y_all[:self.n * self.d].numpy().reshape(self.n, self.d)

    def scatter(self):
        Y = self.Y()
        Y -= Y.mean(0)  # in place: every rank centres its identical copy
        miny = Y.min(0)
        ysh = Y - miny
        maxy = ysh.max()
        n1 = O.best_grid_size(max(int(np.ceil(maxy / self.h)), 14))
        self.N = n1 + 2
        own = ysh[self.lo:self.hi]
        v = own / maxy
        v[v == 1] -= np.finfo(np.float64).eps
        self.ys = v * (n1 - 1)
        self.he = maxy / ((n1 - 1) - np.finfo(np.float64).eps)
        self.own_sh = own
        q = np.concatenate([np.ones((len(own), 1)), own], 1)
        self.grid = torch.as_tensor(O.s2g(self.ys, q, self.N).reshape(-1).copy())
        # attractive term of the own rows: sum_j p_ij (y_i - y_j)/(1 + |y_i - y_j|^2)
        a, b = self.rp[self.lo], self.rp[self.hi]
        rows = np.repeat(np.arange(self.lo, self.hi), np.diff(self.rp[self.lo:self.hi + 1]))
        dif = Y[rows] - Y[self.col[a:b]]
        w = self.val[a:b] / (1.0 + (dif * dif).sum(1))
        self.fattr = np.zeros((self.hi - self.lo, self.d))
        for k in range(self.d):
            self.fattr[:, k] = np.bincount(rows - self.lo, weights=w * dif[:, k],
                                           minlength=self.hi - self.lo)

    def gather(self):
        m = self.d + 1
        V = self.grid.numpy().reshape((m,) + (self.N,) * self.d)
        Phi = O.g2g(V, self.he)
        self.phi = O.g2s(self.ys, Phi)
        y = self.own_sh
        z = ((1 + 2 * (y * y).sum(1)) * self.phi[:, 0]).sum() - 2 * (y * self.phi[:, 1:]).sum()
        self.zsum = torch.tensor([z - (self.hi - self.lo)], dtype=torch.float64)

    def update(self):
        Z = float(self.zsum[0])
        y = self.own_sh
        frep = (y * self.phi[:, :1] - self.phi[:, 1:]) / Z
        alpha = self.alpha0 if self.iter <= self.early_iter else 1.0
        mom = 0.5 if self.iter <= 250 else 0.8
        dY = alpha * self.fattr - frep
        g = np.where(np.sign(dY) != np.sign(self.uY), self.gains + 0.2, self.gains * 0.8)
        self.gains = np.maximum(g, 0.01)
        self.uY = mom * self.uY - 200.0 * self.gains * dY
        Y = self.Y()
        Y[self.lo:self.hi] += self.uY
        self.iter += 1
