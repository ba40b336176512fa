"""CPU stand-in for one rank's kernels of the row-partitioned CG
(csrc/dist_cg.cu), for the multi-process tests without a GPU: the same stages
with the same arithmetic (FP64, scipy SpMV in place of the CSR kernel), on
CPU tensors that gloo can exchange. It mirrors DeviceRank's interface so that
clsparse_b200.distributed.dist_cg drives it unchanged."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from clsparse_b200 import distributed as D


class HostSolverControl:
    def __init__(self, precond, max_iters, rel_tol, abs_tol):
        self.precond, self.max_iters, self.rel, self.abs = precond, int(max_iters), rel_tol, abs_tol
        self.nIters, self.init, self.cur = 0, 0.0, 0.0

    def info(self):
        return {"nIters": self.nIters, "initialResidual": self.init, "currentResidual": self.cur}


class HostRank:
    def __init__(self, plan: D.Plan, rp, col_ext, val, precond: int):
        self.plan = plan
        n = len(rp) - 1
        self.n = n
        self.A = sp.csr_matrix((np.asarray(val, np.float64), np.asarray(col_ext, np.int64),
                                np.asarray(rp, np.int64)), shape=(n, plan.ext_len))
        self.invd = None
        if precond == 1:
            own = plan.own
            d = np.array([self.A[i, own + i] for i in range(n)], dtype=np.float64)
            if np.any(d == 0.0):
                raise ValueError("missing or zero diagonal")
            self.invd = 1.0 / d
        self.xext = torch.zeros(plan.ext_len, dtype=torch.float64)
        self.zext = torch.zeros(plan.ext_len, dtype=torch.float64)
        self.sums = torch.zeros(4, dtype=torch.float64)
        self.r = np.zeros(n)
        self.p = np.zeros(n)
        self.s = np.zeros(n)
        self.w = np.zeros(n)
        self.st = {}

    def ext(self, which):
        return self.xext if which == "x" else self.zext

    def send_view(self, which, q):
        idx = self.plan.send[q]
        return self.ext(which)[self.plan.own + torch.as_tensor(idx)].clone()

    def _own(self, v):
        return v.numpy()[self.plan.own: self.plan.own + self.n]

    def start(self, x, b):
        self.x, self.b = x, b
        self.st = {"done": False}
        self.sums.zero_()
        self._own(self.xext)[:] = x.numpy()

    def residual(self):
        b = self.b.numpy()
        r = b - self.A @ self.xext.numpy()
        z = r * self.invd if self.invd is not None else r.copy()
        self.r[:] = r
        self._own(self.zext)[:] = z
        self._part = [float(r @ z), float(np.abs(r).sum()), float(np.abs(b).sum())]

    def product(self):
        if self.st["done"]:
            self.sums.zero_()
            return
        w = self.A @ self.zext.numpy()
        self.w[:] = w
        rz, nr, nb = self._part
        self.sums[:] = torch.tensor([rz, float(w @ self._own(self.zext)), nr, nb], dtype=torch.float64)

    def update(self, j, sc):
        st = self.st
        if st["done"]:
            return
        g, d, nr, nb_red = (float(v) for v in self.sums)
        nb = nb_red if j == 0 else st["nb"]
        if j == 0 and nb == 0.0:
            self.x.numpy()[:] = self.b.numpy()
            st.update(done=True, iters=0, init=0.0, cur=0.0)
            return
        res = nr / nb
        init = res if j == 0 else st["init"]
        n_iters = 0 if j == 0 else j - 1
        if j == 0:
            st["nb"], st["init"] = nb, res
        st["cur"] = res
        if res <= sc.rel or res <= sc.abs * init or n_iters >= sc.max_iters:
            st.update(done=True, iters=n_iters)
            return
        if j == 0:
            beta, alpha = 0.0, g / d
        else:
            beta = g / st["gamma"]
            alpha = g / (d - beta * g / st["alpha"])
        st["gamma"], st["alpha"] = g, alpha
        z = self._own(self.zext)
        if j == 0:
            self.p[:] = z
            self.s[:] = self.w
        else:
            self.p[:] = z + beta * self.p
            self.s[:] = self.w + beta * self.s
        x = self.x.numpy()
        x += alpha * self.p
        self.r -= alpha * self.s
        zn = self.r * self.invd if self.invd is not None else self.r.copy()
        z[:] = zn
        self._part = [float(self.r @ zn), float(np.abs(self.r).sum()), self._part[2]]

    def state(self, sc):
        st = self.st
        if st["done"]:
            sc.nIters, sc.init, sc.cur = st["iters"], st["init"], st["cur"]
        return st["done"], sc.info()


class HostNet:
    """CPU stand-in for a rank's network in data-parallel training: FP32
    parameters, a least-squares loss per sample 0.5 ||M_s p - c_s||^2 with
    its gradient in a CPU tensor (what gloo reduces), and the Adam step of
    the device kernel (beta 0.9 / 0.999, eps 1e-8, bias-corrected)."""

    def __init__(self, nparams: int, seed: int = 1):
        self.p = np.random.default_rng(seed).normal(0, 0.1, nparams).astype(np.float32)
        self.m = np.zeros_like(self.p)
        self.v = np.zeros_like(self.p)
        self.step = 0
        self.g = torch.zeros(nparams, dtype=torch.float32)

    def loss_grad(self, sample):
        M, c = sample
        res = M @ self.p - c
        self.g.copy_(torch.from_numpy((M.T @ res).astype(np.float32)))
        return float(0.5 * res @ res)

    def grad(self):
        return self.g

    def adam_step(self, lr, scale):
        g = self.g.numpy() * np.float32(scale)
        self.step += 1
        b1, b2 = np.float32(0.9), np.float32(0.999)
        c1 = np.float32(1.0) - b1 ** self.step
        c2 = np.float32(1.0) - b2 ** self.step
        self.m = b1 * self.m + (1 - b1) * g
        self.v = b2 * self.v + (1 - b2) * g * g
        self.p = self.p - np.float32(lr) * (self.m / c1) / (np.sqrt(self.v / c2) + np.float32(1e-8))


def toy_samples(k: int = 6, nparams: int = 40, seed: int = 3):
    rng = np.random.default_rng(seed)
    return [(rng.normal(0, 1, (60, nparams)).astype(np.float32), rng.normal(0, 1, 60).astype(np.float32))
            for _ in range(k)]
