"""Training and evaluation of the learned factorized preconditioner
(clsparseB200Spai*) on matrices of the variable-coefficient diffusion family.

The training data are produced by the library itself: matrices from the
generator and, for each, residual histories of its own Jacobi-CG (FP64, L2
stop test) sampled at several iteration counts. Residuals are scaled into the
network's space (r_hat = D^-1/2 r) and normalised; they enter the loss as
probes. Every kernel of the loop (forward, loss, backward, Adam) is the
library's.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from . import api, matgen


def residual_history(ctrl: api.Control, A: api.CsrMatrix, b: torch.Tensor, checkpoints=(5, 20, 60, 150)):
    """Residuals r_k of Jacobi-CG after k iterations, from x0 = 0: one solve
    whose update kernel keeps r at the checkpoints (device-resident
    snapshots, no host reads during the solve)."""
    n = A.num_rows
    snaps = torch.zeros(len(checkpoints), n, dtype=torch.float64, device=b.device)
    x = torch.zeros(n, dtype=torch.float64, device=b.device)
    # the solve runs max(checkpoints) iterations: no tolerance stops it earlier
    sc = api.SolverControl(L.DIAGONAL, max(checkpoints) - 1, 0.0, 0.0)
    sc.set_norm(2)
    sc.set_snapshots(list(checkpoints), snaps)
    api.solve("cg", x, A, b, sc, ctrl)
    sc.release()
    return [snaps[k] for k in range(len(checkpoints))]


def probes_for(A_np, history):
    """Scaled, normalised probe vectors (FP32, stacked) from residuals."""
    rp, col, val = A_np
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp.astype(np.int64)))
    diag = val[col.astype(np.int64) == rows]
    dinv = torch.tensor(1.0 / np.sqrt(diag), device=history[0].device)
    ps = []
    for r in history:
        v = r * dinv
        nrm = torch.linalg.norm(v)
        if nrm > 0:
            ps.append((v / nrm).float())
    return torch.stack(ps)


class Sample:
    def __init__(self, ctrl, m, seed, corr=0.05, sigma=2.0, with_probes=True):
        self.np = matgen.diffusion2d_grf(m, corr_len=corr, sigma=sigma, seed=seed)
        self.A = api.CsrMatrix.from_numpy(*self.np)
        self.A.create_meta(ctrl)
        n = self.A.num_rows
        self.b = torch.tensor(np.random.default_rng(seed + 1000).uniform(-1, 1, n), device="cuda")
        self.probes = probes_for(self.np, residual_history(ctrl, self.A, self.b)) if with_probes else None


def train(ctrl: api.Control, sizes=(64, 128), seeds=range(8), steps=400, lr=2e-3, lam=0.2, net_seed=1234,
          log=None):
    """Trains a fresh network; returns (spai, loss history)."""
    spai = api.Spai(net_seed)
    samples = [Sample(ctrl, m, s) for m in sizes for s in seeds]
    hist = []
    for it in range(steps):
        smp = samples[it % len(samples)]
        spai.set_matrix(smp.A, ctrl)
        lr_t = lr * (0.1 ** (it / max(steps, 1)))
        loss = spai.train_step(ctrl, smp.probes, lam, lr_t)
        hist.append(loss)
        if log and it % 50 == 0:
            log(f"step {it} loss {loss:.5f}")
    return spai, hist


def pcg_iterations(ctrl, spai, smp: Sample, tol=1e-10, max_iters=200000):
    """(learned-PCG iterations, Jacobi-CG iterations) to an FP64 L2 tolerance."""
    spai.set_matrix(smp.A, ctrl)
    spai.build(ctrl)
    n = smp.A.num_rows
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, max_iters, tol, 0.0)
    info = api.cg_learned(x, smp.A, smp.b, sc, spai, ctrl, inner="fp64")
    sc.release()
    x2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, max_iters, tol, 0.0)
    sc.set_norm(2)
    j = api.solve("cg", x2, smp.A, smp.b, sc, ctrl)
    sc.release()
    return info["innerIterations"], j["nIters"] + 1
