"""Failure paths, made to happen on purpose without faulting the GPU.

* Learned preconditioner fallback: the network's weights are corrupted on the
  host (set to NaN), so the factor G it builds is useless. The learned solve
  (clsparseDcsrcgLearned) must notice the broken inner solve, drop its
  correction, continue with Jacobi, report fellBack = 1 and still reach the
  FP64 residual. This is the stop rule of the reference's solver control
  (src/library/solvers/solver-control.hpp:47-64) extended by the learned
  method's stall test.
* Bounded barrier waits of the persistent solver (loop mode 2): with a test
  switch the first grid barrier is never released and the wait limit is
  2 ms, so every CTA's wait runs out. The solve must return
  clsparseInvalidKernelExecution with device status bit 32 (barrier
  timeout), and the same control must then solve the system correctly: the
  context is intact and no state is left behind.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, matgen

pytestmark = pytest.mark.gpu


def true_residual(rp, col, val, x, b):
    n = len(rp) - 1
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    return np.linalg.norm(b - A @ x) / np.linalg.norm(b)


@pytest.mark.parametrize("inner", ["fp32", "bf16"])
def test_learned_solve_falls_back_to_jacobi_on_corrupted_network(ctrl, inner):
    rp, col, val = matgen.diffusion2d_grf(48, corr_len=0.1, sigma=1.0, seed=21)
    n = len(rp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    spai = api.Spai(3)
    p = spai.params()
    spai.set_params(np.full_like(p, np.nan))
    spai.set_matrix(A, ctrl)
    spai.build(ctrl)
    _, _, G = spai.factor()
    assert not np.isfinite(G).any()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 50000, 1e-10, 0.0)
    info = api.cg_learned(x, A, torch.tensor(b, device="cuda"), sc, spai, ctrl, inner=inner, inner_tol=0.3)
    sc.release()
    spai.release()
    assert info["fell_back"] == 1, info
    assert info["converged"] == 1, info
    xs = x.cpu().numpy()
    assert np.isfinite(xs).all()
    assert true_residual(rp, col, val, xs, b) <= 1.5e-10
    # the broken inner solve stopped at once instead of spending the budget
    xj = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 50000, 1e-10, 0.0)
    ji = api.cg_mixed(xj, A, torch.tensor(b, device="cuda"), sc, ctrl, inner=inner, inner_tol=0.3)
    sc.release()
    assert info["innerIterations"] <= ji["innerIterations"] + 5, (info, ji)


def test_persistent_solver_barrier_timeout_is_reported_and_recovers(ctrl, orc, monkeypatch):
    rp, col, val = matgen.diffusion3d_lognormal(20, sigma=1.0, seed=9)
    n = len(rp) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    ctrl.set_solver_loop_mode(2)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    bt = torch.tensor(b, device="cuda")

    monkeypatch.setenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE", "1")
    monkeypatch.setenv("CLSPARSE_B200_BARRIER_WAIT_NS", "2000000")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 2000, 1e-10, 0.0)
    with pytest.raises(api.ClsparseError) as e:
        api.solve("cg", x, A, bt, sc, ctrl)
    assert e.value.status == L.clsparseInvalidKernelExecution
    assert sc.device_status() & 32
    sc.release()
    torch.cuda.synchronize()  # the context is still usable

    monkeypatch.delenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")
    monkeypatch.delenv("CLSPARSE_B200_BARRIER_WAIT_NS")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 2000, 1e-10, 0.0)
    info = api.solve("cg", x, A, bt, sc, ctrl)
    assert not (sc.device_status() & 32)
    sc.release()
    _, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, L.DIAGONAL, 2000, 1e-10, 0.0)
    assert abs(info["nIters"] - oi.nIters) <= max(3, int(0.03 * oi.nIters))
    l1 = np.abs(b - sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))) @ x.cpu().numpy()).sum()
    assert l1 / np.abs(b).sum() <= 1e-9
