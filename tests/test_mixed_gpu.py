"""Mixed-precision refinement (clsparseDcsrcgMixed) through the C ABI.

Bar: the FP64 true residual ||b - A x||_2 / ||b||_2 (recomputed here on the
host in FP64) meets the requested 1e-10, and the solution agrees with the
FP64 CG oracle's to the accuracy the conditioning allows."""
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
@pytest.mark.parametrize("sigma", [0.5, 1.5])
def test_mixed_refinement_reaches_fp64_residual(ctrl, orc, inner, sigma):
    rp, col, val = matgen.diffusion3d_lognormal(24, sigma=sigma, seed=4)
    n = len(rp) - 1
    b = np.random.default_rng(0).uniform(-1, 1, n)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 20000, 1e-10, 0.0)
    info = api.cg_mixed(x, A, torch.tensor(b, device="cuda"), sc, ctrl, inner=inner, inner_tol=1e-3)
    sc.release()
    xs = x.cpu().numpy()
    res = true_residual(rp, col, val, xs, b)
    # BF16 included: the banded inner copy keeps A's row sums (its FP32
    # diagonal carries each row's rounding), so even the sigma = 1.5
    # high-contrast operator stays SPD and the refinement contracts.
    assert info["converged"] == 1, info
    assert res <= 1.5e-10, (res, info)
    assert abs(info["trueResidual"] - res) <= 1e-11 + 1e-3 * res
    xo, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 20000, 1e-13, 0.0)
    err = np.linalg.norm(xs - xo) / np.linalg.norm(xo)
    assert err <= 1e-6, err


def test_mixed_zero_rhs(ctrl):
    rp, col, val = matgen.poisson2d(16)
    n = len(rp) - 1
    A = api.CsrMatrix.from_numpy(rp, col, val)
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 100, 1e-10, 0.0)
    info = api.cg_mixed(x, A, torch.zeros(n, dtype=torch.float64, device="cuda"), sc, ctrl)
    sc.release()
    assert info["converged"] == 1 and float(x.abs().sum()) == 0.0


def test_l2_norm_option_matches_oracle_residual(ctrl):
    rp, col, val = matgen.poisson2d(64)
    n = len(rp) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 5000, 1e-10, 0.0)
    sc.set_norm(2)
    info = api.solve("cg", x, A, torch.tensor(b, device="cuda"), sc, ctrl)
    sc.release()
    assert info["currentResidual"] <= 1e-10
    assert true_residual(rp, col, val, x.cpu().numpy(), b) <= 2e-10


def convection_diffusion(m, peclet=0.4):
    """2D 5-point diffusion plus first-order upwind convection in x: a
    nonsymmetric, diagonally dominant operator (a BiCGStab case)."""
    rp, col, val = matgen.poisson2d(m)
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)))
    n = m * m
    i = np.arange(n)
    west = (i % m) != 0
    C = sp.csr_matrix((np.full(west.sum(), -peclet), (i[west], i[west] - 1)), shape=(n, n)) + \
        sp.diags(np.where(west, peclet, 0.0))
    M = (A + C).tocsr()
    M.sort_indices()
    return M.indptr.astype(np.uint32), M.indices.astype(np.uint32), M.data


@pytest.mark.parametrize("inner", ["fp32", "bf16"])
def test_mixed_bicgstab_reaches_fp64_residual(ctrl, inner):
    rp, col, val = convection_diffusion(40)
    n = len(rp) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 20000, 1e-10, 0.0)
    info = api.bicgstab_mixed(x, A, torch.tensor(b, device="cuda"), sc, ctrl, inner=inner, inner_tol=1e-3)
    sc.release()
    res = true_residual(rp, col, val, x.cpu().numpy(), b)
    assert info["converged"] == 1, info
    assert res <= 1.5e-10, (res, info)
    import scipy.sparse.linalg as spla
    xd = spla.spsolve(sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))).tocsc(), b)
    assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) <= 1e-8
