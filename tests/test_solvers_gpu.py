"""CG / BiCGStab through the C ABI against the oracle restatement of the
reference solvers (src/library/solvers/conjugate-gradients.hpp,
biconjugate-gradients-stabilized.hpp).

Parity bar: the same stop decision (iteration counts within a small slack --
the GPU sums reductions in a different order), the reported residuals agree,
and the returned x meets the stop criterion on a fresh FP64 check."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, matgen

pytestmark = pytest.mark.gpu

NP = {torch.float64: np.float64, torch.float32: np.float32}


def run(ctrl, kind, rp, col, val, x0, b, dtype, precond, max_iters, rel, abs_, meta=True, loop_mode=0):
    ctrl.set_solver_loop_mode(loop_mode)
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=dtype)
    if meta:
        A.create_meta(ctrl)
    x = torch.tensor(np.asarray(x0), dtype=dtype, device="cuda")
    bt = torch.tensor(np.asarray(b), dtype=dtype, device="cuda")
    sc = api.SolverControl(precond, max_iters, rel, abs_)
    info = api.solve(kind, x, A, bt, sc, ctrl)
    status = sc.device_status()
    sc.release()
    return x.cpu().numpy().astype(np.float64), info, status


def l1_residual(rp, col, val, x, b):
    import scipy.sparse as sp
    n = len(rp) - 1
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    return np.abs(b - A @ x).sum() / np.abs(b).sum()


PROBLEMS = {
    "poisson64": lambda: matgen.poisson2d(64),
    "diffusion3d": lambda: matgen.diffusion3d_lognormal(16, sigma=1.0, seed=2),
    "random_spd": lambda: matgen.random_spd(5000, seed=3),
}


@pytest.mark.parametrize("loop_mode", [0, 2], ids=["graph", "persistent"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("precond", [L.DIAGONAL, L.NOPRECOND], ids=["jacobi", "none"])
@pytest.mark.parametrize("prob", sorted(PROBLEMS))
@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_solver_parity(ctrl, orc, kind, prob, precond, dtype, loop_mode):
    rp, col, val = PROBLEMS[prob]()
    n = len(rp) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    t = NP[dtype]
    x, info, _ = run(ctrl, kind, rp, col, val, np.zeros(n), b, dtype, precond, 5000, rel, 0.0, loop_mode=loop_mode)
    xo, oi = orc.solve(kind, t, rp, col, val, np.zeros(n, t), np.asarray(b, t), precond, 5000, rel, 0.0)
    # BiCGStab's convergence history is irregular and reacts to the order of
    # the reduction sums; CG's is smooth.
    slack = max(3, int(0.03 * oi.nIters)) if kind == "cg" else max(8, int(0.12 * oi.nIters))
    assert abs(info["nIters"] - oi.nIters) <= slack, (info, oi.nIters)
    assert info["initialResidual"] == pytest.approx(oi.initialResidual, rel=1e-5)
    assert info["currentResidual"] <= rel
    r_true = l1_residual(rp, col, np.asarray(val, t).astype(np.float64), x, np.asarray(b, t).astype(np.float64))
    assert r_true <= (10 * rel if dtype == torch.float64 else 50 * rel)


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_solver_loop_modes_agree(ctrl, kind):
    rp, col, val = matgen.poisson2d(48)
    n = len(rp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    x0, i0, _ = run(ctrl, kind, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 3000, 1e-9, 0.0,
                    loop_mode=0)
    x1, i1, _ = run(ctrl, kind, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 3000, 1e-9, 0.0,
                    loop_mode=1)
    assert i0 == i1
    assert np.array_equal(x0, x1)


@pytest.mark.parametrize("ext", [False, True], ids=["plain", "extended"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_persistent_cg_matches_graph_form(ctrl, dtype, ext):
    """Loop mode 2 (one cooperative launch per solve) against the graph form:
    same stop decision up to reduction order, same answer to the tolerance."""
    rp, col, val = matgen.diffusion3d_lognormal(24, sigma=1.0, seed=4)
    n = len(rp) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    ctrl.enable_extended_precision(ext)
    try:
        xg, ig, _ = run(ctrl, "cg", rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 5000, rel, 0.0, loop_mode=0)
        xp, ip, _ = run(ctrl, "cg", rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 5000, rel, 0.0, loop_mode=2)
    finally:
        ctrl.enable_extended_precision(False)
    assert abs(ip["nIters"] - ig["nIters"]) <= max(2, int(0.02 * ig["nIters"]))
    assert ip["initialResidual"] == pytest.approx(ig["initialResidual"], rel=1e-6)
    assert ip["currentResidual"] <= rel
    tol = 1e-7 if dtype == torch.float64 else 1e-2
    assert np.linalg.norm(xp - xg) <= tol * np.linalg.norm(xg)


def test_persistent_cg_long_rows(ctrl, orc):
    """An SPD arrow matrix whose first row and column are dense (the row
    becomes LONG row-block words): the persistent solver's long-row merge."""
    n = 40000
    rng = np.random.default_rng(8)
    import scipy.sparse as sp
    off = sp.random(n, n, density=3.0 / n, random_state=3, format="csr")
    arrow = sp.lil_matrix((n, n))
    arrow[0, 1:] = rng.uniform(-1, 1, n - 1) * 1e-3
    arrow = arrow.tocsr()
    S = off + off.T + arrow + arrow.T
    S = S.tocsr()
    d = np.asarray(abs(S).sum(axis=1)).ravel() + 1.0
    S = (S + sp.diags(d)).tocsr()
    S.sort_indices()
    rp, col, val = S.indptr.astype(np.uint32), S.indices.astype(np.uint32), S.data
    b = rng.uniform(-1, 1, n)
    x, info, _ = run(ctrl, "cg", rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 2000, 1e-10, 0.0,
                     loop_mode=2)
    _, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 2000, 1e-10, 0.0)
    assert abs(info["nIters"] - oi.nIters) <= 3
    assert l1_residual(rp, col, val, x, b) <= 1e-9


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_solver_max_iters_bookkeeping(ctrl, orc, kind):
    rp, col, val = matgen.poisson2d(40)
    n = len(rp) - 1
    b = np.ones(n)
    _, info, _ = run(ctrl, kind, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 7, 1e-30, 0.0)
    _, oi = orc.solve(kind, np.float64, rp, col, val, np.zeros(n), b, 1, 7, 1e-30, 0.0)
    assert info["nIters"] == oi.nIters
    assert info["currentResidual"] == pytest.approx(oi.currentResidual, rel=1e-8)


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_solver_zero_rhs_returns_b(ctrl, kind):
    rp, col, val = matgen.poisson2d(16)
    n = len(rp) - 1
    A = api.CsrMatrix.from_numpy(rp, col, val)
    x = torch.full((n,), 3.0, dtype=torch.float64, device="cuda")
    b = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 100, 1e-6, 1e-8)
    info = api.solve(kind, x, A, b, sc, ctrl)
    assert info["nIters"] == 0
    assert float(x.abs().sum()) == 0.0
    sc.release()


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
def test_solver_exact_initial_guess(ctrl, kind):
    rp, col, val = matgen.poisson2d(16)
    n = len(rp) - 1
    xs = np.random.default_rng(2).uniform(-1, 1, n)
    import scipy.sparse as sp
    b = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))) @ xs
    x, info, _ = run(ctrl, kind, rp, col, val, xs, b, torch.float64, L.DIAGONAL, 100, 1e-8, 0.0)
    assert info["nIters"] == 0
    np.testing.assert_array_equal(x, xs)


def test_cg_vector_path_without_meta(ctrl, orc):
    rp, col, val = matgen.poisson2d(50)
    n = len(rp) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    x, info, _ = run(ctrl, "cg", rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 2000, 1e-10, 0.0,
                     meta=False)
    _, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 2000, 1e-10, 0.0)
    assert abs(info["nIters"] - oi.nIters) <= 3


def test_cg_repeat_uses_cached_graph_and_is_deterministic(ctrl):
    rp, col, val = matgen.poisson2d(64)
    n = len(rp) - 1
    b = np.random.default_rng(4).uniform(-1, 1, n)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    bt = torch.tensor(b, device="cuda")
    outs = []
    for _ in range(3):
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        sc = api.SolverControl(L.DIAGONAL, 1000, 1e-10, 0.0)
        api.solve("cg", x, A, bt, sc, ctrl)
        sc.release()
        outs.append(x.cpu().numpy())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])


def test_missing_diagonal_is_reported(ctrl):
    rp, col, val = matgen.random_lengths([2, 2, 2], 3, seed=1)
    # make row 1 lack its diagonal: columns of row 1 are sorted distinct from {0,1,2}
    col = col.copy()
    col[2:4] = [0, 2]
    n = 3
    _, _, status = run(ctrl, "cg", rp, col, np.abs(val) + 1, np.zeros(n), np.ones(n), torch.float64,
                       L.DIAGONAL, 5, 1e-12, 0.0)
    assert status & 1


def test_solver_argument_errors(ctrl):
    rp, col, val = matgen.poisson2d(8)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    x = torch.zeros(63, dtype=torch.float64, device="cuda")
    b = torch.zeros(64, dtype=torch.float64, device="cuda")
    sc = api.SolverControl()
    with pytest.raises(api.ClsparseError) as e:
        api.solve("cg", x, A, b, sc, ctrl)
    assert e.value.status == L.clsparseInvalidSystemSize
    sc.release()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_residual_snapshots_are_the_residuals_of_capped_solves(ctrl, dtype):
    """clsparseB200SolverSetSnapshots keeps r after k iterations; a solve
    capped after k >= 2 iterations (maxIters = k - 1: the reference's loop
    stops when nIters >= maxIters after an update; maxIters = 0 stops before
    the first one) leaves x_k with b - A x_k = r_k up to the recursion's
    rounding."""
    import scipy.sparse as sp
    rp, col, val = matgen.diffusion3d_lognormal(16, sigma=1.0, seed=2)
    n = len(rp) - 1
    b = np.random.default_rng(9).uniform(-1, 1, n)
    t = NP[dtype]
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=dtype)
    A.create_meta(ctrl)
    bt = torch.tensor(b, dtype=dtype, device="cuda")
    ks = [0, 2, 5, 20, 37]
    snaps = torch.zeros(len(ks), n, dtype=dtype, device="cuda")
    x = torch.zeros(n, dtype=dtype, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, max(ks) - 1, 0.0, 0.0)
    sc.set_snapshots(ks, snaps)
    hist = torch.zeros(64, dtype=torch.float64, device="cuda")
    sc.set_history(hist)
    info = api.solve("cg", x, A, bt, sc, ctrl)
    assert sc.history_length() == max(ks) + 1 and info["nIters"] == max(ks) - 1
    sc.release()
    Am = sp.csr_matrix((np.asarray(val, t).astype(np.float64), col.astype(np.int64), rp.astype(np.int64)))
    bb = np.asarray(b, t).astype(np.float64)
    nb = np.abs(bb).sum()
    for j, k in enumerate(ks):
        xk = torch.zeros(n, dtype=dtype, device="cuda")
        if k > 0:
            sck = api.SolverControl(L.DIAGONAL, k - 1, 0.0, 0.0)
            api.solve("cg", xk, A, bt, sck, ctrl)
            sck.release()
        true_r = bb - Am @ xk.cpu().numpy().astype(np.float64)
        s = snaps[j].cpu().numpy().astype(np.float64)
        tol = 1e-11 if dtype == torch.float64 else 2e-4
        assert np.abs(s - true_r).sum() <= tol * nb, (k, np.abs(s - true_r).sum() / nb)
        # the history's L1 residuum is this vector's norm
        assert hist[k].item() == pytest.approx(np.abs(s).sum() / nb, rel=1e-6 if dtype == torch.float64 else 1e-3)
