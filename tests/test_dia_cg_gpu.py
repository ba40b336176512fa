"""The drop-in clsparse{S,D}csrcg and clsparse{S,D}csrbicgStab on the banded
engine (solver loop mode 3) against the oracle restatements of the
reference CG and BiCGStab (src/library/solvers/conjugate-gradients.hpp:73-226,
biconjugate-gradients-stabilized.hpp:61-266).

Parity bar as for the other loop modes: the same stop decision (iteration
counts within a small slack -- the banded kernel forms each row in the
reference's CSR-Adaptive order with separately rounded operations, but sums
the dot products in another order), the reference-run pins exactly
(tests/test_solver_ref_pin_gpu.py),
the reported residuals agree, and x meets the stop criterion on a fresh FP64
check. The reference's bookkeeping (maxIters, the previous nIters in the
first stop test, x = b for a zero right-hand side, an exact initial guess)
is checked exactly. Matrices the engine does not take (not banded, a zero
diagonal under Jacobi) run on the graph engine with its results."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, matgen

pytestmark = pytest.mark.gpu

NP = {torch.float64: np.float64, torch.float32: np.float32}


def banded9(n: int, seed: int = 4):
    """SPD matrix with nine diagonals at offsets 0, +-1, +-7, +-40, +-41 and
    random weights (diagonally dominant)."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for o in (1, 7, 40, 41):
        w = -rng.uniform(0.2, 1.0, n - o)
        i = np.arange(n - o)
        rows += [i, i + o]
        cols += [i + o, i]
        vals += [w, w]
        diag[i] += -w
        diag[i + o] += -w
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag + 0.05)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sort_indices()
    return A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data.astype(np.float64)


PROBLEMS = {
    "poisson64": lambda: matgen.poisson2d(64),
    "poisson_rect": lambda: matgen.poisson2d(37, 91),
    "diffusion3d": lambda: matgen.diffusion3d_lognormal(16, sigma=1.0, seed=2),
    "banded9": lambda: banded9(6000),
    "tridiag": lambda: tridiag(5000),
    "random_spd": lambda: matgen.random_spd(5000, seed=3),  # not banded: graph engine
}


def run(ctrl, rp, col, val, x0, b, dtype, precond, max_iters, rel, abs_, loop_mode=3, sc=None, norm=0, kind="cg"):
    ctrl.set_solver_loop_mode(loop_mode)
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=dtype)
    A.create_meta(ctrl)
    x = torch.tensor(np.asarray(x0), dtype=dtype, device="cuda")
    bt = torch.tensor(np.asarray(b), dtype=dtype, device="cuda")
    own = sc is None
    if own:
        sc = api.SolverControl(precond, max_iters, rel, abs_)
        if norm:
            sc.set_norm(norm)
    info = api.solve(kind, x, A, bt, sc, ctrl)
    status = sc.device_status()
    if own:
        sc.release()
    ctrl.set_solver_loop_mode(0)
    return x.cpu().numpy().astype(np.float64), info, status


def l1_residual(rp, col, val, x, b):
    n = len(rp) - 1
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    return np.abs(b - A @ x).sum() / np.abs(b).sum()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("precond", [L.DIAGONAL, L.NOPRECOND], ids=["jacobi", "none"])
@pytest.mark.parametrize("prob", sorted(PROBLEMS))
def test_banded_cg_matches_oracle(ctrl, orc, prob, precond, dtype):
    rp, col, val = PROBLEMS[prob]()
    n = len(rp) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    t = NP[dtype]
    x, info, status = run(ctrl, rp, col, val, np.zeros(n), b, dtype, precond, 5000, rel, 0.0)
    _, oi = orc.solve("cg", t, rp, col, val, np.zeros(n, t), np.asarray(b, t), precond, 5000, rel, 0.0)
    slack = max(3, int(0.03 * oi.nIters))
    assert abs(info["nIters"] - oi.nIters) <= slack, (info, oi.nIters)
    assert info["initialResidual"] == pytest.approx(oi.initialResidual, rel=1e-5)
    assert info["currentResidual"] <= rel
    assert status == 0
    r_true = l1_residual(rp, col, np.asarray(val, t).astype(np.float64), x, np.asarray(b, t).astype(np.float64))
    assert r_true <= (10 * rel if dtype == torch.float64 else 50 * rel)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_banded_cg_agrees_with_graph_engine(ctrl, dtype):
    rp, col, val = matgen.diffusion3d_lognormal(20, sigma=1.5, seed=7)
    n = len(rp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    xg, ig, _ = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 5000, rel, 0.0, loop_mode=0)
    xb, ib, _ = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 5000, rel, 0.0, loop_mode=3)
    assert abs(ig["nIters"] - ib["nIters"]) <= max(3, int(0.03 * ig["nIters"]))
    assert ib["initialResidual"] == pytest.approx(ig["initialResidual"], rel=1e-6)
    tol = 1e-7 if dtype == torch.float64 else 5e-3
    assert np.abs(xb - xg).max() <= tol * np.abs(xg).max()


def test_banded_cg_l2_norm_option(ctrl, orc):
    rp, col, val = matgen.poisson2d(50)
    n = len(rp) - 1
    b = np.random.default_rng(8).uniform(-1, 1, n)
    xg, ig, _ = run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 3000, 1e-9, 0.0,
                    loop_mode=0, norm=1)
    xb, ib, _ = run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 3000, 1e-9, 0.0,
                    loop_mode=3, norm=1)
    assert abs(ig["nIters"] - ib["nIters"]) <= 3
    assert ib["initialResidual"] == pytest.approx(ig["initialResidual"], rel=1e-12)
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    assert np.linalg.norm(b - A @ xb) / np.linalg.norm(b) <= 1e-8


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_banded_cg_max_iters_bookkeeping(ctrl, orc, dtype):
    rp, col, val = matgen.poisson2d(40)
    n = len(rp) - 1
    b = np.ones(n)
    t = NP[dtype]
    x, info, _ = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 7, 1e-30, 0.0)
    xo, oi = orc.solve("cg", t, rp, col, val, np.zeros(n, t), np.asarray(b, t), 1, 7, 1e-30, 0.0)
    assert info["nIters"] == oi.nIters
    tol = 1e-10 if dtype == torch.float64 else 1e-4
    assert info["currentResidual"] == pytest.approx(oi.currentResidual, rel=tol)
    np.testing.assert_allclose(x, xo.astype(np.float64), rtol=tol, atol=tol * np.abs(xo).max())


def test_banded_cg_previous_n_iters_enters_first_stop_test(ctrl, orc):
    """The reference's first stop test sees the nIters the control holds from
    the previous solve: a second solve with a control that ran out of
    iterations stops at once."""
    rp, col, val = matgen.poisson2d(30)
    n = len(rp) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    sc = api.SolverControl(L.DIAGONAL, 9, 1e-30, 0.0)
    _, i1, _ = run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 0, 0, 0, sc=sc)
    x0 = np.random.default_rng(3).uniform(-1, 1, n)
    x2, i2, _ = run(ctrl, rp, col, val, x0, b, torch.float64, L.DIAGONAL, 0, 0, 0, sc=sc)
    sc.release()
    _, o1 = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 9, 1e-30, 0.0)
    _, o2 = orc.solve("cg", np.float64, rp, col, val, x0, b, 1, 9, 1e-30, 0.0, n_iters_in=o1.nIters)
    assert (i1["nIters"], i2["nIters"]) == (o1.nIters, o2.nIters)
    assert i2["nIters"] == 0
    np.testing.assert_array_equal(x2, x0)


def test_banded_cg_zero_rhs_returns_b(ctrl):
    rp, col, val = matgen.poisson2d(16)
    n = len(rp) - 1
    ctrl.set_solver_loop_mode(3)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    x = torch.full((n,), 3.0, dtype=torch.float64, device="cuda")
    b = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 100, 1e-6, 1e-8)
    info = api.solve("cg", x, A, b, sc, ctrl)
    ctrl.set_solver_loop_mode(0)
    assert info["nIters"] == 0
    assert float(x.abs().sum()) == 0.0
    sc.release()


def test_banded_cg_exact_initial_guess(ctrl):
    rp, col, val = matgen.poisson2d(16)
    n = len(rp) - 1
    xs = np.random.default_rng(2).uniform(-1, 1, n)
    b = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))) @ xs
    x, info, _ = run(ctrl, rp, col, val, xs, b, torch.float64, L.DIAGONAL, 100, 1e-8, 0.0)
    assert info["nIters"] == 0
    np.testing.assert_array_equal(x, xs)


def test_banded_cg_missing_diagonal_runs_graph_engine(ctrl):
    """Row 1 without a diagonal entry under Jacobi: the banded engine leaves x
    untouched and the graph engine reports the missing diagonal as in the
    other loop modes."""
    rp, col, val = matgen.random_lengths([2, 2, 2], 3, seed=1)
    col = col.copy()
    col[2:4] = [0, 2]
    n = 3
    _, _, s3 = run(ctrl, rp, col, np.abs(val) + 1, np.zeros(n), np.ones(n), torch.float64, L.DIAGONAL, 5, 1e-12, 0.0)
    _, _, s0 = run(ctrl, rp, col, np.abs(val) + 1, np.zeros(n), np.ones(n), torch.float64, L.DIAGONAL, 5, 1e-12, 0.0,
                   loop_mode=0)
    assert s3 & 1 and s3 == s0


def test_banded_cg_is_deterministic(ctrl):
    rp, col, val = matgen.poisson2d(64)
    n = len(rp) - 1
    b = np.random.default_rng(4).uniform(-1, 1, n)
    outs = [run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 1000, 1e-10, 0.0)[0]
            for _ in range(3)]
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])


def test_banded_cg_barrier_timeout_is_reported_and_recovers(ctrl, orc, monkeypatch):
    rp, col, val = matgen.poisson2d(64)
    n = len(rp) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    monkeypatch.setenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE", "1")
    monkeypatch.setenv("CLSPARSE_B200_BARRIER_WAIT_NS", "2000000")
    sc = api.SolverControl(L.DIAGONAL, 2000, 1e-10, 0.0)
    with pytest.raises(api.ClsparseError) as e:
        run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 0, 0, 0, sc=sc)
    ctrl.set_solver_loop_mode(0)
    assert e.value.status == L.clsparseInvalidKernelExecution
    assert sc.device_status() & 32
    sc.release()
    torch.cuda.synchronize()  # the context is still usable
    monkeypatch.delenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")
    monkeypatch.delenv("CLSPARSE_B200_BARRIER_WAIT_NS")
    x, info, status = run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 2000, 1e-10, 0.0)
    assert status == 0
    _, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, L.DIAGONAL, 2000, 1e-10, 0.0)
    assert abs(info["nIters"] - oi.nIters) <= max(3, int(0.03 * oi.nIters))
    assert l1_residual(rp, col, val, x, b) <= 1e-9


def tridiag(n: int, seed: int = 6):
    rng = np.random.default_rng(seed)
    w = -rng.uniform(0.5, 1.5, n - 1)
    d = np.zeros(n)
    d[:-1] -= w
    d[1:] -= w
    A = sp.diags([w, d + 0.01, w], [-1, 0, 1], format="csr")
    A.sort_indices()
    return A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data.astype(np.float64)


def convdiff5(m: int = 40):
    """Five-point convection-diffusion: a banded matrix that is not symmetric."""
    rp, col, val = matgen.poisson2d(m)
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)))
    A = (A + 0.3 * sp.eye(A.shape[0], k=1) - 0.3 * sp.eye(A.shape[0], k=-1)).tocsr()
    A.eliminate_zeros()
    A.sort_indices()
    return A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data.astype(np.float64)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("prob", ["poisson64", "tridiag", "convdiff5", "diffusion3d"])
def test_banded_cg_symmetric_form_is_bitwise_equal(ctrl, monkeypatch, prob, dtype):
    """The form that reads a symmetric matrix's lower diagonals from the upper
    ones (forced on; by default it runs only when the working set exceeds half
    of L2) gives the same x bit for bit; a non-symmetric matrix, or one with
    more diagonals than the form takes, runs the plain form."""
    rp, col, val = {"poisson64": lambda: matgen.poisson2d(64), "tridiag": lambda: tridiag(5000),
                    "convdiff5": convdiff5,
                    "diffusion3d": lambda: matgen.diffusion3d_lognormal(16, sigma=1.0, seed=2)}[prob]()
    n = len(rp) - 1
    b = np.random.default_rng(9).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("CLSPARSE_B200_DIA_SYM", mode)
        out[mode] = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 60 if prob == "convdiff5" else 5000,
                        rel, 0.0)
    assert out["0"][1] == out["1"][1]
    np.testing.assert_array_equal(out["0"][0], out["1"][0])


# ---- BiCGStab (clsparse{S,D}csrbicgStab in loop mode 3)

BICG_PROBLEMS = dict(PROBLEMS, convdiff5=lambda: convdiff5(48))


def bicg_slack(n_ref):
    # BiCGStab's convergence history is irregular and reacts to the order of
    # the reduction sums (the bar of the other loop modes)
    return max(8, int(0.12 * n_ref))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("precond", [L.DIAGONAL, L.NOPRECOND], ids=["jacobi", "none"])
@pytest.mark.parametrize("prob", sorted(BICG_PROBLEMS))
def test_banded_bicgstab_matches_oracle(ctrl, orc, prob, precond, dtype):
    rp, col, val = BICG_PROBLEMS[prob]()
    n = len(rp) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    t = NP[dtype]
    x, info, status = run(ctrl, rp, col, val, np.zeros(n), b, dtype, precond, 5000, rel, 0.0, kind="bicgstab")
    _, oi = orc.solve("bicgstab", t, rp, col, val, np.zeros(n, t), np.asarray(b, t), precond, 5000, rel, 0.0)
    assert abs(info["nIters"] - oi.nIters) <= bicg_slack(oi.nIters), (info, oi.nIters)
    assert info["initialResidual"] == pytest.approx(oi.initialResidual, rel=1e-5)
    assert info["currentResidual"] <= rel
    assert status & ~8 == 0  # a breakdown flag is information, as in the other modes
    r_true = l1_residual(rp, col, np.asarray(val, t).astype(np.float64), x, np.asarray(b, t).astype(np.float64))
    assert r_true <= (10 * rel if dtype == torch.float64 else 50 * rel)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_banded_bicgstab_agrees_with_graph_engine(ctrl, dtype):
    rp, col, val = convdiff5(64)
    n = len(rp) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    rel = 1e-10 if dtype == torch.float64 else 1e-5
    xg, ig, _ = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 5000, rel, 0.0, loop_mode=0,
                    kind="bicgstab")
    xb, ib, _ = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 5000, rel, 0.0, loop_mode=3,
                    kind="bicgstab")
    assert abs(ig["nIters"] - ib["nIters"]) <= bicg_slack(ig["nIters"])
    assert ib["initialResidual"] == pytest.approx(ig["initialResidual"], rel=1e-6)
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    tol = 1e-9 if dtype == torch.float64 else 1e-4
    assert np.abs(b - A @ xb).sum() / np.abs(b).sum() <= tol


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_banded_bicgstab_max_iters_bookkeeping(ctrl, orc, dtype):
    rp, col, val = convdiff5(40)
    n = len(rp) - 1
    b = np.ones(n)
    t = NP[dtype]
    x, info, _ = run(ctrl, rp, col, val, np.zeros(n), b, dtype, L.DIAGONAL, 7, 1e-30, 0.0, kind="bicgstab")
    xo, oi = orc.solve("bicgstab", t, rp, col, val, np.zeros(n, t), np.asarray(b, t), 1, 7, 1e-30, 0.0)
    assert info["nIters"] == oi.nIters
    tol = 1e-9 if dtype == torch.float64 else 2e-3
    assert info["currentResidual"] == pytest.approx(oi.currentResidual, rel=tol)
    np.testing.assert_allclose(x, xo.astype(np.float64), rtol=tol, atol=tol * np.abs(xo).max())


def test_banded_bicgstab_previous_n_iters_enters_first_stop_tests(ctrl, orc):
    rp, col, val = convdiff5(30)
    n = len(rp) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    sc = api.SolverControl(L.DIAGONAL, 9, 1e-30, 0.0)
    _, i1, _ = run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 0, 0, 0, sc=sc, kind="bicgstab")
    x0 = np.random.default_rng(3).uniform(-1, 1, n)
    x2, i2, _ = run(ctrl, rp, col, val, x0, b, torch.float64, L.DIAGONAL, 0, 0, 0, sc=sc, kind="bicgstab")
    sc.release()
    _, o1 = orc.solve("bicgstab", np.float64, rp, col, val, np.zeros(n), b, 1, 9, 1e-30, 0.0)
    _, o2 = orc.solve("bicgstab", np.float64, rp, col, val, x0, b, 1, 9, 1e-30, 0.0, n_iters_in=o1.nIters)
    assert (i1["nIters"], i2["nIters"]) == (o1.nIters, o2.nIters)
    np.testing.assert_array_equal(x2, x0)


def test_banded_bicgstab_exact_initial_guess(ctrl):
    rp, col, val = convdiff5(16)
    n = len(rp) - 1
    xs = np.random.default_rng(2).uniform(-1, 1, n)
    bx = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))) @ xs
    x, info, _ = run(ctrl, rp, col, val, xs, bx, torch.float64, L.DIAGONAL, 100, 1e-8, 0.0, kind="bicgstab")
    assert info["nIters"] == 0
    np.testing.assert_array_equal(x, xs)


def test_banded_bicgstab_zero_rhs_returns_b(ctrl):
    rp, col, val = convdiff5(16)
    n = len(rp) - 1
    x, info, _ = run(ctrl, rp, col, val, np.full(n, 3.0), np.zeros(n), torch.float64, L.DIAGONAL, 100, 1e-6, 1e-8,
                     kind="bicgstab")
    assert info["nIters"] == 0
    assert np.abs(x).sum() == 0.0


def test_banded_bicgstab_barrier_timeout_is_reported_and_recovers(ctrl, orc, monkeypatch):
    rp, col, val = convdiff5(48)
    n = len(rp) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    monkeypatch.setenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE", "1")
    monkeypatch.setenv("CLSPARSE_B200_BARRIER_WAIT_NS", "2000000")
    sc = api.SolverControl(L.DIAGONAL, 2000, 1e-10, 0.0)
    with pytest.raises(api.ClsparseError) as e:
        run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 0, 0, 0, sc=sc, kind="bicgstab")
    ctrl.set_solver_loop_mode(0)
    assert e.value.status == L.clsparseInvalidKernelExecution
    assert sc.device_status() & 32
    sc.release()
    torch.cuda.synchronize()
    monkeypatch.delenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")
    monkeypatch.delenv("CLSPARSE_B200_BARRIER_WAIT_NS")
    x, info, _ = run(ctrl, rp, col, val, np.zeros(n), b, torch.float64, L.DIAGONAL, 2000, 1e-10, 0.0,
                     kind="bicgstab")
    assert l1_residual(rp, col, val, x, b) <= 1e-9
