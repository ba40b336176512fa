"""The banded inner solves of the mixed-precision refinement (diagonal
storage, one fused cooperative launch per inner solve; clsparse_b200/csrc/
dia.cu) against the CSR inner solves they replace (CLSPARSE_B200_DIA=0),
through the C ABI.

Both must reach the FP64 residual 1e-10 (recomputed on the host) and agree
with each other and with the FP64 CG oracle's solution; the inner iteration
counts agree within a small slack (FP32 arithmetic in a different order).
A matrix with too many diagonals stays on CSR. A barrier that is never
released ends the banded launch with the barrier-timeout status."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, learn, matgen

pytestmark = pytest.mark.gpu


def residual(rp, col, val, x, b):
    n = len(rp) - 1
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    return np.linalg.norm(b - A @ x) / np.linalg.norm(b)


def mixed(ctrl, mat, b, inner, dia, monkeypatch, precond=L.DIAGONAL):
    monkeypatch.setenv("CLSPARSE_B200_DIA", "1" if dia else "0")
    A = api.CsrMatrix.from_numpy(*mat)
    A.create_meta(ctrl)
    x = torch.zeros(A.num_rows, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(precond, 100000, 1e-10, 0.0)
    info = api.cg_mixed(x, A, torch.tensor(b, device="cuda"), sc, ctrl, inner=inner, inner_tol=0.3)
    sc.release()
    return x.cpu().numpy(), info


CASES = {
    "poisson2d_96": lambda: matgen.poisson2d(96),
    "diffusion3d_24": lambda: matgen.diffusion3d_lognormal(24, sigma=1.5, seed=4),
    "grf2d_80": lambda: matgen.diffusion2d_grf(80, corr_len=0.1, sigma=2.0, seed=9),
}


@pytest.mark.parametrize("precond", [L.DIAGONAL, L.NOPRECOND], ids=["jacobi", "none"])
@pytest.mark.parametrize("inner", ["fp32", "bf16"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_banded_mixed_matches_csr(ctrl, orc, monkeypatch, case, inner, precond):
    mat = CASES[case]()
    n = len(mat[0]) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    xb, ib = mixed(ctrl, mat, b, inner, True, monkeypatch, precond)
    xc, ic = mixed(ctrl, mat, b, inner, False, monkeypatch, precond)
    xo, _ = orc.solve("cg", np.float64, *mat, np.zeros(n), b, L.DIAGONAL, 100000, 1e-13, 0.0)
    if inner == "bf16":
        # The banded BF16 copy keeps A's row sums (FP32 diagonal carrying each
        # row's rounding), so it stays SPD and must converge; the CSR copy
        # rounds every entry and may not contract on the high-contrast
        # operators (it must then say so, not claim success).
        assert ib["converged"] == 1, ib
        assert residual(*mat, xb, b) <= 1.5e-10
        assert not ic["converged"] or residual(*mat, xc, b) <= 1.5e-10
        if ic["converged"]:
            assert ib["innerIterations"] <= ic["innerIterations"] + max(10, int(0.1 * ic["innerIterations"]))
        assert np.linalg.norm(xb - xo) / np.linalg.norm(xo) <= 1e-7
        return
    assert ib["converged"] == 1 and ic["converged"] == 1, (ib, ic)
    assert residual(*mat, xb, b) <= 1.5e-10
    slack = max(10, int(0.1 * ic["innerIterations"]))
    assert abs(ib["innerIterations"] - ic["innerIterations"]) <= slack, (ib, ic)
    assert np.linalg.norm(xb - xo) / np.linalg.norm(xo) <= 1e-7


def test_banded_learned_matches_csr(ctrl, monkeypatch):
    spai, _ = learn.train(ctrl, sizes=(32,), seeds=range(2), steps=60, lr=3e-3)
    smp = learn.Sample(ctrl, 96, 7, with_probes=False)
    spai.set_matrix(smp.A, ctrl)
    spai.build(ctrl)
    out = {}
    for dia in (True, False):
        monkeypatch.setenv("CLSPARSE_B200_DIA", "1" if dia else "0")
        x = torch.zeros(smp.A.num_rows, dtype=torch.float64, device="cuda")
        sc = api.SolverControl(L.DIAGONAL, 100000, 1e-10, 0.0)
        out[dia] = (api.cg_learned(x, smp.A, smp.b, sc, spai, ctrl, inner="fp32", inner_tol=0.3),
                    x.cpu().numpy())
        sc.release()
    spai.release()
    (ib, xb), (ic, xc) = out[True], out[False]
    assert ib["converged"] == 1 and ib["fell_back"] == 0
    assert abs(ib["innerIterations"] - ic["innerIterations"]) <= max(10, int(0.1 * ic["innerIterations"]))
    b = smp.b.cpu().numpy()
    assert residual(*smp.np, xb, b) <= 1.5e-10
    assert np.linalg.norm(xb - xc) / np.linalg.norm(xc) <= 1e-7


@pytest.mark.parametrize("m", [96, 300])
def test_local_t_form_equals_three_phase_form(ctrl, monkeypatch, m):
    """The learned iteration with t = G r kept per CTA in shared memory (two
    grid exchanges per iteration) computes every value the three-phase form
    computes, in the same order: the solves agree bit for bit. 300^2 rows
    gives slices whose halo reaches into the next CTA's rows."""
    spai, _ = learn.train(ctrl, sizes=(32,), seeds=range(2), steps=40, lr=3e-3)
    smp = learn.Sample(ctrl, m, 7, with_probes=False)
    spai.set_matrix(smp.A, ctrl)
    spai.build(ctrl)
    out = {}
    for local in ("1", "0"):
        monkeypatch.setenv("CLSPARSE_B200_DIA_LOCAL_T", local)
        x = torch.zeros(smp.A.num_rows, dtype=torch.float64, device="cuda")
        sc = api.SolverControl(L.DIAGONAL, 100000, 1e-10, 0.0)
        out[local] = (api.cg_learned(x, smp.A, smp.b, sc, spai, ctrl, inner="fp32", inner_tol=0.3),
                      x.cpu().numpy())
        sc.release()
    spai.release()
    (i1, x1), (i0, x0) = out["1"], out["0"]
    assert i1["converged"] == 1 and i1["fell_back"] == 0
    assert i1["innerIterations"] == i0["innerIterations"]
    np.testing.assert_array_equal(x1, x0)
    assert residual(*smp.np, x1, smp.b.cpu().numpy()) <= 1.5e-10


def test_matrix_with_many_diagonals_stays_on_csr(ctrl, monkeypatch):
    mat = matgen.random_spd(3000, seed=5)
    n = len(mat[0]) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n)
    xb, ib = mixed(ctrl, mat, b, "fp32", True, monkeypatch)
    xc, ic = mixed(ctrl, mat, b, "fp32", False, monkeypatch)
    assert ib["converged"] == 1
    assert ib["innerIterations"] == ic["innerIterations"]
    np.testing.assert_array_equal(xb, xc)


def test_banded_barrier_timeout_is_reported_and_recovers(ctrl, monkeypatch):
    mat = matgen.poisson2d(64)
    n = len(mat[0]) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    monkeypatch.setenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE", "1")
    monkeypatch.setenv("CLSPARSE_B200_BARRIER_WAIT_NS", "2000000")
    with pytest.raises(api.ClsparseError) as e:
        mixed(ctrl, mat, b, "fp32", True, monkeypatch)
    assert e.value.status == L.clsparseInvalidKernelExecution
    torch.cuda.synchronize()
    monkeypatch.delenv("CLSPARSE_B200_TEST_BARRIER_NEVER_RELEASE")
    monkeypatch.delenv("CLSPARSE_B200_BARRIER_WAIT_NS")
    x, info = mixed(ctrl, mat, b, "fp32", True, monkeypatch)
    assert info["converged"] == 1 and residual(*mat, x, b) <= 1.5e-10
