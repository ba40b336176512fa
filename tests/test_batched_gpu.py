"""Batched FP32 Jacobi-CG (clsparseScsrcgBatched) through the C ABI: every
system's solution against an FP64 direct solve of that system, and the FP64
residual each system reports against one recomputed here -- from diagonal
storage (banded systems, the default) and from CSR."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, matgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["diagonal", "csr"])
@pytest.mark.parametrize("lanes", [None, 1, 4])
def test_batched_cg_matches_direct_solves(ctrl, lanes, storage, monkeypatch):
    """Banded systems run from diagonal storage by default;
    CLSPARSE_B200_BATCH_DIA=0 keeps them on CSR (the lanes-per-row path)."""
    if storage == "csr":
        monkeypatch.setenv("CLSPARSE_B200_BATCH_DIA", "0")
    rp, col, val, off, dims = matgen.batched_systems(48, 40, 4000, sigma=1.0, seed=3)
    n = len(rp) - 1
    A64 = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    b = np.random.default_rng(5).uniform(-1, 1, n).astype(np.float32)
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=torch.float32)
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 20000, 1e-6, 0.0)
    ln = None if lanes is None else np.full(48, lanes)
    out = api.cg_batched(x, A, torch.tensor(b, device="cuda"), off, sc, ctrl, lanes=ln)
    sc.release()
    assert out["converged"] == 48, out
    xs = x.cpu().numpy().astype(np.float64)
    A32 = sp.csr_matrix((val.astype(np.float32).astype(np.float64), col.astype(np.int64), rp.astype(np.int64)),
                        shape=(n, n))
    for s in range(48):
        a, e = int(off[s]), int(off[s + 1])
        bs = b[a:e].astype(np.float64)
        rres = np.linalg.norm(bs - A32[a:e, a:e] @ xs[a:e]) / np.linalg.norm(bs)
        assert rres <= 1.05e-6, (s, rres)
        assert abs(out["residuals"][s] - rres) <= 1e-9 + 1e-3 * rres
        xd = spla.spsolve(A64[a:e, a:e].tocsc(), bs)
        cond_bound = 1e-6 * 1e4
        assert np.linalg.norm(xs[a:e] - xd) / np.linalg.norm(xd) <= cond_bound


def test_batched_cg_repeat_is_deterministic(ctrl):
    rp, col, val, off, _ = matgen.batched_systems(16, 100, 2000, seed=9)
    n = len(rp) - 1
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=torch.float32)
    b = torch.tensor(np.random.default_rng(1).uniform(-1, 1, n), dtype=torch.float32, device="cuda")
    outs = []
    for _ in range(2):
        x = torch.zeros(n, dtype=torch.float32, device="cuda")
        sc = api.SolverControl(L.DIAGONAL, 5000, 1e-6, 0.0)
        api.cg_batched(x, A, b, off, sc, ctrl)
        sc.release()
        outs.append(x.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_batched_rejects_bad_offsets(ctrl):
    rp, col, val, off, _ = matgen.batched_systems(4, 50, 200, seed=2)
    n = len(rp) - 1
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=torch.float32)
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 100, 1e-6, 0.0)
    bad = off.copy()
    bad[-1] += 1
    with pytest.raises(api.ClsparseError):
        api.cg_batched(x, A, x, bad, sc, ctrl)
    sc.release()


def test_batch_with_a_non_banded_system_runs_on_csr(ctrl):
    """One system with more column offsets than diagonal storage takes: the
    batch runs from CSR, and every system still meets the tolerance."""
    rp, col, val, off, _ = matgen.batched_systems(12, 200, 3000, sigma=1.0, seed=4)
    S = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(len(rp) - 1,) * 2)
    rrp, rcol, rval = matgen.random_spd(1500, seed=8)
    R = sp.csr_matrix((rval, rcol.astype(np.int64), rrp.astype(np.int64)), shape=(1500, 1500))
    M = sp.block_diag([S, R], format="csr")
    M.sort_indices()
    offs = np.concatenate([off, [off[-1] + 1500]]).astype(np.uint32)
    n = M.shape[0]
    b = np.random.default_rng(6).uniform(-1, 1, n).astype(np.float32)
    A = api.CsrMatrix.from_numpy(M.indptr.astype(np.uint32), M.indices.astype(np.uint32), M.data,
                                 dtype=torch.float32)
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 20000, 1e-6, 0.0)
    out = api.cg_batched(x, A, torch.tensor(b, device="cuda"), offs, sc, ctrl)
    sc.release()
    assert out["converged"] == 13, out
    M32 = sp.csr_matrix((M.data.astype(np.float32).astype(np.float64), M.indices, M.indptr), shape=M.shape)
    xs = x.cpu().numpy().astype(np.float64)
    for s in range(13):
        a, e = int(offs[s]), int(offs[s + 1])
        bs = b[a:e].astype(np.float64)
        assert np.linalg.norm(bs - M32[a:e, a:e] @ xs[a:e]) / np.linalg.norm(bs) <= 1.05e-6
