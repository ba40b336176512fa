"""clsparse{S,D}csrmm (C = alpha*A*B + beta*C, A sparse CSR, B and C dense)
through the C ABI against numpy in float64. Row-major B/C as the reference
indexes them (src/library/kernels/csrmm_general.cl:60-167), column-major
honoured, padded leading dimensions, every group width of the kernel."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, matgen

pytestmark = pytest.mark.gpu
TOL = {torch.float64: 1e-12, torch.float32: 1e-5}


def dense(t: torch.Tensor, rows, cols, ld, major):
    m = L.cldenseMatrix()
    m.num_rows, m.num_cols, m.lead_dim, m.major = rows, cols, ld, major
    m.values = C.c_void_p(t.data_ptr())
    m.off_values = 0
    return m


def layout(M, ld, major, dtype):
    """M (rows x cols) stored with leading dimension ld in the given major order."""
    rows, cols = M.shape
    if major == L.rowMajor:
        buf = np.zeros((rows, ld))
        buf[:, :cols] = M
    else:
        buf = np.zeros((cols, ld))
        buf[:, :rows] = M.T
    return torch.tensor(buf.ravel(), dtype=dtype, device="cuda")


def unlayout(t, rows, cols, ld, major):
    a = t.cpu().numpy().astype(np.float64)
    return a.reshape(rows, ld)[:, :cols] if major == L.rowMajor else a.reshape(cols, ld)[:, :rows].T


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("ncols", [1, 3, 8, 33, 64])
@pytest.mark.parametrize("major", ["row", "col"])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-0.5, 1.0), (2.0, -1.5)])
def test_csrmm_matches_numpy(ctrl, dtype, ncols, major, alpha, beta):
    mj = L.rowMajor if major == "row" else L.columnMajor
    rng = np.random.default_rng(ncols)
    rp, col, val = matgen.irregular(3000, mu=2.0, sigma=1.0, n_dense=2, dense_len=1400, seed=ncols, ncols=2900)
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=2900, dtype=dtype)
    B = rng.uniform(-1, 1, (2900, ncols))
    C0 = rng.uniform(-1, 1, (3000, ncols))
    ldb = (ncols if mj == L.rowMajor else 2900) + 3
    ldc = (ncols if mj == L.rowMajor else 3000) + 5
    tb, tc = layout(B, ldb, mj, dtype), layout(C0, ldc, mj, dtype)
    db, dc = dense(tb, 2900, ncols, ldb, mj), dense(tc, 3000, ncols, ldc, mj)
    a = torch.tensor([alpha], dtype=dtype, device="cuda")
    b = torch.tensor([beta], dtype=dtype, device="cuda")
    fn = api.lib().clsparseDcsrmm if dtype == torch.float64 else api.lib().clsparseScsrmm
    st = fn(C.byref(api.scalar(a)), C.byref(A.s), C.byref(db), C.byref(api.scalar(b)), C.byref(dc), ctrl.handle)
    assert st == 0
    t = np.float64 if dtype == torch.float64 else np.float32
    Am = sp.csr_matrix((np.asarray(val, t).astype(np.float64), col.astype(np.int64), rp.astype(np.int64)),
                       shape=(3000, 2900))
    Bc, Cc = np.asarray(B, t).astype(np.float64), np.asarray(C0, t).astype(np.float64)
    ref = alpha * (Am @ Bc) + beta * Cc
    scale = abs(alpha) * (abs(Am) @ abs(Bc)) + abs(beta) * abs(Cc) + 1e-300
    out = unlayout(tc, 3000, ncols, ldc, mj)
    assert np.max(np.abs(out - ref) / scale) <= TOL[dtype] * 10
    # padding left untouched
    if mj == L.rowMajor:
        pad = tc.cpu().numpy().reshape(3000, ldc)[:, ncols:]
        np.testing.assert_array_equal(pad, 0)


def test_csrmm_beta_zero_ignores_nan(ctrl):
    rp, col, val = matgen.poisson2d(20)
    n = len(rp) - 1
    A = api.CsrMatrix.from_numpy(rp, col, val)
    B = np.ones((n, 4))
    tb = layout(B, 4, L.rowMajor, torch.float64)
    tc = torch.full((n * 4,), float("nan"), dtype=torch.float64, device="cuda")
    one = torch.ones(1, dtype=torch.float64, device="cuda")
    zero = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = api.lib().clsparseDcsrmm(C.byref(api.scalar(one)), C.byref(A.s), C.byref(dense(tb, n, 4, 4, L.rowMajor)),
                                  C.byref(api.scalar(zero)), C.byref(dense(tc, n, 4, 4, L.rowMajor)), ctrl.handle)
    assert st == 0
    out = tc.cpu().numpy().reshape(n, 4)
    Am = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)))
    np.testing.assert_allclose(out, (Am @ B), rtol=0, atol=1e-12)


def test_csrmm_size_errors(ctrl):
    rp, col, val = matgen.poisson2d(8)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    t = torch.zeros(64 * 4, dtype=torch.float64, device="cuda")
    one = torch.ones(1, dtype=torch.float64, device="cuda")
    bad_b = dense(t, 10, 4, 4, L.rowMajor)          # fewer rows than A has columns
    good_c = dense(t, 64, 4, 4, L.rowMajor)
    st = api.lib().clsparseDcsrmm(C.byref(api.scalar(one)), C.byref(A.s), C.byref(bad_b), C.byref(api.scalar(one)),
                                  C.byref(good_c), ctrl.handle)
    assert st == L.clsparseInvalidSize
    bad_ld = dense(t, 64, 4, 2, L.rowMajor)         # leading dimension below the row length
    st = api.lib().clsparseDcsrmm(C.byref(api.scalar(one)), C.byref(A.s), C.byref(bad_ld), C.byref(api.scalar(one)),
                                  C.byref(good_c), ctrl.handle)
    assert st == L.clsparseInvalidSize
