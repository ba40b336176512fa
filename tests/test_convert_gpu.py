"""Format conversions (clsparse{S,D}coo2csr, csr2coo, csr2dense, dense2csr;
reference src/library/transform/) through the C ABI against scipy, including
empty rows, more rows than one scan block, row- and column-major dense
matrices with padded leading dimensions, and round trips."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api

pytestmark = pytest.mark.gpu
DT = {"f64": torch.float64, "f32": torch.float32}
NPT = {"f64": np.float64, "f32": np.float32}


def random_csr(rows, cols, density, seed, empty_every=7):
    M = sp.random(rows, cols, density=density, random_state=seed, format="csr")
    M = M.tolil()
    for r in range(0, rows, empty_every):
        M[r, :] = 0
    M = M.tocsr()
    M.eliminate_zeros()
    M.sort_indices()
    return M


def coo_struct(ri, ci, vv, rows, cols):
    m = L.clsparseCooMatrix()
    api.lib().clsparseInitCooMatrix(C.byref(m))
    m.num_rows, m.num_cols, m.num_nonzeros = rows, cols, vv.numel()
    m.values, m.col_indices, m.row_indices = vv.data_ptr(), ci.data_ptr(), ri.data_ptr()
    return m


def dense_struct(t, rows, cols, ld, major):
    d = L.cldenseMatrix()
    d.num_rows, d.num_cols, d.lead_dim, d.major = rows, cols, ld, major
    d.values = C.c_void_p(t.data_ptr())
    d.off_values = 0
    return d


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_coo2csr_and_back(ctrl, dt):
    dtype, t = DT[dt], NPT[dt]
    M = random_csr(3000, 700, 0.01, 3)
    coo = M.tocoo()
    order = np.lexsort((coo.col, coo.row))
    ri = torch.tensor(coo.row[order].astype(np.int32), device="cuda")
    ci = torch.tensor(coo.col[order].astype(np.int32), device="cuda")
    vv = torch.tensor(coo.data[order].astype(t), device="cuda")
    cm = coo_struct(ri, ci, vv, 3000, 700)
    out = api.CsrMatrix(torch.zeros(3001, dtype=torch.int32, device="cuda"),
                        torch.zeros(M.nnz, dtype=torch.int32, device="cuda"),
                        torch.zeros(M.nnz, dtype=dtype, device="cuda"), 700)
    fn = api.lib().clsparseDcoo2csr if dt == "f64" else api.lib().clsparseScoo2csr
    assert fn(C.byref(cm), C.byref(out.s), ctrl.handle) == 0
    assert (out.s.num_rows, out.s.num_cols, out.s.num_nonzeros) == (3000, 700, M.nnz)
    np.testing.assert_array_equal(out.row_ptr.cpu().numpy(), M.indptr)
    np.testing.assert_array_equal(out.col.cpu().numpy(), M.indices)
    np.testing.assert_array_equal(out.val.cpu().numpy(), M.data.astype(t))
    # and back
    ri2 = torch.zeros_like(ri)
    ci2 = torch.zeros_like(ci)
    vv2 = torch.zeros_like(vv)
    cm2 = coo_struct(ri2, ci2, vv2, 0, 0)
    fn2 = api.lib().clsparseDcsr2coo if dt == "f64" else api.lib().clsparseScsr2coo
    assert fn2(C.byref(out.s), C.byref(cm2), ctrl.handle) == 0
    assert cm2.num_nonzeros == M.nnz and cm2.num_rows == 3000
    np.testing.assert_array_equal(ri2.cpu().numpy(), coo.row[order])
    np.testing.assert_array_equal(ci2.cpu().numpy(), coo.col[order])
    np.testing.assert_array_equal(vv2.cpu().numpy(), coo.data[order].astype(t))


@pytest.mark.parametrize("dt", ["f64", "f32"])
@pytest.mark.parametrize("major", ["row", "col"])
def test_csr2dense_and_dense2csr(ctrl, dt, major):
    dtype, t = DT[dt], NPT[dt]
    mj = L.rowMajor if major == "row" else L.columnMajor
    rows, cols = 2500, 90
    M = random_csr(rows, cols, 0.05, 5, empty_every=5)
    A = api.CsrMatrix.from_numpy(M.indptr, M.indices, M.data, num_cols=cols, dtype=dtype)
    ld = (cols if mj == L.rowMajor else rows) + 3
    buf = torch.full(((rows if mj == L.rowMajor else cols) * ld,), 7.0, dtype=dtype, device="cuda")
    d = dense_struct(buf, rows, cols, ld, mj)
    fn = api.lib().clsparseDcsr2dense if dt == "f64" else api.lib().clsparseScsr2dense
    assert fn(C.byref(A.s), C.byref(d), ctrl.handle) == 0
    full = buf.cpu().numpy()
    dense = full.reshape(rows, ld)[:, :cols] if mj == L.rowMajor else full.reshape(cols, ld)[:, :rows].T
    np.testing.assert_array_equal(dense, M.toarray().astype(t))
    # padding untouched
    pad = full.reshape(-1, ld)[:, -3:]
    assert np.all(pad == 7.0)
    # back to CSR
    out = api.CsrMatrix(torch.zeros(rows + 1, dtype=torch.int32, device="cuda"),
                        torch.zeros(rows * cols, dtype=torch.int32, device="cuda"),
                        torch.zeros(rows * cols, dtype=dtype, device="cuda"), cols)
    fn2 = api.lib().clsparseDdense2csr if dt == "f64" else api.lib().clsparseSdense2csr
    assert fn2(C.byref(d), C.byref(out.s), ctrl.handle) == 0
    assert (out.s.num_rows, out.s.num_cols, out.s.num_nonzeros) == (rows, cols, M.nnz)
    np.testing.assert_array_equal(out.row_ptr.cpu().numpy(), M.indptr)
    np.testing.assert_array_equal(out.col.cpu().numpy()[: M.nnz], M.indices)
    np.testing.assert_array_equal(out.val.cpu().numpy()[: M.nnz], M.data.astype(t))


def test_dense2csr_all_zero_and_reductions_after(ctrl):
    """An all-zero dense matrix gives an empty CSR, and the shared reduction
    scratch still works afterwards."""
    buf = torch.zeros(1500 * 4, dtype=torch.float64, device="cuda")
    d = dense_struct(buf, 1500, 4, 4, L.rowMajor)
    out = api.CsrMatrix(torch.zeros(1501, dtype=torch.int32, device="cuda"),
                        torch.zeros(8, dtype=torch.int32, device="cuda"),
                        torch.zeros(8, dtype=torch.float64, device="cuda"), 4)
    assert api.lib().clsparseDdense2csr(C.byref(d), C.byref(out.s), ctrl.handle) == 0
    assert out.s.num_nonzeros == 0 and int(out.row_ptr.abs().sum()) == 0
    x = torch.arange(1, 5001, dtype=torch.float64, device="cuda")
    r = torch.zeros(1, dtype=torch.float64, device="cuda")
    api.blas1("cldenseDreduce", ("s", r), x, ctrl=ctrl)
    assert float(r) == 5000 * 5001 / 2


@pytest.mark.parametrize("dt", ["f64", "f32"])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-2.0, 0.5)])
def test_coomv_sorted_with_duplicates(ctrl, dt, alpha, beta):
    dtype, t = DT[dt], NPT[dt]
    rng = np.random.default_rng(11)
    M = random_csr(4001, 3000, 0.004, 8).tocoo()  # a row count that leaves idle groups
    # duplicate some entries (kept, summed by the product) and keep row order
    dup = rng.choice(M.nnz, 300, replace=False)
    rows = np.concatenate([M.row, M.row[dup]])
    cols = np.concatenate([M.col, M.col[dup]])
    vals = np.concatenate([M.data, rng.uniform(-1, 1, 300)])
    order = np.argsort(rows, kind="stable")
    rows, cols, vals = rows[order], cols[order], vals[order]
    # the struct holds raw pointers: keep the tensors alive
    keep = (torch.tensor(rows.astype(np.int32), device="cuda"), torch.tensor(cols.astype(np.int32), device="cuda"),
            torch.tensor(vals.astype(t), device="cuda"))
    cm = coo_struct(*keep, 4001, 3000)
    x = rng.uniform(-1, 1, 3000)
    y0 = rng.uniform(-1, 1, 4001)
    xt = torch.tensor(x.astype(t), device="cuda")
    yt = torch.tensor(y0.astype(t), device="cuda")
    a = torch.tensor([alpha], dtype=dtype, device="cuda")
    b = torch.tensor([beta], dtype=dtype, device="cuda")
    fn = api.lib().clsparseDcoomv if dt == "f64" else api.lib().clsparseScoomv
    assert fn(C.byref(api.scalar(a)), C.byref(cm), C.byref(api.vector(xt)), C.byref(api.scalar(b)),
              C.byref(api.vector(yt)), ctrl.handle) == 0
    A = sp.csr_matrix((vals.astype(t).astype(np.float64), (rows, cols)), shape=(4001, 3000))
    ref = alpha * (A @ x.astype(t).astype(np.float64)) + beta * y0.astype(t).astype(np.float64)
    scale = abs(alpha) * (abs(A) @ abs(x.astype(t).astype(np.float64))) + abs(beta * y0) + 1e-300
    tol = 1e-12 if dt == "f64" else 1e-5
    assert np.max(np.abs(yt.cpu().numpy() - ref) / scale) <= 10 * tol
