"""Matrix Market input (clsparseHeaderfromFile, clsparse{S,D}{Csr,Coo}MatrixfromFile,
clsparseB200ReadMatrixMarketHost) against the reader rules of the reference
(src/library/io/mm-reader.cpp): coordinate real/integer/pattern files,
symmetric mirroring, explicit zeros dropped unless asked for, entries sorted by
(row, column) with duplicates kept, '.mtx' paths only. Host parts run on CPU;
the device loaders are gpu-marked."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from clsparse_b200 import _lib as L
from clsparse_b200 import api


def write(path, banner, rows, cols, entries, comments=("% a comment",)):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix {banner}\n")
        for c in comments:
            f.write(c + "\n")
        f.write(f"{rows} {cols} {len(entries)}\n")
        for e in entries:
            f.write(" ".join(str(v) for v in e) + "\n")
    return path


def expected_csr(rows, entries, symmetric=False, keep_zeros=False):
    coo = []
    for e in entries:
        i, j = int(e[0]) - 1, int(e[1]) - 1
        v = float(e[2]) if len(e) > 2 else None
        if v is not None and v == 0.0 and not keep_zeros:
            continue
        coo.append((i, j, v))
        if symmetric and i != j:
            coo.append((j, i, v))
    coo.sort(key=lambda t: (t[0], t[1]))  # stable: duplicates keep file order
    rp = np.zeros(rows + 1, dtype=np.int64)
    for i, _, _ in coo:
        rp[i + 1] += 1
    return np.cumsum(rp), np.array([c[1] for c in coo]), [c[2] for c in coo]


def header(libso, path):
    nnz, r, c = L.clsparseIdx_t(), L.clsparseIdx_t(), L.clsparseIdx_t()
    st = libso.clsparseHeaderfromFile(C.byref(nnz), C.byref(r), C.byref(c), str(path).encode())
    return st, nnz.value, r.value, c.value


GENERAL = [(3, 1, 2.5), (1, 2, -1.0), (2, 2, 0.0), (1, 1, 4.0), (3, 3, 1e-300), (1, 2, 7.0), (4, 4, -3.25)]


@pytest.mark.parametrize("keep", [False, True])
def test_general_real_sorted_zeros_and_duplicates(libso, tmp_path, keep):
    p = write(tmp_path / "g.mtx", "coordinate real general", 4, 5, GENERAL)
    rp, col, val, ncols = api.read_mtx_host(p, keep)
    erp, ecol, evals = expected_csr(4, GENERAL, keep_zeros=keep)
    assert ncols == 5
    np.testing.assert_array_equal(rp, erp)
    np.testing.assert_array_equal(col, ecol)
    np.testing.assert_array_equal(val, evals)
    st, nnz, r, c = header(libso, p)
    assert st == 0 and (nnz, r, c) == (len(GENERAL), 4, 5)


def test_symmetric_is_mirrored(libso, tmp_path):
    ent = [(1, 1, 2.0), (2, 1, -1.0), (2, 2, 2.0), (3, 2, -1.0), (3, 3, 2.0), (3, 1, 0.5)]
    p = write(tmp_path / "s.mtx", "coordinate real symmetric", 3, 3, ent)
    rp, col, val, _ = api.read_mtx_host(p)
    M = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(3, 3)).toarray()
    np.testing.assert_array_equal(M, M.T)
    assert M[0, 2] == 0.5 and M[2, 0] == 0.5 and len(val) == 9
    st, nnz, _, _ = header(libso, p)
    assert st == 0 and nnz == 12  # twice the stored count, as the reference reports


def test_integer_and_pattern(tmp_path):
    p = write(tmp_path / "i.mtx", "coordinate integer general", 3, 3, [(1, 3, 7), (2, 1, -2), (3, 3, 0)])
    rp, col, val, _ = api.read_mtx_host(p)
    np.testing.assert_array_equal(val, [7.0, -2.0])
    np.testing.assert_array_equal(col, [2, 0])
    q = write(tmp_path / "p.mtx", "coordinate pattern general", 4, 4, [(1, 2), (4, 1), (2, 2), (3, 4)])
    rp1, col1, val1, _ = api.read_mtx_host(q)
    rp2, col2, val2, _ = api.read_mtx_host(q)
    np.testing.assert_array_equal(col1, [1, 1, 3, 0])
    np.testing.assert_array_equal(rp1, [0, 1, 2, 3, 4])
    assert np.all((val1 > 0) & (val1 < 5)) and np.array_equal(val1, val2)  # seeded: same values each load


def test_matches_scipy_on_random_matrix(tmp_path):
    A = sp.random(300, 200, density=0.03, random_state=5, format="coo")
    p = tmp_path / "r.mtx"
    scipy.io.mmwrite(str(p), A, precision=17)
    rp, col, val, ncols = api.read_mtx_host(p)
    B = A.tocsr()
    B.sort_indices()
    assert ncols == 200
    np.testing.assert_array_equal(rp, B.indptr)
    np.testing.assert_array_equal(col, B.indices)
    np.testing.assert_array_equal(val, B.data)


def test_errors(libso, tmp_path):
    good = write(tmp_path / "ok.mtx", "coordinate real general", 2, 2, [(1, 1, 1.0)])
    txt = tmp_path / "ok.txt"
    txt.write_text(good.read_text())
    assert header(libso, txt)[0] == L.clsparseInvalidFileFormat
    assert header(libso, tmp_path / "missing.mtx")[0] == L.clsparseInvalidFile
    arr = tmp_path / "a.mtx"
    arr.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    assert header(libso, arr)[0] == L.clsparseInvalidFile
    cpx = write(tmp_path / "c.mtx", "coordinate complex general", 2, 2, [(1, 1, 1.0, 0.5)])
    assert header(libso, cpx)[0] == L.clsparseInvalidFile
    oob = write(tmp_path / "o.mtx", "coordinate real general", 2, 2, [(3, 1, 1.0)])
    with pytest.raises(api.ClsparseError) as e:
        api.read_mtx_host(oob)
    assert e.value.status == L.clsparseInvalidFile
    short = tmp_path / "t.mtx"
    short.write_text("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1.0\n")
    with pytest.raises(api.ClsparseError):
        api.read_mtx_host(short)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype_name", ["f64", "f32"])
def test_device_csr_and_coo_from_file(ctrl, orc, tmp_path, dtype_name):
    import torch
    dtype = torch.float64 if dtype_name == "f64" else torch.float32
    A = sp.random(2000, 2000, density=0.004, random_state=9, format="coo") + sp.eye(2000)
    p = tmp_path / "d.mtx"
    scipy.io.mmwrite(str(p), A.tocoo(), precision=17)
    rp, col, val, _ = api.read_mtx_host(p)
    M = api.CsrMatrix.from_file(p, ctrl, dtype=dtype)
    np.testing.assert_array_equal(M.row_ptr.cpu().numpy().view(np.uint32), rp)
    np.testing.assert_array_equal(M.col.cpu().numpy().view(np.uint32), col)
    np.testing.assert_allclose(M.val.cpu().numpy(), val.astype(np.float32 if dtype == torch.float32 else np.float64))
    # the loaded matrix runs through the adaptive SpMV
    M.create_meta(ctrl)
    x = np.random.default_rng(1).uniform(-1, 1, 2000)
    y = torch.zeros(2000, dtype=dtype, device="cuda")
    api.csrmv(torch.ones(1, dtype=dtype, device="cuda"), M, torch.tensor(x, dtype=dtype, device="cuda"),
              torch.zeros(1, dtype=dtype, device="cuda"), y, ctrl)
    ref = orc.dcsrmv(rp, col, val, 1.0, x, 0.0, np.zeros(2000))
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    assert np.max(np.abs(y.cpu().numpy() - ref)) <= tol * np.max(np.abs(ref)) * 10
    # COO variant
    coo = L.clsparseCooMatrix()
    libso = api.lib()
    libso.clsparseInitCooMatrix(C.byref(coo))
    n = len(val)
    ri = torch.zeros(n, dtype=torch.int32, device="cuda")
    ci = torch.zeros(n, dtype=torch.int32, device="cuda")
    vv = torch.zeros(n, dtype=dtype, device="cuda")
    coo.values, coo.col_indices, coo.row_indices = vv.data_ptr(), ci.data_ptr(), ri.data_ptr()
    fn = libso.clsparseDCooMatrixfromFile if dtype == torch.float64 else libso.clsparseSCooMatrixfromFile
    assert fn(C.byref(coo), str(p).encode(), ctrl.handle, 0) == 0
    assert coo.num_nonzeros == n and coo.num_rows == 2000
    np.testing.assert_array_equal(ri.cpu().numpy(), np.repeat(np.arange(2000), np.diff(rp.astype(np.int64))))
    np.testing.assert_array_equal(ci.cpu().numpy().view(np.uint32), col)
