"""The oracle and the library's host binning against the reference's own
row-block words (tests/golden/rowblocks.npz, made by the reference's
ComputeRowBlocks compiled from its sources), and the oracle's arithmetic
against independent dense references. CPU only."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "rowblocks.npz"


def _cases():
    d = np.load(GOLD)
    names = sorted({k.split("__")[0] for k in d.files})
    return [(n, d[f"{n}__rp"], d[f"{n}__words"], d[f"{n}__size"]) for n in names]


@pytest.mark.parametrize("name,rp,words,size", _cases(), ids=[c[0] for c in _cases()])
def test_oracle_row_blocks_match_reference(orc, name, rp, words, size):
    w, s, dry = orc.row_blocks(rp)
    assert s == size[0] and dry == size[1]
    np.testing.assert_array_equal(w, words)


@pytest.mark.parametrize("name,rp,words,size", _cases(), ids=[c[0] for c in _cases()])
def test_library_host_binning_matches_reference(libso, name, rp, words, size):
    from clsparse_b200 import _lib as L
    n = len(rp) - 1
    rp = np.ascontiguousarray(rp, dtype=np.uint32)
    rbs = L.clsparseIdx_t()
    p = rp.ctypes.data_as(C.POINTER(L.clsparseIdx_t))
    assert libso.clsparseB200ComputeRowBlocksHost(p, n, None, 0, C.byref(rbs)) == 0
    assert rbs.value == size[1]
    out = np.zeros(size[1] // 2 + 1, dtype=np.uint64)
    assert libso.clsparseB200ComputeRowBlocksHost(p, n, out.ctypes.data_as(C.POINTER(L.cl_ulong)),
                                                  len(out), C.byref(rbs)) == 0
    assert rbs.value == size[0]
    np.testing.assert_array_equal(out[: size[0] // 2], words)


GOLD_SHAPES = Path(__file__).resolve().parent / "golden" / "rowblocks_shapes.npz"


def _shape_cases():
    rps = np.load(GOLD)
    d = np.load(GOLD_SHAPES)
    out = []
    for key in sorted(k for k in d.files if k.endswith("__words")):
        tag, name, _ = key.split("__")
        shape = tuple(int(v) for v in tag.split("x"))
        out.append((f"{tag}-{name}", shape, rps[f"{name}__rp"], d[key], d[f"{tag}__{name}__size"]))
    return out


@pytest.mark.parametrize("cid,shape,rp,words,size", _shape_cases(), ids=[c[0] for c in _shape_cases()])
def test_oracle_row_blocks_shapes_match_reference(orc, cid, shape, rp, words, size):
    """Non-default row-block shapes (the autotuner's knobs) against the
    reference's ComputeRowBlocks called with the same shape."""
    w, s, dry = orc.row_blocks(rp, shape)
    assert s == size[0] and dry == size[1]
    np.testing.assert_array_equal(w, words)


def test_probe_case_layout():
    """Rows {3,3,2000,4}: one stream block of 2 rows (128 threads/row), one
    vector row, one trailing row -- the layout of csr-meta.hpp:70-90."""
    d = np.load(GOLD)
    w = d["probe_3_3_2000_4__words"]
    assert [int(x) for x in w] == [128, 2 << 32, 3 << 32, 4 << 32]


def test_oracle_against_live_reference_random(orc):
    """Random row-length patterns, oracle vs the reference build (where present)."""
    if orc.ref_lib() is None:
        pytest.skip("reference build absent")
    rng = np.random.default_rng(11)
    for _ in range(50):
        n = int(rng.integers(0, 2000))
        lens = rng.choice([0, 1, 5, 31, 33, 129, 500, 1024, 1025, 3100, 9000], n)
        rp = np.zeros(n + 1, np.uint32)
        rp[1:] = np.cumsum(lens)
        a = orc.row_blocks(rp)
        b = orc.ref_row_blocks(rp)
        assert a[1] == b[1] and a[2] == b[2]
        np.testing.assert_array_equal(a[0], b[0])


def _dense(rp, col, val, n, m):
    A = np.zeros((n, m))
    for r in range(n):
        A[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
    return A


def test_oracle_spmv_matches_dense(orc):
    from clsparse_b200 import matgen
    rp, col, val = matgen.random_lengths([0, 3, 17, 1, 0, 40, 2], 50, seed=3)
    A = _dense(rp, col, val, 7, 50)
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, 50)
    y = rng.uniform(-1, 1, 7)
    for alpha, beta in ((1.0, 0.0), (2.5, 1.0), (-0.5, 3.0)):
        ref = alpha * A @ x + beta * y
        np.testing.assert_allclose(orc.dcsrmv(rp, col, val, alpha, x, beta, y), ref, rtol=1e-13, atol=1e-14)
        ys = orc.scsrmv(rp, col, val.astype(np.float32), alpha, x.astype(np.float32), beta,
                        y.astype(np.float32))
        np.testing.assert_allclose(ys, ref, rtol=1e-4, atol=1e-5)


def test_oracle_beta_zero_ignores_nan(orc):
    from clsparse_b200 import matgen
    rp, col, val = matgen.random_lengths([2, 3], 5, seed=1)
    y = np.array([np.nan, np.inf])
    out = orc.dcsrmv(rp, col, val, 1.0, np.ones(5), 0.0, y)
    assert np.all(np.isfinite(out))


def test_oracle_cg_converges_like_scipy(orc):
    from clsparse_b200 import matgen
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    rp, col, val = matgen.poisson2d(20)
    n = len(rp) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n)
    x, info = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 1000, 1e-10, 0.0)
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-8
    assert info.currentResidual <= 1e-10 and info.nIters > 10


def test_oracle_bicgstab_solves_nonsymmetric(orc):
    from clsparse_b200 import matgen
    import scipy.sparse as sp
    rp, col, val = matgen.random_spd(300, seed=4)
    val = val * np.random.default_rng(2).uniform(0.9, 1.1, len(val))  # break symmetry
    n = len(rp) - 1
    b = np.ones(n)
    for pre in (0, 1):
        x, info = orc.solve("bicgstab", np.float64, rp, col, val, np.zeros(n), b, pre, 500, 1e-12, 0.0)
        A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
        assert np.linalg.norm(A @ x - b, 1) / np.linalg.norm(b, 1) < 1e-10


def test_oracle_cg_iteration_bookkeeping(orc):
    """maxIters stops after maxIters+1 updates and reports nIters = maxIters,
    as conjugate-gradients.hpp:162-224 does."""
    from clsparse_b200 import matgen
    rp, col, val = matgen.poisson2d(30)
    n = len(rp) - 1
    b = np.ones(n)
    _, info = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 5, 1e-30, 0.0)
    assert info.nIters == 5
    _, info0 = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), np.zeros(n), 1, 5, 1e-3, 0.0)
    assert info0.zero_b == 1 and info0.nIters == 0 and info0.relTol == 0.0
