"""Parity of clsparse{S,D}csrmv (through the C ABI) with the CPU oracle.

The oracle is the reference test suite's host SpMV (src/tests/test-blas2.cpp:
146-163 for FP32 with double accumulation, :231-252 for FP64 with compensated
summation). Tolerances are the path's stated bars, relative to the row's
absolute scale sum_j |alpha a_ij x_j| + |beta y_i| (robust to cancellation)
and as a norm-wise relative error:
    FP64: 1e-12        FP32: 1e-5
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from clsparse_b200 import api, matgen

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.float32: 1e-5}
NP = {torch.float64: np.float64, torch.float32: np.float32}


def gpu_spmv(ctrl, rp, col, val, x, y0, alpha, beta, dtype, meta=True, ncols=None):
    ncols = len(x) if ncols is None else ncols
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=ncols, dtype=dtype)
    if meta:
        A.create_meta(ctrl)
    xt = torch.tensor(np.asarray(x), dtype=dtype, device="cuda")
    yt = torch.tensor(np.asarray(y0), dtype=dtype, device="cuda")
    at = torch.tensor([alpha], dtype=dtype, device="cuda")
    bt = torch.tensor([beta], dtype=dtype, device="cuda")
    api.csrmv(at, A, xt, bt, yt, ctrl)
    return yt.cpu().numpy(), A


def oracle_spmv(orc, rp, col, val, x, y0, alpha, beta, dtype):
    if dtype == torch.float64:
        return orc.dcsrmv(rp, col, val, alpha, x, beta, y0)
    return orc.scsrmv(rp, col, np.asarray(val, np.float32), np.float32(alpha), np.asarray(x, np.float32),
                      np.float32(beta), np.asarray(y0, np.float32)).astype(np.float64)


def assert_parity(orc, rp, col, val, x, y0, alpha, beta, out, dtype):
    t = NP[dtype]
    valc = np.asarray(val, t).astype(np.float64)
    xc = np.asarray(x, t).astype(np.float64)
    yc = np.asarray(y0, t).astype(np.float64)
    ref = oracle_spmv(orc, rp, col, val, x, y0, alpha, beta, dtype)
    scale = orc.dcsrmv_absscale(rp, col, valc, float(t(alpha)), xc, float(t(beta)), yc)
    err = np.abs(out.astype(np.float64) - ref)
    tol = TOL[dtype]
    tiny = np.finfo(t).tiny
    bad = err > tol * scale + tiny
    assert not bad.any(), f"{bad.sum()} rows off; worst {(err / (scale + tiny)).max():.3e}"
    if np.linalg.norm(ref) > 0:
        assert np.linalg.norm(err) <= tol * max(np.linalg.norm(ref), np.linalg.norm(scale) * 1e-3)


def vecs(n_rows, n_cols, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, n_cols), rng.uniform(-1, 1, n_rows)


EDGE_LENGTHS = {
    "threshold_rows": [0, 1, 31, 32, 33, 127, 128, 129, 1023, 1024, 1025, 3072, 3073, 6145, 2, 0, 5],
    "many_short": list(np.random.default_rng(1).integers(0, 6, 4000)),
    "all_empty": [0] * 777,
    "one_row": [17],
    "one_long_row": [50_000],
    "long_rows_between_short": [3] * 100 + [9000, 7000] + [2] * 500 + [20000] + [1] * 10,
    "lognormal": list(np.maximum(1, np.rint(np.exp(np.random.default_rng(2).normal(2.5, 1.2, 5000))))
                      .astype(int)),
    "stream_runs": list(np.random.default_rng(3).integers(100, 300, 800)),
}


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("meta", [True, False], ids=["adaptive", "vector"])
@pytest.mark.parametrize("case", sorted(EDGE_LENGTHS))
def test_spmv_edge_matrices(ctrl, orc, dtype, meta, case):
    lens = EDGE_LENGTHS[case]
    ncols = max(60_000, 1)
    rp, col, val = matgen.random_lengths(lens, ncols, seed=len(lens))
    x, y0 = vecs(len(lens), ncols, 5)
    for alpha, beta in ((1.0, 0.0), (2.5, -1.5), (-0.75, 1.0)):
        out, _ = gpu_spmv(ctrl, rp, col, val, x, y0, alpha, beta, dtype, meta)
        assert_parity(orc, rp, col, val, x, y0, alpha, beta, out, dtype)


SHORT_ROW_CASES = {
    "poisson": None,
    "lengths_0_to_16": list(np.random.default_rng(7).integers(0, 17, 30_000)),
    "sixteen_then_seventeen": [16] * 3000 + [17] + [4] * 3000,  # longest row 17: row-block kernel
    "all_empty": [0] * 1000,
}


@pytest.mark.parametrize("ext", [False, True], ids=["plain", "extended"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("case", sorted(SHORT_ROW_CASES))
def test_spmv_short_rows_both_kernels(ctrl, orc, monkeypatch, dtype, case, ext):
    """Matrices whose rows are all at most 16 long run one thread per row; the
    same products through the row-block kernel (CLSPARSE_B200_SHORT_ROWS=0) and
    both against the oracle."""
    if case == "poisson":
        rp, col, val = matgen.poisson2d(96)
        ncols = len(rp) - 1
    else:
        ncols = 20_000
        rp, col, val = matgen.random_lengths(SHORT_ROW_CASES[case], ncols, seed=3)
    n = len(rp) - 1
    x, y0 = vecs(n, ncols, 8)
    ctrl.enable_extended_precision(ext)
    outs = []
    for mode in ("1", "0"):
        monkeypatch.setenv("CLSPARSE_B200_SHORT_ROWS", mode)
        for alpha, beta in ((1.0, 0.0), (-0.75, 1.25)):
            out, _ = gpu_spmv(ctrl, rp, col, val, x, y0, alpha, beta, dtype, meta=True, ncols=ncols)
            assert_parity(orc, rp, col, val, x, y0, alpha, beta, out, dtype)
            outs.append(out)
    ctrl.enable_extended_precision(False)
    if case == "sixteen_then_seventeen":  # both settings ran the row-block kernel
        np.testing.assert_array_equal(outs[0], outs[2])
        np.testing.assert_array_equal(outs[1], outs[3])


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_spmv_extended_precision(ctrl, orc, dtype):
    ctrl.enable_extended_precision(True)
    rp, col, val = matgen.irregular(20_000, n_dense=5, dense_len=9_000, seed=9)
    x, y0 = vecs(20_000, 20_000, 6)
    out, _ = gpu_spmv(ctrl, rp, col, val, x, y0, 1.0, 0.5, dtype)
    assert_parity(orc, rp, col, val, x, y0, 1.0, 0.5, out, dtype)


def test_meta_words_equal_reference_binning(ctrl, orc):
    rp, col, val = matgen.irregular(30_000, n_dense=7, dense_len=12_000, seed=4)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    size = A.meta_size(ctrl)
    A.create_meta(ctrl)
    words, s, dry = orc.row_blocks(rp)
    assert size == dry
    assert A.meta_size(ctrl) == s
    np.testing.assert_array_equal(A.row_blocks(), words)
    if orc.ref_lib() is not None:
        np.testing.assert_array_equal(A.row_blocks(), orc.ref_row_blocks(rp)[0])


TUNED_SHAPES = [(512, 1, 1, 128), (512, 8, 4, 128), (2048, 3, 1, 256), (2048, 1, 4, 128), (1024, 8, 2, 256),
                (1024, 3, 1, 256)]


@pytest.mark.parametrize("shape", TUNED_SHAPES, ids=["x".join(map(str, s)) for s in TUNED_SHAPES])
def test_tuned_meta_words_match_reference(ctrl, shape):
    """clsparseB200CsrMetaCreateTuned's words against the reference's
    ComputeRowBlocks with the same shape (tests/golden/rowblocks_shapes.npz)."""
    from pathlib import Path
    gold = Path(__file__).resolve().parent / "golden"
    rps = np.load(gold / "rowblocks.npz")
    d = np.load(gold / "rowblocks_shapes.npz")
    tag = "x".join(str(v) for v in shape[:3])
    names = sorted({k.split("__")[1] for k in d.files if k.startswith(tag + "__")})
    if not names:
        pytest.skip("shape not in the golden set")
    for name in names:
        rp = rps[f"{name}__rp"]
        if len(rp) < 2 or int(rp[-1]) == 0:
            continue
        n = len(rp) - 1
        col = np.zeros(int(rp[-1]), dtype=np.uint32)
        A = api.CsrMatrix.from_numpy(rp, col, np.ones(int(rp[-1])), num_cols=1)
        A.create_meta(ctrl, shape=shape)
        np.testing.assert_array_equal(A.row_blocks(), d[f"{tag}__{name}__words"], err_msg=name)
        assert n == A.num_rows


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("shape", TUNED_SHAPES, ids=["x".join(map(str, s)) for s in TUNED_SHAPES])
@pytest.mark.parametrize("case", ["threshold_rows", "long_rows_between_short", "lognormal", "many_short"])
def test_spmv_tuned_shapes(ctrl, orc, dtype, shape, case):
    """SpMV parity for every row-block shape the autotuner may pick."""
    lens = EDGE_LENGTHS[case]
    ncols = 60_000
    rp, col, val = matgen.random_lengths(lens, ncols, seed=len(lens))
    x, y0 = vecs(len(lens), ncols, 5)
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=ncols, dtype=dtype)
    A.create_meta(ctrl, shape=shape)
    xt = torch.tensor(x, dtype=dtype, device="cuda")
    for alpha, beta in ((1.0, 0.0), (2.5, -1.5)):
        yt = torch.tensor(y0, dtype=dtype, device="cuda")
        api.csrmv(torch.tensor([alpha], dtype=dtype, device="cuda"), A, xt,
                  torch.tensor([beta], dtype=dtype, device="cuda"), yt, ctrl)
        assert_parity(orc, rp, col, val, x, y0, alpha, beta, yt.cpu().numpy(), dtype)


def test_tuned_meta_rejects_bad_shapes(ctrl):
    rp, col, val = matgen.poisson2d(8)
    A = api.CsrMatrix.from_numpy(rp, col, val)
    for bad in ((256, 3, 1, 128), (512, 3, 1, 256), (1024, 0, 1, 128), (1024, 3, 0, 128), (1024, 3, 1, 64)):
        with pytest.raises(api.ClsparseError):
            A.create_meta(ctrl, shape=bad)


def test_spmv_beta_zero_does_not_read_y(ctrl):
    rp, col, val = matgen.random_lengths([3, 0, 5000, 40, 12000, 1], 20_000, seed=2)
    for meta in (True, False):
        y0 = np.full(6, np.nan)
        out, _ = gpu_spmv(ctrl, rp, col, val, np.ones(20_000), y0, 1.0, 0.0, torch.float64, meta)
        assert np.all(np.isfinite(out))


def test_spmv_offsets_and_rectangular(ctrl, orc):
    rng = np.random.default_rng(8)
    rp, col, val = matgen.random_lengths(rng.integers(0, 50, 3000), 777, seed=8)
    x, y0 = vecs(3000, 777, 9)
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=777)
    A.create_meta(ctrl)
    xt = torch.zeros(777 + 13, dtype=torch.float64, device="cuda")
    xt[13:] = torch.tensor(x, device="cuda")
    yt = torch.zeros(3000 + 5, dtype=torch.float64, device="cuda")
    yt[5:] = torch.tensor(y0, device="cuda")
    one = torch.tensor([0.0, 1.0], dtype=torch.float64, device="cuda")
    A_vec = api.vector
    from clsparse_b200 import _lib as L
    import ctypes as C
    al = L.clsparseScalar(C.c_void_p(one.data_ptr()), 1)
    be = L.clsparseScalar(C.c_void_p(one.data_ptr()), 1)
    st = L.load().clsparseDcsrmv(C.byref(al), C.byref(A.s), C.byref(A_vec(xt, 13)), C.byref(be),
                                 C.byref(A_vec(yt, 5)), ctrl.handle)
    assert st == 0
    assert_parity(orc, rp, col, val, x, y0, 1.0, 1.0, yt[5:].cpu().numpy(), torch.float64)
    assert float(yt[:5].abs().sum()) == 0.0


def test_spmv_deterministic(ctrl):
    rp, col, val = matgen.irregular(50_000, n_dense=10, dense_len=20_000, seed=12)
    x, y0 = vecs(50_000, 50_000, 1)
    a, _ = gpu_spmv(ctrl, rp, col, val, x, y0, 1.0, 1.0, torch.float64)
    b, _ = gpu_spmv(ctrl, rp, col, val, x, y0, 1.0, 1.0, torch.float64)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_spmv_size_errors(ctrl):
    rp, col, val = matgen.random_lengths([1, 2], 4, seed=0)
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=4)
    x = torch.zeros(3, dtype=torch.float64, device="cuda")
    y = torch.zeros(2, dtype=torch.float64, device="cuda")
    s = torch.ones(1, dtype=torch.float64, device="cuda")
    with pytest.raises(api.ClsparseError) as e:
        api.csrmv(s, A, x, s, y, ctrl)
    assert e.value.status == -1021  # clsparseInvalidSize


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_spmv_irregular_full_size(ctrl, orc, dtype):
    """The 2M-row irregular workload (log-normal rows + 50 rows of 200k), full
    parity against the oracle plus linearity A(x1+x2) = Ax1 + Ax2."""
    rp, col, val = matgen.irregular(2_000_000, seed=7)
    x, y0 = vecs(2_000_000, 2_000_000, 3)
    out, A = gpu_spmv(ctrl, rp, col, val, x, y0, 1.0, 0.0, dtype)
    assert_parity(orc, rp, col, val, x, y0, 1.0, 0.0, out, dtype)
    x2 = np.random.default_rng(4).uniform(-1, 1, 2_000_000)
    t = NP[dtype]
    xa = torch.tensor(np.asarray(x, t), device="cuda")
    xb = torch.tensor(np.asarray(x2, t), device="cuda")
    one = torch.ones(1, dtype=dtype, device="cuda")
    zero = torch.zeros(1, dtype=dtype, device="cuda")
    ya = torch.zeros(2_000_000, dtype=dtype, device="cuda")
    yb = torch.zeros_like(ya)
    yab = torch.zeros_like(ya)
    api.csrmv(one, A, xa, zero, ya, ctrl)
    api.csrmv(one, A, xb, zero, yb, ctrl)
    api.csrmv(one, A, xa + xb, zero, yab, ctrl)
    lin = (yab - ya - yb).abs().double().cpu().numpy()
    valc = np.asarray(val, t).astype(np.float64)
    s1 = orc.dcsrmv_absscale(rp, col, valc, 1.0, np.asarray(x, t).astype(np.float64), 0.0, y0)
    s2 = orc.dcsrmv_absscale(rp, col, valc, 1.0, np.asarray(x2, t).astype(np.float64), 0.0, y0)
    assert np.all(lin <= 4 * TOL[dtype] * (s1 + s2) + np.finfo(t).tiny)


@pytest.mark.parametrize("where", ["first", "middle", "last"])
def test_meta_create_rejects_out_of_range_column(ctrl, where):
    """clsparseCsrMetaCreate checks the structure before any kernel trusts
    it (the reference only checks buffer sizes, in debug builds:
    src/library/internal/clsparse-validate.cpp:69-133): a column index >=
    num_cols anywhere -- in the unaligned head, the vectorised body or the
    tail of the index array -- is clsparseInvalidValue, and nothing is
    attached to the matrix."""
    from clsparse_b200 import _lib as L
    rp, col, val = matgen.random_lengths(np.full(500, 7), 1000, seed=3)
    col = col.copy()
    pos = {"first": 0, "middle": len(col) // 2 + 1, "last": len(col) - 1}[where]
    col[pos] = 1000
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=1000)
    with pytest.raises(api.ClsparseError) as e:
        A.create_meta(ctrl)
    assert e.value.status == L.clsparseInvalidValue
    assert not A.s.meta
    col[pos] = 999
    B = api.CsrMatrix.from_numpy(rp, col, val, num_cols=1000)
    B.create_meta(ctrl)
    assert B.s.meta


def test_meta_create_rejects_bad_row_pointers(ctrl):
    from clsparse_b200 import _lib as L
    rp, col, val = matgen.random_lengths([3, 4, 5], 10, seed=1)
    bad = rp.copy()
    bad[1], bad[2] = bad[2], bad[1]  # not monotone
    A = api.CsrMatrix.from_numpy(bad, col, val, num_cols=10)
    with pytest.raises(api.ClsparseError) as e:
        A.create_meta(ctrl)
    assert e.value.status == L.clsparseInvalidValue
    # row pointers spanning fewer entries than num_nonzeros
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=10)
    A.s.num_nonzeros = len(col) - 1
    with pytest.raises(api.ClsparseError) as e:
        A.create_meta(ctrl)
    assert e.value.status == L.clsparseInvalidValue
    # the same arrays with consistent sizes pass
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=10)
    A.create_meta(ctrl)
