"""The learned factorized preconditioner on the GPU (clsparseB200Spai*):
forward, loss and gradients against the float64 CPU oracle, checkpoint
round trip, the solver it feeds, and what training gains over Jacobi."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from clsparse_b200 import _lib as L
from clsparse_b200 import api, learn, matgen
from oracle import gnn_oracle as go

pytestmark = pytest.mark.gpu


def _setup(ctrl, m=12, seed=4):
    rp, c, v = matgen.diffusion2d_grf(m, corr_len=0.2, sigma=1.5, seed=seed)
    A = api.CsrMatrix.from_numpy(rp, c, v)
    spai = api.Spai(7)
    spai.set_matrix(A, ctrl)
    return (rp, c, v), A, spai


def test_gpu_loss_and_gradient_match_oracle(ctrl):
    (rp, c, v), A, spai = _setup(ctrl)
    gr = go.Graph(rp, c, v)
    rng = np.random.default_rng(0)
    p = spai.params().astype(np.float64)
    probes = rng.normal(size=(2, gr.n))
    Lo, go_grad = go.loss_grad(p, gr, list(probes), 0.3)
    Lg, gg = spai.loss_grad(ctrl, torch.tensor(probes, dtype=torch.float32, device="cuda"), 0.3,
                            fp32_weights=True)
    assert abs(Lg - Lo) <= 1e-4 * max(1.0, abs(Lo)), (Lg, Lo)
    rel = np.linalg.norm(gg - go_grad) / np.linalg.norm(go_grad)
    assert rel <= 2e-3, rel
    spai.release()


def test_bf16_weights_close_to_fp32(ctrl):
    (rp, c, v), A, spai = _setup(ctrl, m=16, seed=5)
    L32, g32 = spai.loss_grad(ctrl, fp32_weights=True)
    L16, g16 = spai.loss_grad(ctrl, fp32_weights=False)
    assert abs(L16 - L32) <= 0.05 * max(1.0, abs(L32))
    assert np.dot(g16, g32) > 0.9 * np.linalg.norm(g16) * np.linalg.norm(g32)
    spai.release()


@pytest.mark.parametrize("m", [24, 300], ids=["576 rows", "90000 rows"])
def test_bf16_forward_matches_oracle(ctrl, m):
    """The BF16 inference pass (dense layers on tensor cores, BF16 weights and
    layer inputs, FP32 accumulation) against the oracle's restatement of the
    same roundings in FP64: the exported factor agrees to 2e-3 in norm (FP32
    activations may round to a neighbouring BF16 value where the oracle's FP64
    ones do not). 576 rows leave a partial 128-row tile; 90000 rows give
    every CTA of the persistent grid several tiles."""
    rp, c, v = matgen.diffusion2d_grf(m, corr_len=0.2, sigma=1.5, seed=8)
    A = api.CsrMatrix.from_numpy(rp, c, v)
    spai = api.Spai(11)
    spai.set_matrix(A, ctrl)
    spai.build(ctrl)
    _, _, G = spai.factor()
    gr = go.Graph(rp, c, v, with_blocks=False)
    g = G / gr.dinv[gr.Lcol]  # the network's output on the scaled operator
    p = spai.params().astype(np.float64)
    g16, _ = go.forward(p, gr, bf16=True)
    g64, _ = go.forward(p, gr, bf16=False)
    rel = np.linalg.norm(g - g16) / np.linalg.norm(g16)
    assert rel <= 2e-3, rel
    # the BF16 roundings themselves are visible: the test can tell the modes apart
    assert np.linalg.norm(g64 - g16) / np.linalg.norm(g16) > 5 * rel
    spai.release()


def test_factor_pattern_and_positive_diagonal(ctrl):
    (rp, c, v), A, spai = _setup(ctrl)
    spai.build(ctrl)
    frp, fcol, fval = spai.factor()
    Aop = sp.csr_matrix((v, c.astype(np.int64), rp.astype(np.int64)))
    T = sp.tril(Aop).tocsr()
    assert np.array_equal(frp.astype(np.int64), T.indptr) and np.array_equal(fcol.astype(np.int64), T.indices)
    n = len(rp) - 1
    G = sp.csr_matrix((fval, fcol.astype(np.int64), frp.astype(np.int64)), shape=(n, n))
    assert np.all(G.diagonal() > 0)
    M = (G.T @ G).toarray()
    assert np.linalg.eigvalsh(M).min() > 0
    spai.release()


def test_checkpoint_round_trip(ctrl, tmp_path):
    (rp, c, v), A, spai = _setup(ctrl)
    spai.train_step(ctrl, lr=1e-3)
    path = tmp_path / "net.bin"
    spai.save(path)
    other = api.Spai(99)
    other.load(path)
    assert np.array_equal(other.params(), spai.params())
    raw = bytearray(path.read_bytes())
    raw[40] ^= 0xFF
    path.write_bytes(bytes(raw))
    with pytest.raises(api.ClsparseError):
        other.load(path)
    other.release()
    spai.release()


def test_training_reduces_loss_and_beats_jacobi(ctrl):
    """The trained network's G^T G-PCG needs fewer iterations than Jacobi-CG
    on held-out matrices of the same family (the gain the network brings)."""
    spai, hist = learn.train(ctrl, sizes=(32, 48), seeds=range(4), steps=240, lr=3e-3)
    assert np.mean(hist[-20:]) < np.mean(hist[:8])
    ratios = []
    for seed in (101, 102):
        smp = learn.Sample(ctrl, 64, seed, with_probes=False)
        it_l, it_j = learn.pcg_iterations(ctrl, spai, smp)
        ratios.append(it_l / it_j)
    assert max(ratios) < 0.85, ratios
    spai.release()


@pytest.mark.parametrize("loop_mode", [0, 2], ids=["graph", "persistent"])
@pytest.mark.parametrize("inner", ["fp64", "fp32"])
def test_learned_solver_reaches_fp64_residual(ctrl, inner, loop_mode):
    ctrl.set_solver_loop_mode(loop_mode)
    spai, _ = learn.train(ctrl, sizes=(32,), seeds=range(2), steps=60, lr=3e-3)
    smp = learn.Sample(ctrl, 48, 7, with_probes=False)
    spai.set_matrix(smp.A, ctrl)
    spai.build(ctrl)
    n = smp.A.num_rows
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 100000, 1e-10, 0.0)
    info = api.cg_learned(x, smp.A, smp.b, sc, spai, ctrl, inner=inner, inner_tol=1e-3)
    sc.release()
    rp, c, v = smp.np
    A = sp.csr_matrix((v, c.astype(np.int64), rp.astype(np.int64)))
    b = smp.b.cpu().numpy()
    res = np.linalg.norm(b - A @ x.cpu().numpy()) / np.linalg.norm(b)
    assert res <= 2e-10, (res, info)
    spai.release()


def test_graph_cache_reuse_and_in_place_change(ctrl, monkeypatch):
    """Setting the network to a matrix it was set to before reuses the cached
    graph: the built factor is bitwise that of a network without the cache
    (CLSPARSE_B200_SPAI_CACHE=0). A matrix changed in place at the same
    addresses is rebuilt, not taken for the cached one."""
    mats = [matgen.diffusion2d_grf(20, corr_len=0.2, sigma=1.5, seed=s) for s in (31, 32)]
    As = [api.CsrMatrix.from_numpy(*m) for m in mats]

    def factors(seq):
        spai = api.Spai(5)
        out = []
        for k in seq:
            spai.set_matrix(As[k], ctrl)
            spai.build(ctrl)
            out.append(spai.factor()[2].copy())
        spai.release()
        return out

    seq = [0, 1, 0, 1, 0]
    cached = factors(seq)
    monkeypatch.setenv("CLSPARSE_B200_SPAI_CACHE", "0")
    fresh = factors(seq)
    monkeypatch.delenv("CLSPARSE_B200_SPAI_CACHE")
    for a, b in zip(cached, fresh):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(cached[0], cached[2])
    # change A0's values in place (same device buffers): the factor must follow
    spai = api.Spai(5)
    spai.set_matrix(As[0], ctrl)
    spai.build(ctrl)
    before = spai.factor()[2].copy()
    spai.set_matrix(As[1], ctrl)
    As[0].val.mul_(2.0)
    spai.set_matrix(As[0], ctrl)
    spai.build(ctrl)
    after = spai.factor()[2]
    ref = api.Spai(5)
    monkeypatch.setenv("CLSPARSE_B200_SPAI_CACHE", "0")
    ref.set_matrix(As[0], ctrl)
    ref.build(ctrl)
    np.testing.assert_array_equal(after, ref.factor()[2])
    assert not np.array_equal(after, before)
    spai.release()
    ref.release()


def test_training_same_with_and_without_graph_cache(ctrl, monkeypatch):
    """Training cycles through its matrices; the cached graphs give the same
    loss history, bit for bit, as rebuilding every step."""
    s1, h1 = learn.train(ctrl, sizes=(24,), seeds=range(3), steps=12, lr=3e-3)
    monkeypatch.setenv("CLSPARSE_B200_SPAI_CACHE", "0")
    s0, h0 = learn.train(ctrl, sizes=(24,), seeds=range(3), steps=12, lr=3e-3)
    s1.release()
    s0.release()
    assert h1 == h0


def laplacian27(m, seed=0):
    """3D 27-point operator on an m^3 grid: every neighbour at Chebyshev
    distance 1 couples with a positive random weight, the diagonal is the sum
    of the row's weights plus a margin (SPD, 14 entries per row of tril(A))."""
    n = m ** 3
    idx = np.arange(n).reshape(m, m, m)
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dz, dy, dx) == (0, 0, 0):
                    continue
                src = idx[max(0, -dz):m - max(0, dz), max(0, -dy):m - max(0, dy), max(0, -dx):m - max(0, dx)]
                dst = idx[max(0, dz):m - max(0, -dz), max(0, dy):m - max(0, -dy), max(0, dx):m - max(0, -dx)]
                rows.append(src.ravel())
                cols.append(dst.ravel())
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    lo = np.minimum(r, c)
    hi = np.maximum(r, c)
    w = rng.uniform(0.5, 1.5, len(r))
    key = lo.astype(np.int64) * n + hi
    _, first = np.unique(key, return_index=True)
    wsym = dict(zip(key[first].tolist(), w[first].tolist()))
    vals = -np.array([wsym[k] for k in key.tolist()])
    off = sp.csr_matrix((vals, (r, c)), shape=(n, n))
    d = -np.asarray(off.sum(axis=1)).ravel() + 0.05
    M = (off + sp.diags(d)).tocsr()
    M.sort_indices()
    return M.indptr.astype(np.uint32), M.indices.astype(np.uint32), M.data


def test_27_point_stencil_trains_builds_and_solves(ctrl):
    """Rows of tril(A) with 14 entries: the device graph build takes them, the
    network trains on them (local blocks of 14 x 14), and the learned solve
    reaches the FP64 residual."""
    rp, col, val = laplacian27(12, seed=3)
    n = len(rp) - 1
    assert max(np.diff(sp.tril(sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)))).tocsr().indptr)) == 14
    A = api.CsrMatrix.from_numpy(rp, col, val)
    A.create_meta(ctrl)
    spai = api.Spai(17)
    spai.set_matrix(A, ctrl)
    losses = [spai.train_step(ctrl, lr=2e-3) for _ in range(40)]
    assert np.mean(losses[-5:]) < losses[0]
    spai.build(ctrl)
    frp, fcol, G = spai.factor()
    T = sp.tril(sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)))).tocsr()
    assert np.array_equal(frp.astype(np.int64), T.indptr) and np.array_equal(fcol.astype(np.int64), T.indices)
    b = np.random.default_rng(2).uniform(-1, 1, n)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    sc = api.SolverControl(L.DIAGONAL, 50000, 1e-10, 0.0)
    info = api.cg_learned(x, A, torch.tensor(b, device="cuda"), sc, spai, ctrl, inner="fp32", inner_tol=0.3)
    sc.release()
    spai.release()
    Ao = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)))
    assert info["converged"] == 1
    assert np.linalg.norm(b - Ao @ x.cpu().numpy()) / np.linalg.norm(b) <= 1.5e-10


def test_device_graph_build_rejects_unsuitable_matrices(ctrl):
    """The graph is built on the device; matrices it cannot take are refused
    with clsparseInvalidValue: an asymmetric pattern, a non-positive
    diagonal."""
    rp, col, val = matgen.poisson2d(8)
    M = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))).tolil()
    M[0, 20] = -0.01  # (0, 20) without (20, 0)
    M = M.tocsr()
    M.sort_indices()
    for bad in (M, None):
        if bad is None:
            v = val.copy()
            v[0] = -1.0  # a_00 < 0
            A = api.CsrMatrix.from_numpy(rp, col, v)
        else:
            A = api.CsrMatrix.from_numpy(bad.indptr.astype(np.uint32), bad.indices.astype(np.uint32), bad.data)
        spai = api.Spai(1)
        with pytest.raises(api.ClsparseError) as e:
            spai.set_matrix(A, ctrl)
        assert e.value.status == L.clsparseInvalidValue
        spai.release()


def test_data_parallel_training_on_device(ctrl):
    """clsparse_b200.distributed.dp_train with two network replicas on one GPU
    (LocalComm sums the device gradient buffers in rank order): the replicas
    stay bit for bit equal. One rank reproduces clsparseB200SpaiTrainStep
    exactly (the same loss, gradient and Adam step), and the residual
    snapshots that make the probes come from one solve."""
    from clsparse_b200 import distributed as D
    samples = [learn.Sample(ctrl, 32, s) for s in range(4)]
    assert samples[0].probes.shape == (4, 32 * 32)
    reps = [api.Spai(77), api.Spai(77)]
    nets = [D.DeviceNet(s, ctrl) for s in reps]
    losses = D.dp_train(nets, D.LocalComm(), samples, steps=12, lr=3e-3)
    np.testing.assert_array_equal(reps[0].params(), reps[1].params())
    assert all(np.isfinite(losses)) and losses[-1] < losses[0]
    # one rank == the fused train step
    a, b = api.Spai(5), api.Spai(5)
    D.dp_train([D.DeviceNet(a, ctrl)], D.LocalComm(), samples, steps=6, lr=2e-3, lam=0.2)
    for t in range(6):
        smp = samples[t % len(samples)]
        b.set_matrix(smp.A, ctrl)
        b.train_step(ctrl, smp.probes, 0.2, 2e-3 * (0.1 ** (t / 6)))
    np.testing.assert_array_equal(a.params(), b.params())
