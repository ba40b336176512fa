"""The row-partitioned CG's device path (csrc/dist_cg.cu through
clsparse_b200.distributed.DeviceRank) on one GPU: several ranks' kernels run
in one process with LocalComm (copies for the exchange, an ordered sum for the
all-reduce; no kernel waits on another), and one rank over a real NCCL
process group of size 1. Checked against the CPU stand-in of the same stages
(tests/dist_host_rank.py), across rank counts, and against the oracle's
reference-order CG (src/library/solvers/conjugate-gradients.hpp:65-226)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from clsparse_b200 import api
from clsparse_b200 import distributed as D
from clsparse_b200 import matgen
from dist_host_rank import HostRank, HostSolverControl

pytestmark = pytest.mark.gpu


def _plans(rp, col, val, world, mode=None):
    parts = D.row_partition(rp, world)
    needed = [D.needed_columns(D.local_rows(rp, col, val, *parts[k])[1], *parts[k]) for k in range(world)]
    return parts, D.make_plans(needed, parts, mode)


def device_cg(ctrl, rp, col, val, b, world, precond=1, max_iters=5000, rel=1e-10, mode=None, x0=None):
    parts, plans = _plans(rp, col, val, world, mode)
    rks, xs, bs, scs = [], [], [], []
    for k in range(world):
        lrp, lcol, lval = D.setup_local(rp, col, val, parts, k, plans[k])
        rks.append(D.DeviceRank(plans[k], lrp, lcol, lval, precond, ctrl))
        r0, r1 = parts[k]
        xs.append(torch.tensor(np.zeros(r1 - r0) if x0 is None else x0[r0:r1], device="cuda"))
        bs.append(torch.tensor(b[r0:r1], device="cuda"))
        scs.append(api.SolverControl(precond, max_iters, rel, 0.0))
    try:
        info = D.dist_cg(rks, D.LocalComm(), xs, bs, scs)
    finally:
        for rk in rks:
            rk.release()
        for sc in scs:
            sc.release()
    return info, np.concatenate([x.cpu().numpy() for x in xs]), plans[0].mode


def host_cg(rp, col, val, b, world, precond=1, max_iters=5000, rel=1e-10, mode=None):
    parts, plans = _plans(rp, col, val, world, mode)
    rks, xs, bs, scs = [], [], [], []
    for k in range(world):
        lrp, lcol, lval = D.setup_local(rp, col, val, parts, k, plans[k])
        rks.append(HostRank(plans[k], lrp, lcol, lval, precond))
        r0, r1 = parts[k]
        xs.append(torch.zeros(r1 - r0, dtype=torch.float64))
        bs.append(torch.tensor(b[r0:r1]))
        scs.append(HostSolverControl(precond, max_iters, rel, 0.0))
    info = D.dist_cg(rks, D.LocalComm(), xs, bs, scs)
    return info, np.concatenate([x.numpy() for x in xs])


PROBLEMS = {
    "stencil3d": lambda: matgen.diffusion3d_lognormal(20, sigma=1.0, seed=5),
    "poisson2d": lambda: matgen.poisson2d(96),
    "irregular": lambda: matgen.random_spd(20_000, per_row=8, seed=4),
}


@pytest.mark.parametrize("mode", [None, D.HALO, D.ALLGATHER], ids=["auto", "halo", "allgather"])
@pytest.mark.parametrize("world", [1, 2, 4])
@pytest.mark.parametrize("prob", sorted(PROBLEMS))
def test_device_ranks_match_stand_in_and_oracle(ctrl, orc, prob, world, mode):
    rp, col, val = PROBLEMS[prob]()
    n = len(rp) - 1
    b = np.random.default_rng(7).uniform(-1, 1, n)
    info, x, used = device_cg(ctrl, rp, col, val, b, world, mode=mode)
    if mode is None:
        assert used == (D.ALLGATHER if prob == "irregular" and world > 1 else D.HALO)
    hinfo, hx = host_cg(rp, col, val, b, world, mode=mode)
    assert abs(info["nIters"] - hinfo["nIters"]) <= 1, (info, hinfo)
    assert info["initialResidual"] == pytest.approx(hinfo["initialResidual"], rel=1e-13)
    assert info["currentResidual"] <= 1e-10
    xo, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, 1, 5000, 1e-10, 0.0)
    assert abs(info["nIters"] - oi.nIters) <= max(2, oi.nIters // 50), (info, oi.nIters)
    assert np.abs(x - xo).max() <= 1e-7 * np.abs(xo).max()
    assert np.abs(x - hx).max() <= 1e-7 * np.abs(hx).max()


def test_rank_counts_agree_and_repeat_bitwise(ctrl):
    rp, col, val = matgen.diffusion3d_lognormal(24, sigma=1.0, seed=2)
    b = np.random.default_rng(3).uniform(-1, 1, len(rp) - 1)
    runs = {w: device_cg(ctrl, rp, col, val, b, w) for w in (1, 2, 3, 8)}
    its = {w: r[0]["nIters"] for w, r in runs.items()}
    assert max(its.values()) - min(its.values()) <= 1, its
    again = device_cg(ctrl, rp, col, val, b, 3)
    assert again[0] == runs[3][0]
    np.testing.assert_array_equal(again[1], runs[3][1])


def test_iteration_limit_zero_rhs_and_warm_start(ctrl):
    rp, col, val = matgen.poisson2d(64)
    n = len(rp) - 1
    b = np.random.default_rng(4).uniform(-1, 1, n)
    info, _, _ = device_cg(ctrl, rp, col, val, b, 2, max_iters=7)
    assert info["nIters"] == 7 and info["currentResidual"] > 1e-10
    info, x, _ = device_cg(ctrl, rp, col, val, np.zeros(n), 2)
    assert info["nIters"] == 0 and info["initialResidual"] == 0.0 and not x.any()
    # an exact initial guess stops before the first iteration
    import scipy.sparse as sp
    xs = np.random.default_rng(5).uniform(-1, 1, n)
    bb = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64))) @ xs
    info, x, _ = device_cg(ctrl, rp, col, val, bb, 2, rel=1e-12, x0=xs)
    assert info["nIters"] == 0
    np.testing.assert_array_equal(x, xs)
    # no preconditioner
    info, x, _ = device_cg(ctrl, rp, col, val, b, 2, precond=0, rel=1e-8)
    hinfo, hx = host_cg(rp, col, val, b, 2, precond=0, rel=1e-8)
    assert abs(info["nIters"] - hinfo["nIters"]) <= 1


def test_create_rejects_bad_columns_and_missing_diagonal(ctrl):
    from clsparse_b200 import _lib as L
    rp, col, val = matgen.poisson2d(8)
    parts, plans = _plans(rp, col, val, 2)
    lrp, lcol, lval = D.setup_local(rp, col, val, parts, 0, plans[0])
    bad = lcol.copy()
    bad[3] = plans[0].ext_len
    with pytest.raises(RuntimeError, match=str(L.clsparseInvalidValue)):
        D.DeviceRank(plans[0], lrp, bad, lval, 1, ctrl)
    nodiag = lval.copy()
    own = np.repeat(np.arange(len(lrp) - 1), np.diff(lrp.astype(np.int64)))
    nodiag[lcol == own] = 0.0
    with pytest.raises(RuntimeError, match=str(L.clsparseInvalidValue)):
        D.DeviceRank(plans[0], lrp, lcol, nodiag, 1, ctrl)
    D.DeviceRank(plans[0], lrp, lcol, nodiag, 0, ctrl).release()  # fine without Jacobi


def test_one_rank_over_nccl(ctrl, orc):
    """The torch.distributed path (TorchComm) on a real NCCL group of one
    rank: the all-reduce runs on the device view of the sums."""
    import datetime
    import os
    import socket

    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        rp, col, val = matgen.poisson2d(128)
        n = len(rp) - 1
        b = np.random.default_rng(8).uniform(-1, 1, n)
        parts = D.row_partition(rp, 1)
        plan = D.plan_for_rank(col, parts, 0)
        lrp, lcol, lval = D.setup_local(rp, col, val, parts, 0, plan)
        rk = D.DeviceRank(plan, lrp, lcol, lval, 1, ctrl)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        sc = api.SolverControl(1, 5000, 1e-10, 0.0)
        info = D.dist_cg([rk], D.TorchComm(), [x], [torch.tensor(b, device="cuda")], [sc])
        rk.release()
        sc.release()
        linfo, lx, _ = device_cg(ctrl, rp, col, val, b, 1)
        assert info == linfo
        np.testing.assert_array_equal(x.cpu().numpy(), lx)
    finally:
        dist.destroy_process_group()
