"""The multi-GPU host logic (clsparse_b200.distributed) on CPU: partitions,
exchange plans, and the row-partitioned CG driver and the batched sharding
run as a world-size-2 gloo process group (spawned processes, 127.0.0.1) with
the rank's kernels replaced by a CPU stand-in (tests/dist_host_rank.py). A
rank that leaves is noticed by the others through a failing collective (the
process group's timeout), not by a hang."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from clsparse_b200 import distributed as D
from clsparse_b200 import matgen


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s=30):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _finish(q):
    # flush the queue's feeder thread before the process ends
    q.close()
    q.join_thread()


def _problem():
    rp, col, val = matgen.diffusion3d_lognormal(12, sigma=1.0, seed=5)
    b = np.random.default_rng(2).uniform(-1, 1, len(rp) - 1)
    return rp, col, val, b


def _cg_problems():
    """(name, rp, col, val, b, precond, max_iters, rel): a stencil (halo
    exchange), an irregular matrix (all-gather), the iteration limit, no
    preconditioner and a zero right-hand side."""
    rp, col, val, b = _problem()
    rs = matgen.random_spd(3000, per_row=8, seed=4)
    bs = np.random.default_rng(5).uniform(-1, 1, 3000)
    return [("stencil", rp, col, val, b, 1, 5000, 1e-10),
            ("irregular", *rs, bs, 1, 5000, 1e-10),
            ("limit", rp, col, val, b, 1, 5, 1e-10),
            ("none", rp, col, val, b, 0, 5000, 1e-8),
            ("zero_b", rp, col, val, np.zeros_like(b), 1, 100, 1e-10)]


def _host_cg(rp, col, val, b, precond, max_iters, rel, parts, ranks_here, plans, comm):
    """Runs the driver over HostRank stand-ins for the ranks in ranks_here;
    returns (info, [x of each rank])."""
    import torch
    from dist_host_rank import HostRank, HostSolverControl
    rks, xs, bs, scs = [], [], [], []
    for k in ranks_here:
        lrp, lcol, lval = D.setup_local(rp, col, val, parts, k, plans[k])
        rks.append(HostRank(plans[k], lrp, lcol, lval, precond))
        r0, r1 = parts[k]
        xs.append(torch.zeros(r1 - r0, dtype=torch.float64))
        bs.append(torch.tensor(b[r0:r1]))
        scs.append(HostSolverControl(precond, max_iters, rel, 0.0))
    info = D.dist_cg(rks, comm, xs, bs, scs, check_every=4)
    return info, [x.numpy() for x in xs]


def _rank_main(rank, world, port, q):
    """Row-partitioned CG (gloo, CPU stand-in kernels), then the batched
    sharding, on one gloo group."""
    dist = _init(rank, world, port)
    try:
        out = {}
        for name, rp, col, val, b, pre, mi, rel in _cg_problems():
            parts = D.row_partition(rp, world)
            r0, r1 = parts[rank]
            _, lcol, _ = D.local_rows(rp, col, val, r0, r1)
            plan = D.plan_for_rank(lcol, parts, rank)
            plans = {rank: plan}
            info, (x,) = _host_cg(rp, col, val, b, pre, mi, rel, parts, [rank], plans, D.TorchComm())
            out[name] = (info, x, plan.mode)

        def solve_share(idx):
            return [[10.0 * i, float(rank)] for i in idx]

        gathered = D.dist_batched(solve_share, [7, 1, 5, 5, 2, 9, 3])
        from dist_host_rank import HostNet, toy_samples
        net = HostNet(40)
        losses = D.dp_train([net], D.TorchComm(), toy_samples(), steps=30, lr=0.05)
        q.put((rank, out, gathered, (losses, net.p)))
    finally:
        dist.destroy_process_group()
        _finish(q)


def _dying_rank(rank, world, port, q):
    import torch
    dist = _init(rank, world, port, timeout_s=5)
    if rank == 1:
        q.put((rank, "left"))
        _finish(q)
        os._exit(0)  # leaves between steps, without joining the next collective
    try:
        t = torch.ones(1)
        dist.all_reduce(t)
        q.put((rank, "no error"))
    except Exception as e:  # the peer is gone: the collective fails instead of hanging
        q.put((rank, type(e).__name__))
    _finish(q)
    os._exit(0)


def _spawn(target, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    return sorted(out, key=lambda t: t[0]), procs


def test_row_partition_balances_nonzeros():
    rp, _, _ = matgen.irregular(50_000, n_dense=3, dense_len=10_000, seed=3)
    for world in (1, 2, 3, 8):
        parts = D.row_partition(rp, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(rp) - 1
        assert all(parts[k][1] == parts[k + 1][0] for k in range(world - 1))
        loads = [int(rp[r1]) - int(rp[r0]) for r0, r1 in parts]
        longest = int(np.diff(rp.astype(np.int64)).max())
        assert max(loads) - min(loads) <= 2 * longest + 2


def test_lpt_partition_assigns_each_once_and_bounds_makespan():
    w = np.random.default_rng(1).lognormal(8, 1, 500)
    for world in (2, 3, 8):
        shares = D.lpt_partition(w, world)
        np.testing.assert_array_equal(np.sort(np.concatenate(shares)), np.arange(len(w)))
        loads = [w[s].sum() for s in shares]
        assert max(loads) <= w.sum() / world + w.max()
    assert [list(s) for s in D.lpt_partition([5, 1, 4, 3], 2)] == [[0, 1], [2, 3]]


@pytest.fixture(scope="module")
def two_ranks():
    out, procs = _spawn(_rank_main, 2)
    assert all(p.exitcode == 0 for p in procs)
    return out


@pytest.mark.parametrize("name", ["stencil", "irregular", "limit", "none", "zero_b"])
def test_distributed_cg_matches_single_rank(two_ranks, orc, name):
    """The gloo world-size-2 run (one process per rank, CPU stand-in kernels)
    against the same driver with one rank and with both ranks in one process
    (LocalComm), and against the oracle's reference-order CG."""
    (_, rp, col, val, b, pre, mi, rel), = [p for p in _cg_problems() if p[0] == name]
    n = len(rp) - 1
    parts1 = D.row_partition(rp, 1)
    plans1 = D.make_plans([D.needed_columns(col, 0, n)], parts1)
    info1, (x1,) = _host_cg(rp, col, val, b, pre, mi, rel, parts1, [0], plans1, D.LocalComm())
    parts2 = D.row_partition(rp, 2)
    needed = [D.needed_columns(D.local_rows(rp, col, val, *parts2[k])[1], *parts2[k]) for k in range(2)]
    plans2 = D.make_plans(needed, parts2)
    info2, xs2 = _host_cg(rp, col, val, b, pre, mi, rel, parts2, [0, 1], plans2, D.LocalComm())
    x2 = np.concatenate(xs2)
    want_mode = {"irregular": D.ALLGATHER}.get(name, D.HALO)
    for rank, out, *_ in two_ranks:
        info, x, mode = out[name]
        assert mode == want_mode
        r0, r1 = parts2[rank]
        # the process-per-rank run is the in-process two-rank run, bit for bit
        assert info == info2
        np.testing.assert_array_equal(x, x2[r0:r1])
    assert info2["nIters"] == info1["nIters"]
    assert info2["initialResidual"] == pytest.approx(info1["initialResidual"], rel=1e-13)
    scale = max(np.abs(x1).max(), 1e-300)
    assert np.abs(x2 - x1).max() <= 1e-9 * scale
    xo, oi = orc.solve("cg", np.float64, rp, col, val, np.zeros(n), b, pre, mi, rel, 0.0)
    assert abs(info1["nIters"] - oi.nIters) <= 1, (info1, oi.nIters)
    assert info1["initialResidual"] == pytest.approx(oi.initialResidual, rel=1e-13)
    if name == "zero_b":
        assert info1["nIters"] == 0 and not x1.any()
    elif name == "limit":
        assert info1["nIters"] == 5
    else:
        assert info1["currentResidual"] <= rel
        assert np.abs(x1 - xo).max() <= 1e-6 * max(np.abs(xo).max(), 1e-300)


def test_exchange_plans_cover_every_column():
    """Every column a rank's rows reference maps into its extended vector,
    onto the entry that holds that global column after the exchange."""
    for rp, col, val in (matgen.poisson2d(40), matgen.random_spd(2000, seed=2),
                         matgen.irregular(3000, n_dense=3, dense_len=1000, seed=1)):
        n = len(rp) - 1
        for world in (2, 3, 5):
            parts = D.row_partition(rp, world)
            needed = [D.needed_columns(D.local_rows(rp, col, val, *parts[k])[1], *parts[k]) for k in range(world)]
            for mode in (D.HALO, D.ALLGATHER):
                plans = D.make_plans(needed, parts, mode)
                g = np.arange(n, dtype=np.float64)  # entry value = global column
                for k in range(world):
                    p = plans[k]
                    ext = np.full(p.ext_len, -1.0)
                    r0, r1 = parts[k]
                    ext[p.own:p.own + r1 - r0] = g[r0:r1]
                    if mode == D.HALO:
                        for q, (off, cnt) in p.recv.items():
                            src = plans[q].send[k] + parts[q][0]
                            assert len(src) == cnt
                            ext[off:off + cnt] = g[src]
                    else:
                        for q in range(world):
                            a, b = parts[q]
                            ext[q * p.chunk:q * p.chunk + b - a] = g[a:b]
                    _, lcol, _ = D.local_rows(rp, col, val, r0, r1)
                    np.testing.assert_array_equal(ext[p.ext_columns(lcol)], lcol.astype(np.float64))


def test_distributed_batched_gathers_every_system(two_ranks):
    shares = D.lpt_partition([7, 1, 5, 5, 2, 9, 3], 2)
    owner = {int(i): r for r, s in enumerate(shares) for i in s}
    for t in two_ranks:
        res = t[2]
        np.testing.assert_array_equal(res[:, 0], 10.0 * np.arange(7))
        np.testing.assert_array_equal(res[:, 1], [owner[i] for i in range(7)])


def test_dead_rank_ends_collective_with_error():
    out, _ = _spawn(_dying_rank, 2)
    d = dict(out)
    assert d[1] == "left" and d[0] != "no error"


def test_data_parallel_training_keeps_replicas_identical(two_ranks):
    """Two gloo ranks training the CPU stand-in network on different samples
    with a gradient all-reduce per step: both replicas end bit for bit equal,
    equal to the same two ranks run in one process (LocalComm), and the loss
    falls."""
    from dist_host_rank import HostNet, toy_samples
    nets = [HostNet(40), HostNet(40)]
    losses = D.dp_train(nets, D.LocalComm(), toy_samples(), steps=30, lr=0.05)
    np.testing.assert_array_equal(nets[0].p, nets[1].p)
    for _, _, _, (l_r, p_r) in two_ranks:
        np.testing.assert_array_equal(p_r, nets[0].p)
        assert l_r == losses
    assert losses[-1] < 0.75 * losses[0]  # a least-squares floor remains
