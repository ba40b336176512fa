"""The multi-GPU host logic (clsparse_b200.distributed) on CPU: partitions,
and the row-partitioned CG and the batched sharding run as a world-size-2
gloo process group (spawned processes, 127.0.0.1) with the local SpMV done by
scipy. A rank that leaves is noticed by the others through a failing
collective (the process group's timeout), not by a hang."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
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


def _rank_main(rank, world, port, q):
    """Row-partitioned CG, then the batched sharding, on one gloo group."""
    import torch
    dist = _init(rank, world, port)
    try:
        rp, col, val, b = _problem()
        n = len(rp) - 1
        parts = D.row_partition(rp, world)
        r0, r1 = parts[rank]
        lrp, lcol, lval = D.local_rows(rp, col, val, r0, r1)
        Aloc = sp.csr_matrix((lval, lcol.astype(np.int64), lrp.astype(np.int64)), shape=(r1 - r0, n))
        A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
        dinv = torch.tensor(1.0 / A.diagonal()[r0:r1])

        def spmv(p_full):
            return torch.from_numpy(Aloc @ p_full.numpy())

        x, it, res = D.dist_cg(spmv, torch.tensor(b[r0:r1]), dinv, parts, rel_tol=1e-10, max_iters=5000)
        xs = D.all_gather_rows(x, parts).numpy()

        def solve_share(idx):
            return [[10.0 * i, float(rank)] for i in idx]

        gathered = D.dist_batched(solve_share, [7, 1, 5, 5, 2, 9, 3])
        q.put((rank, it, res, xs, gathered))
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


def _serial_cg(A, b, tol=1e-10, max_iters=5000):
    """The same Jacobi-PCG on one process (reference for the iteration count)."""
    dinv = 1.0 / A.diagonal()
    x = np.zeros_like(b)
    r = b.copy()
    z = r * dinv
    p = z.copy()
    rz = r @ z
    nb = np.linalg.norm(b)
    for it in range(1, max_iters + 1):
        q = A @ p
        alpha = rz / (p @ q)
        x += alpha * p
        r -= alpha * q
        z = r * dinv
        rz_new = r @ z
        if np.linalg.norm(r) / nb <= tol:
            return x, it
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iters


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


def test_distributed_cg_matches_single_rank(two_ranks):
    rp, col, val, b = _problem()
    n = len(rp) - 1
    A = sp.csr_matrix((val, col.astype(np.int64), rp.astype(np.int64)), shape=(n, n))
    _, it1 = _serial_cg(A, b)
    its = {t[1] for t in two_ranks}
    assert len(its) == 1  # every rank took the same stop decision
    assert abs(its.pop() - it1) <= 1 and all(t[2] <= 1e-10 for t in two_ranks)
    xd = spla.spsolve(A.tocsc(), b)
    for t in two_ranks:
        assert np.linalg.norm(t[3] - xd) / np.linalg.norm(xd) <= 1e-7
        np.testing.assert_array_equal(t[3], two_ranks[0][3])


def test_distributed_batched_gathers_every_system(two_ranks):
    shares = D.lpt_partition([7, 1, 5, 5, 2, 9, 3], 2)
    owner = {int(i): r for r, s in enumerate(shares) for i in s}
    for t in two_ranks:
        res = t[4]
        np.testing.assert_array_equal(res[:, 0], 10.0 * np.arange(7))
        np.testing.assert_array_equal(res[:, 1], [owner[i] for i in range(7)])


def test_dead_rank_ends_collective_with_error():
    out, _ = _spawn(_dying_rank, 2)
    d = dict(out)
    assert d[1] == "left" and d[0] != "no error"
