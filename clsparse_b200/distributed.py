"""Multi-GPU layer: one process per GPU, torch.distributed for the plumbing.

The hot path shards by rows: every rank owns a contiguous, nnz-balanced range
of rows (with global column indices) and computes those rows of y = A x with
the library's SpMV; an iterative method then all-gathers the new vector so
every rank holds the whole of it for the next product (the x needed by a
row block touches arbitrary columns on irregular matrices; on stencils a halo
would do, the all-gather is the general case). CG all-reduces its dot
products, one message per reduction point.

Batched solves are independent units: systems are spread over ranks by the
LPT rule (longest processing time first, weight = nonzeros), each rank solves
its share in one batched launch, and rank results are gathered.

The collectives are torch.distributed (NCCL on GPUs, gloo on CPU for the
tests); remote data always lands in local memory before a kernel reads it.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def row_partition(rp, world: int):
    """Contiguous row ranges [(r0, r1)] per rank, balanced by nonzeros (each
    rank's first row is the first whose row-pointer reaches its share)."""
    rp = np.asarray(rp, dtype=np.int64)
    n = len(rp) - 1
    nnz = int(rp[-1] - rp[0])
    cuts = [0]
    for k in range(1, world):
        target = rp[0] + nnz * k // world
        cuts.append(int(min(max(np.searchsorted(rp, target, side="left"), cuts[-1]), n)))
    cuts.append(n)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


def local_rows(rp, col, val, r0: int, r1: int):
    """CSR of rows [r0, r1) with global column indices."""
    rp = np.asarray(rp, dtype=np.int64)
    a, b = int(rp[r0]), int(rp[r1])
    return (rp[r0:r1 + 1] - a).astype(np.uint32), np.asarray(col)[a:b], np.asarray(val)[a:b]


def lpt_partition(weights, world: int):
    """LPT assignment of items to ranks: items by decreasing weight (ties by
    index), each to the least-loaded rank (ties by rank). Returns one sorted
    index array per rank. The makespan is at most 4/3 of the optimum."""
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += w[i]
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def all_gather_rows(y_loc: torch.Tensor, parts, group=None) -> torch.Tensor:
    """The full vector from every rank's row range (ranges may differ in
    length: each rank's part is padded to the longest before the gather)."""
    world = len(parts)
    m = max(r1 - r0 for r0, r1 in parts)
    pad = torch.zeros(m, dtype=y_loc.dtype, device=y_loc.device)
    pad[: y_loc.numel()] = y_loc
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([bufs[k][: parts[k][1] - parts[k][0]] for k in range(world)])


def dist_cg(local_spmv, b_loc: torch.Tensor, inv_diag_loc: torch.Tensor, parts, rel_tol: float = 1e-10,
            max_iters: int = 10000, group=None):
    """Row-partitioned Jacobi-PCG, the reference's operation order
    (src/library/solvers/conjugate-gradients.hpp:65-226) with the L2 stop
    test ||r||_2 / ||b||_2 <= rel_tol. local_spmv(p_full) returns this rank's
    rows of A p. Returns (x_loc, iterations, relative residual)."""
    def allsum(*vals):
        t = torch.stack([v.to(torch.float64) for v in vals])
        dist.all_reduce(t, group=group)
        return t

    x = torch.zeros_like(b_loc)
    r = b_loc.clone()
    z = r * inv_diag_loc
    p = z.clone()
    nb, rz = allsum((b_loc * b_loc).sum(), (r * z).sum())
    nb = float(nb.sqrt())
    if nb == 0.0:
        return x, 0, 0.0
    res = 1.0
    it = 0
    while it < max_iters:
        q = local_spmv(all_gather_rows(p, parts, group))
        pq = float(allsum((p * q).sum())[0])
        alpha = float(rz) / pq
        x += alpha * p
        r -= alpha * q
        z = r * inv_diag_loc
        rz_new, rr = allsum((r * z).sum(), (r * r).sum())
        it += 1
        res = float(rr.sqrt()) / nb
        if res <= rel_tol:
            break
        beta = float(rz_new) / float(rz)
        rz = rz_new
        p = z + beta * p
    return x, it, res


def dist_batched(solve_share, weights, group=None):
    """Spreads independent systems over the ranks with lpt_partition and
    gathers the per-system results. solve_share(indices) solves this rank's
    systems and returns one float64 row per system (e.g. iterations,
    residual). Returns the gathered (num_systems, k) array on every rank."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else \
        torch.device("cpu")
    shares = lpt_partition(weights, world)
    mine = shares[rank]
    res = torch.as_tensor(np.asarray(solve_share(mine), dtype=np.float64)).reshape(len(mine), -1).to(dev)
    k = res.shape[1] if res.numel() else 0
    kk = torch.tensor([k], dtype=torch.int64, device=dev)
    dist.all_reduce(kk, op=dist.ReduceOp.MAX, group=group)
    k = int(kk)
    m = max(len(s) for s in shares)
    pad = torch.zeros(m, k, dtype=torch.float64, device=dev)
    if len(mine):
        pad[: len(mine)] = res
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    out = torch.zeros(len(weights), k, dtype=torch.float64)
    for r, s in enumerate(shares):
        if len(s):
            out[torch.as_tensor(s)] = bufs[r][: len(s)].cpu()
    return out.numpy()
