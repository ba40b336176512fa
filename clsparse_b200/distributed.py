"""Multi-GPU layer: one process per GPU, torch.distributed for the plumbing.

The hot path shards by rows: every rank owns a contiguous, nnz-balanced range
of rows (row_partition) and runs its part of CG through the library's
row-partitioned CG (clsparseB200DistCg*, csrc/dist_cg.cu). Per iteration a
rank launches two kernels and takes part in two collectives:

  * the exchange of the vector the SpMV reads. Its rows reference other
    ranks' entries; those land in the rank's own memory before the SpMV runs:
    for a stencil (each rank needs a few boundary planes of its neighbours) a
    HALO of point-to-point sends and receives (batch_isend_irecv, NCCL
    send/recv) into the tail of a local "extended" vector, and for an
    irregular matrix (rows reference most of the vector) an ALL-GATHER
    (all_gather_into_tensor) of fixed-size chunks;
  * ONE all-reduce of three FP64 sums (<r,z>, <w,z>, ||r||_1): the CG is in
    the Chronopoulos-Gear arrangement (see csrc/dist_cg.cu), which forms all
    of an iteration's sums after its one SpMV.

The stop decision is taken on the device from the all-reduced sums (bitwise
the same on every rank), so the host enqueues iterations in chunks and reads
the state once per chunk, at the same step on every rank.

The driver (dist_cg) works on a list of ranks with a communicator: in a
torch.distributed job each process passes its one rank and a TorchComm;
LocalComm runs several ranks' device work in one process, on one GPU, with
plain copies for the exchange and an ordered sum for the all-reduce (the same
kernels and the same sequence of stages, nothing waiting on anything). The
multi-process CPU tests drive the same code with a CPU stand-in for the
rank's kernels over gloo.

Batched solves are independent units: systems are spread over ranks by the
LPT rule (longest processing time first, weight = nonzeros), each rank solves
its share in one batched launch, and rank results are gathered.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

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


# ---------------------------------------------------------------- exchange plan

HALO, ALLGATHER = "halo", "allgather"


@dataclass
class Plan:
    """How one rank's extended vector is laid out and filled.

    halo:      ext = [own rows | entries from peer q1 | from q2 | ...] (peers
               in rank order, each block sorted by column); recv[q] = (offset,
               count) of q's block, send[q] = local indices of the own entries
               q needs (sorted).
    allgather: ext = world chunks of `chunk` entries, rank k's rows at
               k * chunk (the tail of a chunk is padding)."""
    mode: str
    rank: int
    world: int
    parts: list
    ext_len: int
    own: int
    chunk: int = 0
    recv: dict = field(default_factory=dict)
    send: dict = field(default_factory=dict)
    halo_cols: dict = field(default_factory=dict)  # peer -> the global columns received from it

    @property
    def n_local(self):
        r0, r1 = self.parts[self.rank]
        return r1 - r0

    def ext_columns(self, cols):
        """Global column indices of this rank's rows -> positions in ext."""
        cols = np.asarray(cols, dtype=np.int64)
        r0, r1 = self.parts[self.rank]
        if self.mode == ALLGATHER:
            starts = np.array([a for a, _ in self.parts], dtype=np.int64)
            owner = np.searchsorted(starts, cols, side="right") - 1
            return (owner * self.chunk + cols - starts[owner]).astype(np.uint32)
        out = cols - r0
        remote = (cols < r0) | (cols >= r1)
        halo = np.concatenate([self.halo_cols[q] for q in sorted(self.halo_cols)]) \
            if self.halo_cols else np.zeros(0, np.int64)
        out[remote] = self.n_local + np.searchsorted(halo, cols[remote])
        return out.astype(np.uint32)


def needed_columns(cols, r0: int, r1: int):
    """Sorted distinct columns outside [r0, r1) that rows [r0, r1) reference."""
    c = np.unique(np.asarray(cols, dtype=np.int64))
    return c[(c < r0) | (c >= r1)]


def make_plans(needed, parts, mode: str | None = None):
    """Plans of every rank from every rank's needed_columns (the same result
    on every rank). mode None picks the halo when no rank needs more entries
    than half its own row count, else the all-gather."""
    world = len(parts)
    starts = np.array([a for a, _ in parts], dtype=np.int64)
    if mode is None:
        mode = HALO if all(len(needed[k]) <= max(1, (parts[k][1] - parts[k][0]) // 2) for k in range(world)) \
            else ALLGATHER
    plans = []
    chunk = max(max(r1 - r0 for r0, r1 in parts), 1)
    for k in range(world):
        r0, r1 = parts[k]
        if mode == ALLGATHER:
            plans.append(Plan(ALLGATHER, k, world, parts, world * chunk, k * chunk, chunk=chunk))
            continue
        nk = np.asarray(needed[k], dtype=np.int64)
        owner = np.searchsorted(starts, nk, side="right") - 1
        recv, halo_cols, off = {}, {}, r1 - r0
        for q in range(world):
            cq = nk[owner == q]
            if len(cq):
                recv[q] = (off, len(cq))
                halo_cols[q] = cq
                off += len(cq)
        plans.append(Plan(HALO, k, world, parts, off, 0, recv=recv, halo_cols=halo_cols))
    if mode == HALO:
        for k in range(world):
            r0, _ = parts[k]
            for q in range(world):
                if k in plans[q].recv:
                    plans[k].send[q] = (plans[q].halo_cols[k] - r0).astype(np.int64)
    return plans


def _contiguous(idx):
    return len(idx) > 0 and int(idx[-1]) - int(idx[0]) + 1 == len(idx)


# ---------------------------------------------------------------- device rank

class _DevArray:
    """A view of library-owned device memory that torch can wrap."""

    def __init__(self, ptr: int, n: int, device: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}
        self.device = device


def _wrap(ptr: int, n: int, device: int) -> torch.Tensor:
    return torch.as_tensor(_DevArray(ptr, n, device), device=torch.device("cuda", device))


class DeviceRank:
    """One rank's part of the row-partitioned CG on its GPU (the library's
    clsparseB200DistCg*). rp/col_ext/val: the rank's rows, columns already in
    extended positions (Plan.ext_columns)."""

    def __init__(self, plan: Plan, rp, col_ext, val, precond: int, ctrl):
        from . import _lib as L
        from .api import check, lib
        self.L, self.lib, self.check = L, lib(), check
        self.plan, self.ctrl = plan, ctrl
        dev = torch.cuda.current_device()
        self.device = dev
        n = len(rp) - 1
        assert n == plan.n_local
        self.rp = torch.as_tensor(np.asarray(rp, np.uint32).view(np.int32), device="cuda")
        self.col = torch.as_tensor(np.asarray(col_ext, np.uint32).view(np.int32), device="cuda")
        self.val = torch.as_tensor(np.asarray(val, np.float64), device="cuda")
        self.csr = L.clsparseCsrMatrix(num_rows=n, num_cols=plan.ext_len, num_nonzeros=len(val),
                                       values=self.val.data_ptr(), col_indices=self.col.data_ptr(),
                                       row_pointer=self.rp.data_ptr())
        self.h = C.c_void_p()
        check(self.lib.clsparseB200DistCgCreate(C.byref(self.h), C.byref(self.csr), plan.ext_len, plan.own,
                                                int(precond), ctrl.handle), "clsparseB200DistCgCreate")
        px, pz, ps = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
        check(self.lib.clsparseB200DistCgBuffers(self.h, C.byref(px), C.byref(pz), C.byref(ps)),
              "clsparseB200DistCgBuffers")
        addr = lambda p: C.cast(p, C.c_void_p).value  # noqa: E731
        self.xext = _wrap(addr(px), plan.ext_len, dev)
        self.zext = _wrap(addr(pz), plan.ext_len, dev)
        self.sums = _wrap(addr(ps), 4, dev)
        self._send_idx = {q: torch.as_tensor(idx.astype(np.int32), device="cuda")
                          for q, idx in plan.send.items() if not _contiguous(idx)}
        self._send_buf = {q: torch.empty(len(idx), dtype=torch.float64, device="cuda")
                          for q, idx in plan.send.items() if not _contiguous(idx)}

    def release(self):
        if self.h:
            self.lib.clsparseB200DistCgRelease(self.h)
            self.h = C.c_void_p()

    def ext(self, which: str) -> torch.Tensor:
        return self.xext if which == "x" else self.zext

    def send_view(self, which: str, q: int) -> torch.Tensor:
        """The entries peer q needs, contiguous (a slice, or packed)."""
        idx = self.plan.send[q]
        v = self.ext(which)
        own = self.plan.own
        if _contiguous(idx):
            return v[own + int(idx[0]): own + int(idx[-1]) + 1]
        buf = self._send_buf[q]
        base = v[own:]
        self.check(self.lib.clsparseB200DistCgGather(C.c_void_p(buf.data_ptr()), C.c_void_p(base.data_ptr()),
                                                     C.c_void_p(self._send_idx[q].data_ptr()), len(idx),
                                                     self.ctrl.handle), "clsparseB200DistCgGather")
        return buf

    def start(self, x: torch.Tensor, b: torch.Tensor):
        from .api import vector
        self._x, self._b = x, b
        self.check(self.lib.clsparseB200DistCgStart(self.h, C.byref(vector(x)), C.byref(vector(b)),
                                                    self.ctrl.handle), "clsparseB200DistCgStart")

    def residual(self):
        self.check(self.lib.clsparseB200DistCgResidual(self.h, self.ctrl.handle), "clsparseB200DistCgResidual")

    def product(self):
        self.check(self.lib.clsparseB200DistCgProduct(self.h, self.ctrl.handle), "clsparseB200DistCgProduct")

    def update(self, step: int, sc):
        self.check(self.lib.clsparseB200DistCgUpdate(self.h, step, sc.handle, self.ctrl.handle),
                   "clsparseB200DistCgUpdate")

    def state(self, sc):
        done = C.c_int()
        self.check(self.lib.clsparseB200DistCgState(self.h, C.byref(done), sc.handle, self.ctrl.handle),
                   "clsparseB200DistCgState")
        return bool(done.value), sc.info()


# ---------------------------------------------------------------- communicators

class TorchComm:
    """The exchanges over a torch.distributed process group (NCCL on GPUs,
    gloo on CPU): this process holds one rank."""

    def __init__(self, group=None):
        self.group = group
        self.inplace_gather = dist.get_backend(group) == "nccl"

    def exchange(self, ranks, which: str):
        (rk,) = ranks
        plan = rk.plan
        v = rk.ext(which)
        if plan.mode == ALLGATHER:
            if plan.world == 1:
                return
            mine = v[plan.own: plan.own + plan.chunk]
            dist.all_gather_into_tensor(v, mine if self.inplace_gather else mine.clone(), group=self.group)
            return
        ops = []
        for q, (off, cnt) in sorted(plan.recv.items()):
            ops.append(dist.P2POp(dist.irecv, v[off:off + cnt], q, self.group))
        for q in sorted(plan.send):
            ops.append(dist.P2POp(dist.isend, rk.send_view(which, q), q, self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce(self, ranks, k: int):
        (rk,) = ranks
        dist.all_reduce(rk.sums[:k], group=self.group)

    def world(self, items):
        return dist.get_world_size(self.group)

    def ranks(self, items):
        return [dist.get_rank(self.group)]

    def allreduce_tensors(self, tensors):
        (t,) = tensors
        dist.all_reduce(t, group=self.group)

    def allreduce_host(self, t: torch.Tensor) -> torch.Tensor:
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(self.group) == "nccl" else None
        u = t.to(dev) if dev is not None else t.clone()
        dist.all_reduce(u, group=self.group)
        return u.cpu()


class LocalComm:
    """Several ranks in one process: the exchange copies every rank's needed
    entries from their owners' extended vectors, the all-reduce adds the
    ranks' sums in rank order and gives every rank the total."""

    def exchange(self, ranks, which: str):
        if len(ranks) == 1:
            return
        for rk in ranks:
            plan = rk.plan
            v = rk.ext(which)
            if plan.mode == ALLGATHER:
                for q, other in enumerate(ranks):
                    if q != plan.rank:
                        o = other.plan.own
                        v[o: o + other.plan.chunk] = other.ext(which)[o: o + other.plan.chunk]
                continue
            for q, (off, cnt) in plan.recv.items():
                v[off:off + cnt] = ranks[q].send_view(which, plan.rank)

    def allreduce(self, ranks, k: int):
        if len(ranks) == 1:
            return
        self.allreduce_tensors([rk.sums[:k] for rk in ranks])

    def world(self, items):
        return len(items)

    def ranks(self, items):
        return list(range(len(items)))

    def allreduce_tensors(self, tensors):
        if len(tensors) == 1:
            return
        tot = tensors[0].clone()
        for t in tensors[1:]:
            tot += t
        for t in tensors:
            t.copy_(tot)

    def allreduce_host(self, t: torch.Tensor) -> torch.Tensor:
        return t


# ---------------------------------------------------------------- the solve

def dist_cg(ranks, comm, xs, bs, scs, check_every: int = 8):
    """Row-partitioned CG over `ranks` (each with its x, b and solver control
    in xs, bs, scs). Every rank runs the same stages in the same order and
    reads its state at the same steps. Returns the solver info of the first
    rank (all ranks agree)."""
    for rk, x, b in zip(ranks, xs, bs):
        rk.start(x, b)
    comm.exchange(ranks, "x")
    for rk in ranks:
        rk.residual()
    comm.exchange(ranks, "z")
    for rk in ranks:
        rk.product()
    comm.allreduce(ranks, 4)
    max_iters = max(sc.max_iters for sc in scs)
    step = 0
    while True:
        for rk, sc in zip(ranks, scs):
            rk.update(step, sc)
        step += 1
        if step % check_every == 0 or step > max_iters + 1:
            states = [rk.state(sc) for rk, sc in zip(ranks, scs)]
            if all(d for d, _ in states):
                return states[0][1]
            if any(d for d, _ in states):
                raise RuntimeError("ranks disagree on the stop decision")
            if step > max_iters + 2 + check_every:
                raise RuntimeError("row-partitioned CG did not stop at the iteration limit")
        comm.exchange(ranks, "z")
        for rk in ranks:
            rk.product()
        comm.allreduce(ranks, 3)


def setup_local(rp, col, val, parts, rank: int, plan: Plan):
    """(rp, ext columns, values) of `rank`'s rows under `plan`."""
    r0, r1 = parts[rank]
    lrp, lcol, lval = local_rows(rp, col, val, r0, r1)
    return lrp, plan.ext_columns(lcol), lval


def plan_for_rank(lcol_global, parts, rank: int, group=None, mode: str | None = None):
    """This rank's plan in a torch.distributed job: the ranks' needed columns
    are gathered so that every rank derives the same plans."""
    r0, r1 = parts[rank]
    mine = needed_columns(lcol_global, r0, r1)
    world = len(parts)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    return make_plans(gathered, parts, mode)[rank]


# ---------------------------------------------------------------- training

class DeviceNet:
    """One rank's network for data-parallel training (api.Spai on its GPU)."""

    def __init__(self, spai, ctrl):
        self.spai, self.ctrl = spai, ctrl

    def loss_grad(self, sample):
        """Loss of `sample` (an object with A and probes); the gradient stays
        in grad()."""
        self.spai.set_matrix(sample.A, self.ctrl)
        return self.spai.loss_grad_device(self.ctrl, sample.probes, self.lam)

    def grad(self) -> torch.Tensor:
        return self.spai.grad_buffer()

    def adam_step(self, lr, scale):
        self.spai.adam_step(self.ctrl, lr, scale)


def dp_train(nets, comm, samples, steps: int, lr: float, lam: float = 0.2):
    """Data-parallel training: at step t rank r takes sample (t * world + r)
    mod len(samples), every rank's gradient is summed over the ranks (one
    all-reduce of the FP32 gradient, in place on the device) and each rank
    applies the same Adam step to the mean, so the replicas stay identical.
    nets: this process's rank(s) (one per process with TorchComm; all with
    LocalComm). Returns the mean loss per step."""
    world = comm.world(nets)
    ranks = comm.ranks(nets)
    losses = []
    for net in nets:
        net.lam = lam
    for t in range(steps):
        ls = torch.zeros(1, dtype=torch.float64)
        for net, r in zip(nets, ranks):
            ls += net.loss_grad(samples[(t * world + r) % len(samples)])
        comm.allreduce_tensors([net.grad() for net in nets])
        ls = comm.allreduce_host(ls)
        lr_t = lr * (0.1 ** (t / max(steps, 1)))
        for net in nets:
            net.adam_step(lr_t, 1.0 / world)
        losses.append(float(ls) / world)
    return losses


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
