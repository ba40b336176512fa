"""Python mirror of the clSPARSE C API over torch device tensors.

Each function here is a thin call through the C ABI (clsparse_b200._lib): the
arguments are packed into the reference's structs (clsparseCsrMatrix,
cldenseVector, clsparseScalar) pointing at torch CUDA storage, and a non-zero
clsparseStatus raises ClsparseError. Names follow the reference API
(src/include/clSPARSE.h). torch only provides device memory and the stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L


class ClsparseError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what} failed with clsparseStatus {status}")
        self.status = status


def lib():
    return L.load()


def check(status: int, what: str):
    if int(status) != L.clsparseSuccess:
        raise ClsparseError(int(status), what)


def setup():
    check(lib().clsparseSetup(), "clsparseSetup")


def teardown():
    check(lib().clsparseTeardown(), "clsparseTeardown")


def _dtype_prefix(t: torch.Tensor) -> str:
    if t.dtype == torch.float64:
        return "D"
    if t.dtype == torch.float32:
        return "S"
    raise TypeError(f"unsupported value dtype {t.dtype}")


class Control:
    """clsparseControl bound to a CUDA stream (default: torch's current stream)."""

    def __init__(self, stream: torch.cuda.Stream | None = None):
        setup()
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        res = lib().clsparseCreateControl(C.c_void_p(self.stream.cuda_stream))
        check(res.status, "clsparseCreateControl")
        self.handle = res.control

    def enable_async(self, on: bool = True):
        check(lib().clsparseEnableAsync(self.handle, 1 if on else 0), "clsparseEnableAsync")

    def enable_extended_precision(self, on: bool = True):
        check(lib().clsparseEnableExtendedPrecision(self.handle, 1 if on else 0),
              "clsparseEnableExtendedPrecision")

    def set_solver_loop_mode(self, mode: int):
        check(lib().clsparseB200SetSolverLoopMode(self.handle, mode), "clsparseB200SetSolverLoopMode")

    def release(self):
        if self.handle:
            check(lib().clsparseReleaseControl(self.handle), "clsparseReleaseControl")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()


def vector(t: torch.Tensor, offset: int = 0, num_values: int | None = None) -> L.cldenseVector:
    n = t.numel() - offset if num_values is None else num_values
    return L.cldenseVector(n, C.c_void_p(t.data_ptr()), offset)


def scalar(t: torch.Tensor, offset: int = 0) -> L.clsparseScalar:
    return L.clsparseScalar(C.c_void_p(t.data_ptr()), offset)


class CsrMatrix:
    """A clsparseCsrMatrix over torch tensors (row_ptr / col as int32 storage of
    the uint32 indices, values float32 or float64)."""

    def __init__(self, row_ptr: torch.Tensor, col: torch.Tensor, val: torch.Tensor, num_cols: int):
        self.row_ptr, self.col, self.val = row_ptr, col, val
        self.s = L.clsparseCsrMatrix()
        lib().clsparseInitCsrMatrix(C.byref(self.s))
        self.s.num_rows = row_ptr.numel() - 1
        self.s.num_cols = num_cols
        self.s.num_nonzeros = val.numel()
        self.s.values = C.c_void_p(val.data_ptr()) if val.numel() else None
        self.s.col_indices = C.c_void_p(col.data_ptr()) if col.numel() else None
        self.s.row_pointer = C.c_void_p(row_ptr.data_ptr())

    @classmethod
    def from_numpy(cls, rp, col, val, num_cols=None, dtype=torch.float64, device="cuda"):
        rp = np.asarray(rp, dtype=np.uint32)
        col = np.asarray(col, dtype=np.uint32)
        ncols = (len(rp) - 1) if num_cols is None else num_cols
        t_rp = torch.from_numpy(rp.view(np.int32).copy()).to(device)
        t_col = torch.from_numpy(col.view(np.int32).copy()).to(device)
        t_val = torch.from_numpy(np.asarray(val)).to(device=device, dtype=dtype)
        return cls(t_rp, t_col, t_val, ncols)

    @classmethod
    def from_file(cls, path, ctrl: "Control", dtype=torch.float64, read_explicit_zeroes: bool = False):
        """clsparseHeaderfromFile + clsparse{S,D}CsrMatrixfromFile into new
        device tensors (allocated with the header's sizes)."""
        nnz, nr, nc = L.clsparseIdx_t(), L.clsparseIdx_t(), L.clsparseIdx_t()
        check(lib().clsparseHeaderfromFile(C.byref(nnz), C.byref(nr), C.byref(nc), str(path).encode()),
              "clsparseHeaderfromFile")
        rp = torch.zeros(nr.value + 1, dtype=torch.int32, device="cuda")
        col = torch.zeros(max(nnz.value, 1), dtype=torch.int32, device="cuda")
        val = torch.zeros(max(nnz.value, 1), dtype=dtype, device="cuda")
        m = cls(rp, col, val, nc.value)
        fn = "clsparseDCsrMatrixfromFile" if dtype == torch.float64 else "clsparseSCsrMatrixfromFile"
        check(getattr(lib(), fn)(C.byref(m.s), str(path).encode(), ctrl.handle, 1 if read_explicit_zeroes else 0), fn)
        k = m.s.num_nonzeros
        m.col, m.val = m.col[:k], m.val[:k]
        return m

    @property
    def num_rows(self):
        return self.s.num_rows

    @property
    def num_cols(self):
        return self.s.num_cols

    @property
    def nnz(self):
        return self.s.num_nonzeros

    def meta_size(self, ctrl: Control) -> int:
        r = lib().clsparseCsrMetaSize(C.byref(self.s), ctrl.handle)
        check(r.status, "clsparseCsrMetaSize")
        return int(r.metaSize)

    def create_meta(self, ctrl: Control, shape=None):
        """CSR-Adaptive meta; shape = (blk_size, blk_multiplier, rows_for_vector,
        cta_threads) for clsparseB200CsrMetaCreateTuned, None for the
        reference's shape (clsparseCsrMetaCreate)."""
        if shape is None:
            check(lib().clsparseCsrMetaCreate(C.byref(self.s), ctrl.handle), "clsparseCsrMetaCreate")
        else:
            if self.s.meta:
                self.delete_meta()
            blk, mult, rfv, nt = (int(v) for v in shape)
            check(lib().clsparseB200CsrMetaCreateTuned(C.byref(self.s), blk, mult, rfv, nt, ctrl.handle),
                  "clsparseB200CsrMetaCreateTuned")

    def delete_meta(self):
        check(lib().clsparseCsrMetaDelete(C.byref(self.s)), "clsparseCsrMetaDelete")

    def row_blocks(self) -> np.ndarray:
        n = C.c_size_t()
        check(lib().clsparseB200CsrMetaGetRowBlocks(C.byref(self.s), None, 0, C.byref(n)), "GetRowBlocks")
        out = np.zeros(n.value, dtype=np.uint64)
        check(lib().clsparseB200CsrMetaGetRowBlocks(C.byref(self.s), out.ctypes.data_as(C.POINTER(L.cl_ulong)),
                                                    n.value, C.byref(n)), "GetRowBlocks")
        return out

    def __del__(self):
        try:
            if self.s.meta:
                lib().clsparseCsrMetaDelete(C.byref(self.s))
        except Exception:
            pass


def csrmv(alpha: torch.Tensor, A: CsrMatrix, x: torch.Tensor, beta: torch.Tensor, y: torch.Tensor,
          ctrl: Control, x_off: int = 0, y_off: int = 0):
    """y = alpha*A*x + beta*y through clsparse{S,D}csrmv."""
    p = _dtype_prefix(A.val)
    fn = getattr(lib(), f"clsparse{p}csrmv")
    xv = vector(x, x_off)
    yv = vector(y, y_off)
    check(fn(C.byref(scalar(alpha)), C.byref(A.s), C.byref(xv), C.byref(scalar(beta)), C.byref(yv),
             ctrl.handle), f"clsparse{p}csrmv")


class SolverControl:
    def __init__(self, precond: int = L.DIAGONAL, max_iters: int = 100, rel_tol: float = 1e-2,
                 abs_tol: float = 1e-5):
        r = lib().clsparseCreateSolverControl(precond, max_iters, rel_tol, abs_tol)
        check(r.status, "clsparseCreateSolverControl")
        self.handle = r.control
        self.max_iters = int(max_iters)

    def set_params(self, precond, max_iters, rel_tol, abs_tol):
        check(lib().clsparseSetSolverParams(self.handle, precond, max_iters, rel_tol, abs_tol),
              "clsparseSetSolverParams")
        self.max_iters = int(max_iters)

    def print_mode(self, mode):
        check(lib().clsparseSolverPrintMode(self.handle, mode), "clsparseSolverPrintMode")

    def info(self):
        it = L.cl_int()
        r0 = C.c_double()
        r1 = C.c_double()
        check(lib().clsparseB200SolverGetInfo(self.handle, C.byref(it), C.byref(r0), C.byref(r1)), "GetInfo")
        return {"nIters": it.value, "initialResidual": r0.value, "currentResidual": r1.value}

    def set_norm(self, norm: int):
        """1: the reference's ||r||_1/||b||_1 stop test, 2: ||r||_2/||b||_2."""
        check(lib().clsparseB200SolverSetNormType(self.handle, norm), "clsparseB200SolverSetNormType")

    def set_history(self, hist: torch.Tensor | None):
        """Records the residuum of the start and of every iteration of the
        next solves into the FP64 device tensor hist (None: off)."""
        if hist is None:
            check(lib().clsparseB200SolverSetHistory(self.handle, None, 0), "clsparseB200SolverSetHistory")
            return
        assert hist.dtype == torch.float64 and hist.is_cuda and hist.is_contiguous()
        self._hist = hist
        check(lib().clsparseB200SolverSetHistory(self.handle, C.c_void_p(hist.data_ptr()), hist.numel()),
              "clsparseB200SolverSetHistory")

    def history_length(self) -> int:
        n = L.cl_uint()
        check(lib().clsparseB200SolverGetHistoryLength(self.handle, C.byref(n)), "GetHistoryLength")
        return n.value

    def set_snapshots(self, iterations, vectors: torch.Tensor | None):
        """Keeps the CG residual vector after each listed iteration count in
        the rows of vectors (len(iterations) x n, the solve's dtype)."""
        if vectors is None or not len(iterations):
            check(lib().clsparseB200SolverSetSnapshots(self.handle, None, 0, None), "clsparseB200SolverSetSnapshots")
            return
        assert vectors.is_cuda and vectors.is_contiguous() and vectors.shape[0] == len(iterations)
        self._snap = vectors
        its = (L.cl_int * len(iterations))(*[int(k) for k in iterations])
        check(lib().clsparseB200SolverSetSnapshots(self.handle, its, len(iterations), C.c_void_p(vectors.data_ptr())),
              "clsparseB200SolverSetSnapshots")

    def device_status(self) -> int:
        b = L.cl_uint()
        check(lib().clsparseB200SolverGetDeviceStatus(self.handle, C.byref(b)), "GetDeviceStatus")
        return b.value

    def release(self):
        if self.handle:
            check(lib().clsparseReleaseSolverControl(self.handle), "clsparseReleaseSolverControl")
            self.handle = None


def solve(kind: str, x: torch.Tensor, A: CsrMatrix, b: torch.Tensor, sc: SolverControl, ctrl: Control):
    """kind 'cg' -> clsparse{S,D}csrcg, 'bicgstab' -> clsparse{S,D}csrbicgStab."""
    p = _dtype_prefix(A.val)
    name = f"clsparse{p}csrcg" if kind == "cg" else f"clsparse{p}csrbicgStab"
    fn = getattr(lib(), name)
    st = fn(C.byref(vector(x)), C.byref(A.s), C.byref(vector(b)), sc.handle, ctrl.handle)
    check(st, name)
    return sc.info()


def cg_mixed(x: torch.Tensor, A: CsrMatrix, b: torch.Tensor, sc: SolverControl, ctrl: Control,
             inner: str = "fp32", inner_tol: float = 1e-4) -> dict:
    """FP64 iterative refinement with FP32- or BF16-valued inner CG
    (clsparseDcsrcgMixed); returns the refinement statistics."""
    info = L.clsparseB200MixedInfo()
    prec = {"fp32": 0, "bf16": 1}[inner]
    check(lib().clsparseDcsrcgMixed(C.byref(vector(x)), C.byref(A.s), C.byref(vector(b)), sc.handle, prec,
                                    inner_tol, C.byref(info), ctrl.handle), "clsparseDcsrcgMixed")
    return {f[0]: getattr(info, f[0]) for f in info._fields_}


def bicgstab_mixed(x: torch.Tensor, A: CsrMatrix, b: torch.Tensor, sc: SolverControl, ctrl: Control,
                   inner: str = "fp32", inner_tol: float = 1e-4) -> dict:
    """FP64 iterative refinement with an FP32- or BF16-valued inner BiCGStab
    (clsparseDcsrbicgStabMixed); returns the refinement statistics."""
    info = L.clsparseB200MixedInfo()
    prec = {"fp32": 0, "bf16": 1}[inner]
    check(lib().clsparseDcsrbicgStabMixed(C.byref(vector(x)), C.byref(A.s), C.byref(vector(b)), sc.handle, prec,
                                          inner_tol, C.byref(info), ctrl.handle), "clsparseDcsrbicgStabMixed")
    return {f[0]: getattr(info, f[0]) for f in info._fields_}


def read_mtx_host(path, read_explicit_zeroes: bool = False):
    """A Matrix Market file as host CSR (rp, col, val) via
    clsparseB200ReadMatrixMarketHost (no GPU)."""
    nr, nc, nnz = L.clsparseIdx_t(), L.clsparseIdx_t(), L.clsparseIdx_t()
    p = str(path).encode()
    z = 1 if read_explicit_zeroes else 0
    check(lib().clsparseB200ReadMatrixMarketHost(p, z, C.byref(nr), C.byref(nc), C.byref(nnz), None, None, None, 0),
          "clsparseB200ReadMatrixMarketHost")
    rp = np.zeros(nr.value + 1, dtype=np.uint32)
    col = np.zeros(max(nnz.value, 1), dtype=np.uint32)
    val = np.zeros(max(nnz.value, 1), dtype=np.float64)
    check(lib().clsparseB200ReadMatrixMarketHost(
        p, z, C.byref(nr), C.byref(nc), C.byref(nnz), rp.ctypes.data_as(C.POINTER(L.clsparseIdx_t)),
        col.ctypes.data_as(C.POINTER(L.clsparseIdx_t)), val.ctypes.data_as(C.POINTER(C.c_double)), len(col)),
        "clsparseB200ReadMatrixMarketHost")
    return rp, col[: nnz.value], val[: nnz.value], nc.value


def blas1(name: str, *args, ctrl: Control):
    """Calls a cldense* entry point; tensors become vectors, 1-element tensors
    passed as ('s', t) become scalars."""
    conv = []
    for a in args:
        if isinstance(a, tuple) and a[0] == "s":
            conv.append(C.byref(scalar(a[1])))
        else:
            conv.append(C.byref(vector(a)))
    check(getattr(lib(), name)(*conv, ctrl.handle), name)


def cg_batched(x: torch.Tensor, A: CsrMatrix, b: torch.Tensor, offsets, sc: SolverControl, ctrl: Control,
               lanes=None) -> dict:
    """Batched FP32 Jacobi-CG over the block-diagonal systems of A
    (clsparseScsrcgBatched). offsets: numpy/sequence of num_systems+1 row offsets."""
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    nsys = len(off) - 1
    iters = np.zeros(nsys, dtype=np.int32)
    res = np.zeros(nsys, dtype=np.float64)
    out = L.clsparseB200BatchResult(iters.ctypes.data_as(C.POINTER(L.cl_int)),
                                    res.ctypes.data_as(C.POINTER(C.c_double)), 0, 0, 0.0)
    lp = None
    if lanes is not None:
        lanes = np.ascontiguousarray(lanes, dtype=np.int32)
        lp = lanes.ctypes.data_as(C.POINTER(L.cl_int))
    check(lib().clsparseScsrcgBatched(C.byref(vector(x)), C.byref(A.s), C.byref(vector(b)),
                                      off.ctypes.data_as(C.POINTER(L.clsparseIdx_t)), nsys, lp, sc.handle,
                                      C.byref(out), ctrl.handle), "clsparseScsrcgBatched")
    return {"iterations": iters, "residuals": res, "converged": out.systemsConverged,
            "max_iterations": out.maxIterations, "worst_residual": out.worstResidual}


class Spai:
    """The learned factorized sparse approximate inverse (clsparseB200Spai*)."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        check(lib().clsparseB200SpaiCreate(C.byref(h), seed), "clsparseB200SpaiCreate")
        self.handle = h

    def set_matrix(self, A: CsrMatrix, ctrl: Control):
        check(lib().clsparseB200SpaiSetMatrix(self.handle, C.byref(A.s), ctrl.handle), "clsparseB200SpaiSetMatrix")
        self._A = A

    def params(self) -> np.ndarray:
        n = C.c_size_t()
        check(lib().clsparseB200SpaiParams(self.handle, None, 0, C.byref(n), 0), "SpaiParams")
        out = np.zeros(n.value, dtype=np.float32)
        check(lib().clsparseB200SpaiParams(self.handle, out.ctypes.data_as(C.POINTER(C.c_float)), n.value,
                                           C.byref(n), 0), "SpaiParams")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        n = C.c_size_t()
        check(lib().clsparseB200SpaiParams(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size,
                                           C.byref(n), 1), "SpaiParams")

    def _probes(self, probes):
        if probes is None:
            return None, 0
        t = probes.reshape(-1).contiguous()
        return C.byref(vector(t)), int(probes.shape[0])

    def loss_grad(self, ctrl: Control, probes: torch.Tensor | None = None, lam: float = 0.0,
                  fp32_weights: bool = False):
        pv, K = self._probes(probes)
        loss = C.c_double()
        g = np.zeros(self.params().size, dtype=np.float32)
        check(lib().clsparseB200SpaiLossGrad(self.handle, pv, K, lam, 1 if fp32_weights else 0, C.byref(loss),
                                             g.ctypes.data_as(C.POINTER(C.c_float)), g.size, ctrl.handle),
              "clsparseB200SpaiLossGrad")
        return loss.value, g

    def train_step(self, ctrl: Control, probes: torch.Tensor | None = None, lam: float = 0.0,
                   lr: float = 1e-3) -> float:
        pv, K = self._probes(probes)
        loss = C.c_double()
        check(lib().clsparseB200SpaiTrainStep(self.handle, pv, K, lam, lr, C.byref(loss), ctrl.handle),
              "clsparseB200SpaiTrainStep")
        return loss.value

    def loss_grad_device(self, ctrl: Control, probes: torch.Tensor | None = None, lam: float = 0.0) -> float:
        """Loss and gradient at the current weights, the gradient left in the
        network's device buffer (grad_buffer) with no host copy."""
        pv, K = self._probes(probes)
        loss = C.c_double()
        check(lib().clsparseB200SpaiLossGrad(self.handle, pv, K, lam, 0, C.byref(loss), None, 0, ctrl.handle),
              "clsparseB200SpaiLossGrad")
        return loss.value

    def grad_buffer(self) -> torch.Tensor:
        """The device gradient buffer as a float32 tensor (a view)."""
        p = C.POINTER(C.c_float)()
        n = C.c_size_t()
        check(lib().clsparseB200SpaiGradient(self.handle, C.byref(p), C.byref(n)), "clsparseB200SpaiGradient")

        class _View:
            pass
        v = _View()
        v.__cuda_array_interface__ = {"shape": (n.value,), "typestr": "<f4",
                                      "data": (C.cast(p, C.c_void_p).value, False), "version": 3, "strides": None}
        return torch.as_tensor(v, device="cuda")

    def adam_step(self, ctrl: Control, lr: float, grad_scale: float = 1.0):
        check(lib().clsparseB200SpaiAdamStep(self.handle, lr, grad_scale, ctrl.handle), "clsparseB200SpaiAdamStep")

    def build(self, ctrl: Control):
        check(lib().clsparseB200SpaiBuild(self.handle, ctrl.handle), "clsparseB200SpaiBuild")

    def factor(self):
        nnz = C.c_size_t()
        check(lib().clsparseB200SpaiGetFactor(self.handle, None, None, None, 0, C.byref(nnz)), "GetFactor")
        n = self._A.num_rows
        rp = np.zeros(n + 1, dtype=np.uint32)
        col = np.zeros(nnz.value, dtype=np.uint32)
        val = np.zeros(nnz.value, dtype=np.float64)
        check(lib().clsparseB200SpaiGetFactor(self.handle, rp.ctypes.data_as(C.POINTER(L.clsparseIdx_t)),
                                              col.ctypes.data_as(C.POINTER(L.clsparseIdx_t)),
                                              val.ctypes.data_as(C.POINTER(C.c_double)), nnz.value, C.byref(nnz)),
              "GetFactor")
        return rp, col, val

    def save(self, path: str):
        check(lib().clsparseB200SpaiSave(self.handle, str(path).encode()), "clsparseB200SpaiSave")

    def load(self, path: str):
        check(lib().clsparseB200SpaiLoad(self.handle, str(path).encode()), "clsparseB200SpaiLoad")

    def release(self):
        if self.handle:
            check(lib().clsparseB200SpaiRelease(self.handle), "clsparseB200SpaiRelease")
            self.handle = None


def cg_learned(x: torch.Tensor, A: CsrMatrix, b: torch.Tensor, sc: SolverControl, spai: Spai, ctrl: Control,
               inner: str = "fp32", inner_tol: float = 1e-3) -> dict:
    """CG preconditioned with the learned G^T G (clsparseDcsrcgLearned)."""
    info = L.clsparseB200MixedInfo()
    fb = L.cl_int()
    prec = {"fp32": 0, "bf16": 1, "fp64": 2}[inner]
    check(lib().clsparseDcsrcgLearned(C.byref(vector(x)), C.byref(A.s), C.byref(vector(b)), sc.handle,
                                      spai.handle, prec, inner_tol, C.byref(info), C.byref(fb), ctrl.handle),
          "clsparseDcsrcgLearned")
    out = {f[0]: getattr(info, f[0]) for f in info._fields_}
    out["fell_back"] = fb.value
    return out
