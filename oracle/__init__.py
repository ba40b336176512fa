"""CPU oracle of the clSPARSE hot path -- test infrastructure only.

Python side of oracle/oracle.c (the project's C restatement of the reference
algorithms), of oracle/_ref/librefbins.so (the reference's own
ComputeRowBlocks compiled from its sources) and of oracle/_ref/librefspmv.so
(the reference's own SpMV kernels, csrmv_adaptive.cl and csrmv_general.cl,
compiled from its sources and run on host threads through oracle/clc_shim.h). Only tests, __graft_entry__.smoke()
and bench.py's CPU baseline use this package, as the checker or the timed CPU
baseline; the product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None
_ref = None
_refspmv = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


class SolveInfo(C.Structure):
    _fields_ = [("nIters", C.c_int), ("zero_b", C.c_int), ("initialResidual", C.c_double),
                ("currentResidual", C.c_double), ("relTol", C.c_double), ("absTol", C.c_double)]


def build():
    """Builds liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.oracle_row_blocks.restype = C.c_uint32
        L.oracle_row_blocks.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]
        L.oracle_dcsrmv.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, C.c_double, _f64p, C.c_double, _f64p]
        L.oracle_scsrmv.argtypes = [C.c_uint32, _u32p, _u32p, _f32p, C.c_float, _f32p, C.c_float, _f32p]
        L.oracle_dcsrmv_absscale.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, C.c_double, _f64p,
                                             C.c_double, _f64p, _f64p]
        L.oracle_dcsrmv_mt.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, C.c_double, _f64p, C.c_double,
                                       _f64p, C.c_int]
        L.oracle_dcg_mt.restype = C.c_int
        L.oracle_dcg_mt.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, _f64p, _f64p, C.c_int, C.c_double, C.c_int,
                                    C.POINTER(C.c_double)]
        for sfx, fp in (("d", _f64p), ("s", _f32p)):
            for name in (f"oracle_{sfx}cg", f"oracle_{sfx}bicgstab"):
                f = getattr(L, name)
                f.restype = C.c_int
                f.argtypes = [C.c_uint32, _u32p, _u32p, fp, fp, fp, C.c_int, C.c_int, C.c_double,
                              C.c_double, C.c_int, C.POINTER(SolveInfo)]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own binning, or None where oracle/_ref was not built."""
    global _ref
    if _ref is None:
        path = HERE / "_ref" / "librefbins.so"
        if not path.exists():
            return None
        L = C.CDLL(str(path))
        L.ref_row_blocks_size.restype = C.c_uint32
        L.ref_row_blocks_size.argtypes = [_u32p, C.c_uint32]
        L.ref_row_blocks.restype = C.c_uint32
        L.ref_row_blocks.argtypes = [_u32p, C.c_uint32, _u64p, C.c_uint32]
        L.ref_row_blocks_shape_size.restype = C.c_uint32
        L.ref_row_blocks_shape_size.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.ref_row_blocks_shape.restype = C.c_uint32
        L.ref_row_blocks_shape.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _u64p,
                                           C.c_uint32]
        _ref = L
    return _ref


def row_blocks(rp: np.ndarray, shape=(1024, 3, 1)):
    """Row-block words and rowBlockSize of the oracle restatement; shape =
    (BLKSIZE, BLOCK_MULTIPLIER, ROWS_FOR_VECTOR), the reference's by default."""
    rp = np.ascontiguousarray(rp, dtype=np.uint32)
    n = len(rp) - 1
    L = lib()
    blk, mult, rfv = (int(v) for v in shape[:3])
    dry = L.oracle_row_blocks(rp, n, blk, mult, rfv, None)
    words = np.zeros(dry // 2 + 1, dtype=np.uint64)
    size = L.oracle_row_blocks(rp, n, blk, mult, rfv, words.ctypes.data)
    return words[: size // 2].copy(), size, dry


def ref_row_blocks(rp: np.ndarray, shape=None):
    """Row-block words and rowBlockSize of the reference's own ComputeRowBlocks
    (its compiled-in shape, or shape = (BLKSIZE, BLOCK_MULTIPLIER, ROWS_FOR_VECTOR))."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/librefbins.so not built (reference tree absent)")
    rp = np.ascontiguousarray(rp, dtype=np.uint32)
    n = len(rp) - 1
    if shape is None:
        dry = L.ref_row_blocks_size(rp, n)
        words = np.zeros(dry // 2 + 1, dtype=np.uint64)
        size = L.ref_row_blocks(rp, n, words, dry // 2 + 1)
    else:
        blk, mult, rfv = (int(v) for v in shape[:3])
        dry = L.ref_row_blocks_shape_size(rp, n, blk, mult, rfv)
        words = np.zeros(dry // 2 + 1, dtype=np.uint64)
        size = L.ref_row_blocks_shape(rp, n, blk, mult, rfv, words, dry // 2 + 1)
    return words[: size // 2].copy(), size, dry


def dcsrmv(rp, col, val, alpha, x, beta, y):
    y = np.array(y, dtype=np.float64, copy=True)
    lib().oracle_dcsrmv(len(rp) - 1, _u32(rp), _u32(col), np.ascontiguousarray(val, np.float64),
                        float(alpha), np.ascontiguousarray(x, np.float64), float(beta), y)
    return y


def scsrmv(rp, col, val, alpha, x, beta, y):
    y = np.array(y, dtype=np.float32, copy=True)
    lib().oracle_scsrmv(len(rp) - 1, _u32(rp), _u32(col), np.ascontiguousarray(val, np.float32),
                        float(alpha), np.ascontiguousarray(x, np.float32), float(beta), y)
    return y


def dcsrmv_absscale(rp, col, val, alpha, x, beta, y):
    out = np.zeros(len(rp) - 1, dtype=np.float64)
    lib().oracle_dcsrmv_absscale(len(rp) - 1, _u32(rp), _u32(col), np.ascontiguousarray(val, np.float64),
                                 float(alpha), np.ascontiguousarray(x, np.float64), float(beta),
                                 np.ascontiguousarray(y, np.float64), out)
    return out


def dcsrmv_mt(rp, col, val, alpha, x, beta, y, threads):
    lib().oracle_dcsrmv_mt(len(rp) - 1, rp, col, val, float(alpha), x, float(beta), y, int(threads))
    return y


def reference_solution(rp, col, val, b, rel_tol=1e-12, max_iters=1_000_000, threads=None):
    """FP64 Jacobi-PCG (oracle_dcg_mt: the reference CG's operation order on a
    pool of host threads, L2 stop test) from x = 0 to ||b - A x||_2 / ||b||_2
    <= rel_tol. Returns (x, iterations, final relative residual of the
    recursion). Used as the FP64 oracle solution of the large configurations."""
    import os
    n = len(rp) - 1
    x = np.zeros(n)
    res = C.c_double(0.0)
    it = lib().oracle_dcg_mt(n, np.ascontiguousarray(rp, np.uint32), np.ascontiguousarray(col, np.uint32),
                             np.ascontiguousarray(val, np.float64), x, np.ascontiguousarray(b, np.float64),
                             int(max_iters), float(rel_tol), int(threads or os.cpu_count() or 1), C.byref(res))
    return x, it, res.value


def ref_spmv_lib():
    """The reference's own SpMV kernels run on the host (oracle/_ref/librefspmv.so,
    built by oracle/Makefile from src/library/kernels/csrmv_{adaptive,general}.cl),
    or None where oracle/_ref was not built."""
    global _refspmv
    if _refspmv is None:
        path = HERE / "_ref" / "librefspmv.so"
        if not path.exists():
            return None
        _refspmv = C.CDLL(str(path))
    return _refspmv


def _tag(dtype, extended):
    return ("d" if np.dtype(dtype) == np.float64 else "s") + ("_ext" if extended else "_plain")


def ref_csrmv_adaptive(rp, col, val, x, y, alpha, beta, dtype=np.float64, extended=False):
    """y = alpha*A*x + beta*y by the reference's csrmv_adaptive kernel
    (csrmv_adaptive.cl:312-687) with the row blocks of the reference's own
    ComputeRowBlocks; returns the new y (a copy). Work-groups run one after
    another on host threads, so large matrices take seconds."""
    L, R = ref_spmv_lib(), ref_lib()
    if L is None or R is None:
        raise RuntimeError("oracle/_ref not built")
    t = np.dtype(dtype)
    rp = np.ascontiguousarray(rp, np.uint32)
    n = len(rp) - 1
    dry = R.ref_row_blocks_size(rp, n)
    words = np.zeros(dry // 2 + 1, np.uint64)
    used = R.ref_row_blocks(rp, n, words, len(words))
    meta = np.zeros(max(dry, used) + 2, np.uint64)  # the reference's meta buffer: words, then error slots
    meta[: used // 2] = words[: used // 2]
    pad = 1024  # BLOCKSIZE: the stream loads read up to a block past the last nonzero
    cols = np.concatenate([np.asarray(col, np.uint32), np.zeros(pad, np.uint32)])
    vals = np.concatenate([np.asarray(val, t), np.zeros(pad, t)])
    xv = np.ascontiguousarray(x, t)
    yv = np.array(y, dtype=t, copy=True)
    a = np.array([alpha], t)
    b = np.array([beta], t)
    fn = getattr(L, "ref_csrmv_adaptive_" + _tag(t, extended))
    fn.restype = C.c_int
    rc = fn(vals.ctypes.data_as(C.c_void_p), cols.ctypes.data_as(C.c_void_p), rp.ctypes.data_as(C.c_void_p),
            xv.ctypes.data_as(C.c_void_p), yv.ctypes.data_as(C.c_void_p), meta.ctypes.data_as(C.c_void_p),
            C.c_uint(used), a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise RuntimeError(f"reference kernel launch failed ({rc})")
    return yv


def ref_subwave(nnz, nrows, wave_size=64):
    """The sub-wave width the reference's csrmv_vector picks from the average
    row length (csrmv-vector.hpp:34-49)."""
    per_row = nnz // nrows if nrows else 0
    sw = wave_size
    if wave_size > 32 and per_row < 64:
        sw = 32
    if per_row < 32:
        sw = 16
    if per_row < 16:
        sw = 8
    if per_row < 8:
        sw = 4
    if per_row < 4:
        sw = 2
    return sw


def ref_csrmv_general(rp, col, val, x, y, alpha, beta, dtype=np.float64, extended=False, subwave=None):
    """y = alpha*A*x + beta*y by the reference's csrmv_general kernel
    (csrmv_general.cl:178-259), the path it takes without a meta; returns the
    new y (a copy)."""
    L = ref_spmv_lib()
    if L is None:
        raise RuntimeError("oracle/_ref not built")
    t = np.dtype(dtype)
    rp = np.ascontiguousarray(rp, np.uint32)
    n = len(rp) - 1
    sw = subwave or ref_subwave(int(rp[-1] - rp[0]), n)
    cols = np.ascontiguousarray(col, np.uint32)
    vals = np.ascontiguousarray(val, t)
    xv = np.ascontiguousarray(x, t)
    yv = np.array(y, dtype=t, copy=True)
    a = np.array([alpha], t)
    b = np.array([beta], t)
    fn = getattr(L, f"ref_csrmv_general_{_tag(t, extended)}_sw{sw}")
    fn.restype = C.c_int
    rc = fn(C.c_uint(n), rp.ctypes.data_as(C.c_void_p), cols.ctypes.data_as(C.c_void_p),
            vals.ctypes.data_as(C.c_void_p), xv.ctypes.data_as(C.c_void_p), yv.ctypes.data_as(C.c_void_p),
            a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise RuntimeError(f"reference kernel launch failed ({rc})")
    return yv


def solve(kind, dtype, rp, col, val, x0, b, precond, max_iters, rel_tol, abs_tol, n_iters_in=0):
    """Runs oracle CG ('cg') or BiCGStab ('bicgstab') in float32 or float64."""
    sfx = "d" if np.dtype(dtype) == np.float64 else "s"
    fn = getattr(lib(), f"oracle_{sfx}{kind}")
    x = np.array(x0, dtype=dtype, copy=True)
    info = SolveInfo()
    fn(len(rp) - 1, _u32(rp), _u32(col), np.ascontiguousarray(val, dtype), x,
       np.ascontiguousarray(b, dtype), int(precond), int(max_iters), float(rel_tol), float(abs_tol),
       int(n_iters_in), C.byref(info))
    return x, info


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)
