"""CPU oracle of the clSPARSE hot path -- test infrastructure only.

Python side of oracle/oracle.c (the project's C restatement of the reference
algorithms) and of oracle/_ref/librefbins.so (the reference's own
ComputeRowBlocks compiled from its sources). Only tests, __graft_entry__.smoke()
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
