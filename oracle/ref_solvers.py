"""The reference's CG and BiCGStab run on the host with the reference's OWN
kernels -- TEST INFRASTRUCTURE ONLY (fixture generation; the product never
imports it).

The reference's solvers are host C++ (src/library/solvers/
conjugate-gradients.hpp:47-228, biconjugate-gradients-stabilized.hpp:41-268)
over its OpenCL runtime, which cannot be built here. Every kernel they launch
is, though: oracle/Makefile compiles csrmv_adaptive.cl / csrmv_general.cl
(oracle/_ref/librefspmv.so) and dot.cl, reduce.cl, atomic_reduce.cl,
blas1.cl, elementwise_transform.cl, matrix_utils.cl (oracle/_ref/
librefblas1.so) from the reference sources and runs them on the host
(oracle/clc_shim.h: a work-group's work-items as fibers, from barrier to
barrier in work-item order). This module issues those kernels in the order of the
reference's host code, one call per line of it, with the host code's own
launch parameters (the wrappers in oracle/ref_blas1.c state them). Scalars
live in one-element arrays, as the reference keeps them in device buffers;
the host reads them where the reference maps them (norm_b, the residuals
the stop test sees). Work-items run in a fixed order, so the second-stage
atomic additions (atomic_reduce.cl) happen in group order and a run is
reproducible bit for bit (on a GPU their order, and so the last bits, vary).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import ref_csrmv_adaptive, ref_csrmv_general, ref_subwave

HERE = Path(__file__).resolve().parent
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = HERE / "_ref" / "librefblas1.so"
        if not path.exists():
            return None
        _lib = C.CDLL(str(path))
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Kernels:
    """The reference's kernels for one value type, with the launch sequence of
    the host wrappers that call them."""

    def __init__(self, dtype):
        if lib() is None:
            raise RuntimeError("oracle/_ref/librefblas1.so not built")
        self.t = np.dtype(dtype)
        self.s = "d" if self.t == np.float64 else "s"
        self.L = lib()

    def _call(self, name, *args):
        f = getattr(self.L, name)
        f.restype = C.c_int
        if f(*args) != 0:
            raise RuntimeError(f"{name} failed")

    def scalar(self, v=0.0):
        return np.array([v], self.t)

    def vec(self, n, v=0.0):
        return np.full(n, v, self.t)

    # cldense-dot.hpp:96-152: init_scalar, inner_product, atomic_reduce
    def dot(self, r, x, y):
        r[0] = 0
        part = np.zeros(256, self.t)
        self._call(f"ref_inner_product_{self.s}", C.c_uint(len(x)), _p(part), _p(x), _p(y))
        self._call(f"ref_atomic_reduce_{self.s}", _p(r), _p(part))

    # cldense-nrm1.hpp:27-32 -> reduce.hpp:102-165 with RO_FABS
    def norm1(self, r, x):
        r[0] = 0
        part = np.zeros(256, self.t)
        self._call(f"ref_global_reduce_fabs_{self.s}", C.c_uint(len(x)), _p(x), _p(part))
        self._call(f"ref_atomic_reduce_{self.s}", _p(r), _p(part))

    # elementwise-transform.hpp (r = x OP y); also scalar::div / mul on one element
    def transform(self, op, r, x, y):
        self._call(f"ref_transform_{op}_{self.s}", C.c_uint(len(r)), _p(r), _p(x), _p(y))

    # cldense-axpy.hpp: y = z OP alpha * x
    def axpy(self, op, y, alpha, x, z):
        self._call(f"ref_axpy_{op}_{self.s}", C.c_uint(len(y)), _p(y), _p(alpha), _p(x), _p(z))

    # cldense-axpby.hpp: y = alpha * x OP beta * z
    def axpby(self, op, y, alpha, x, beta, z):
        self._call(f"ref_axpby_{op}_{self.s}", C.c_uint(len(y)), _p(y), _p(alpha), _p(x), _p(beta), _p(z))


class Matrix:
    """A CSR matrix as the reference's kernels see it; with a meta the SpMV
    runs csrmv_adaptive (the meta buffer is kept between calls, flag bits
    and all, as the reference's is), without one csrmv_general."""

    def __init__(self, rp, col, val, dtype, meta):
        self.rp = np.ascontiguousarray(rp, np.uint32)
        self.col = np.ascontiguousarray(col, np.uint32)
        self.val = np.ascontiguousarray(val, dtype)
        self.n = len(self.rp) - 1
        self.dtype = np.dtype(dtype)
        self.meta = meta

    def spmv(self, alpha, x, beta, y):
        """y = alpha * A * x + beta * y in place (clsparse-csrmv.hpp:103-132)."""
        if self.meta:
            out = ref_csrmv_adaptive(self.rp, self.col, self.val, x, y, alpha[0], beta[0], self.dtype)
        else:
            out = ref_csrmv_general(self.rp, self.col, self.val, x, y, alpha[0], beta[0], self.dtype)
        y[:] = out

    def inv_diagonal(self, k):
        """extract_diagonal<T, true> (preconditioner_utils.hpp:28-134): the
        subwave from the average row length, rows without a diagonal keep
        their (here zero) entry."""
        d = k.vec(self.n)
        sw = ref_subwave(int(self.rp[-1] - self.rp[0]), self.n)
        k._call(f"ref_extract_diag_inv_{k.s}_sw{sw}", C.c_uint(self.n), _p(d), _p(self.rp), _p(self.col),
                _p(self.val))
        return d


def _finished(res, rel, abs_, init, n_iters, max_iters):
    """solver-control.hpp:47-64."""
    return res <= rel or res <= abs_ * init or n_iters >= max_iters


def cg(rp, col, val, x0, b, dtype, precond, max_iters, rel_tol, abs_tol, meta=False):
    """conjugate-gradients.hpp:65-226. precond: 1 = Jacobi (diagonal.hpp),
    0 = none (void.hpp). Returns (x, nIters, initialResidual,
    currentResidual, residual history)."""
    k = Kernels(dtype)
    A = Matrix(rp, col, val, dtype, meta)
    x = np.array(x0, dtype, copy=True)
    b = np.ascontiguousarray(b, dtype)
    n = A.n
    invd = A.inv_diagonal(k) if precond == 1 else None

    def M(src, dst):  # diagonal.hpp:64-72 (element-wise product) / void.hpp (copy)
        if invd is not None:
            k.transform("MULTIPLY", dst, src, invd)
        else:
            dst[:] = src

    norm_b = k.scalar()
    k.norm1(norm_b, b)                                     # :77
    if norm_b[0] == 0:                                     # :87-95
        return b.copy(), 0, 0.0, 0.0, []
    y, z, r, p = k.vec(n), k.vec(n), k.vec(n), k.vec(n)    # :102-105
    one, zero = k.scalar(1), k.scalar(0)
    A.spmv(one, x, zero, y)                                # :111 y = A x
    k.transform("MINUS", r, b, y)                          # :115 r = b - y
    norm_r = k.scalar()
    k.norm1(norm_r, r)                                     # :120
    residuum = k.scalar()
    k.transform("DIV", residuum, norm_r, norm_b)           # :127
    init = float(residuum[0])
    if _finished(init, rel_tol, abs_tol, init, 0, max_iters):  # :134-138, a fresh control's nIters
        return x, 0, init, init, [init]
    M(r, z)                                                # :140
    p[:] = z                                               # :143
    rz = k.scalar()
    k.dot(rz, r, z)                                        # :147
    alpha, beta, yp, rz_old = k.scalar(), k.scalar(), k.scalar(), k.scalar()
    iteration = 0
    hist = [init]
    cur = init
    while True:
        n_iters = iteration                                # :164
        A.spmv(one, p, zero, y)                            # :167
        k.dot(yp, y, p)                                    # :171
        k.transform("DIV", alpha, rz, yp)                  # :176
        k.axpy("PLUS", x, alpha, p, x)                     # :183 x = x + alpha p
        k.axpy("MINUS", r, alpha, y, r)                    # :187 r = r - alpha y
        M(r, z)                                            # :192
        rz_old[:] = rz                                     # :196
        k.dot(rz, r, z)                                    # :199
        k.transform("DIV", beta, rz, rz_old)               # :205
        k.axpby("PLUS", p, one, z, beta, p)                # :211 p = z + beta p
        k.norm1(norm_r, r)                                 # :215
        k.transform("DIV", residuum, norm_r, norm_b)       # :219
        iteration += 1
        cur = float(residuum[0])
        hist.append(cur)
        if _finished(cur, rel_tol, abs_tol, init, n_iters, max_iters):  # :223, sees nIters of :164
            return x, n_iters, init, cur, hist


def bicgstab(rp, col, val, x0, b, dtype, precond, max_iters, rel_tol, abs_tol, meta=False):
    """biconjugate-gradients-stabilized.hpp:61-266 (right-preconditioned).
    Returns (x, nIters, initialResidual, currentResidual, residual history)."""
    k = Kernels(dtype)
    A = Matrix(rp, col, val, dtype, meta)
    x = np.array(x0, dtype, copy=True)
    b = np.ascontiguousarray(b, dtype)
    n = A.n
    invd = A.inv_diagonal(k) if precond == 1 else None

    def M(src, dst):
        if invd is not None:
            k.transform("MULTIPLY", dst, src, invd)
        else:
            dst[:] = src

    norm_b = k.scalar()
    k.norm1(norm_b, b)                                     # :69
    if norm_b[0] <= np.finfo(dtype).tiny:                  # :75-83
        return b.copy(), 0, 0.0, 0.0, []
    one, zero = k.scalar(1), k.scalar(0)
    y, r = k.vec(n), k.vec(n)
    A.spmv(one, x, zero, y)                                # :104
    k.transform("MINUS", r, b, y)                          # :108
    norm_r = k.scalar()
    k.norm1(norm_r, r)                                     # :112
    residuum = k.scalar()
    k.transform("DIV", residuum, norm_r, norm_b)           # :116
    init = float(residuum[0])
    if _finished(init, rel_tol, abs_tol, init, 0, max_iters):  # :124
        return x, 0, init, init, [init]
    p = r.copy()                                           # :131
    r_star = r.copy()                                      # :134
    rsr_old = k.scalar()
    k.dot(rsr_old, r_star, r)                              # :141
    Mp, AMp, s, Ms, AMs = k.vec(n), k.vec(n), k.vec(n), k.vec(n), k.vec(n)
    alpha, beta, omega = k.scalar(), k.scalar(), k.scalar()
    rsamp, norm_s, amss, amsams, rsr_new = k.scalar(), k.scalar(), k.scalar(), k.scalar(), k.scalar()
    iteration = 0
    hist = [init]
    while True:
        n_iters = iteration
        M(p, Mp)                                           # :166
        A.spmv(one, Mp, zero, AMp)                         # :169
        k.dot(rsamp, r_star, AMp)                          # :173
        k.transform("DIV", alpha, rsr_old, rsamp)          # :176
        k.axpby("MINUS", s, one, r, alpha, AMp)            # :180 s = r - alpha AMp
        k.norm1(norm_s, s)                                 # :183
        k.transform("DIV", residuum, norm_s, norm_b)       # :186
        cur = float(residuum[0])
        if _finished(cur, rel_tol, abs_tol, init, n_iters, max_iters):  # :187-195
            k.axpby("PLUS", x, one, x, alpha, Mp)          # :192 x = x + alpha Mp
            hist.append(cur)
            return x, n_iters, init, cur, hist
        M(s, Ms)                                           # :198
        A.spmv(one, Ms, zero, AMs)                         # :201
        k.dot(amss, AMs, s)                                # :204
        k.dot(amsams, AMs, AMs)                            # :207
        k.transform("DIV", omega, amss, amsams)            # :209
        k.axpy("PLUS", x, alpha, Mp, x)                    # :217 x = x + alpha Mp
        k.axpy("PLUS", x, omega, Ms, x)                    # :220 x = x + omega Ms
        k.axpy("MINUS", r, omega, AMs, s)                  # :224 r = s - omega AMs
        k.norm1(norm_r, r)                                 # :227
        k.transform("DIV", residuum, norm_r, norm_b)       # :230
        iteration += 1
        cur = float(residuum[0])
        hist.append(cur)
        if _finished(cur, rel_tol, abs_tol, init, n_iters, max_iters):  # :233
            return x, n_iters, init, cur, hist
        k.dot(rsr_new, r_star, r)                          # :241
        k.transform("DIV", beta, rsr_new, rsr_old)         # :245
        k.transform("MULTIPLY", beta, beta, alpha)         # :247 beta *= alpha
        k.transform("DIV", beta, beta, omega)              # :249 beta /= omega
        rsr_old[:] = rsr_new                               # :252
        k.axpy("PLUS", p, beta, p, r)                      # :255 p = r + beta p
        k.transform("MULTIPLY", beta, beta, omega)         # :257 beta *= omega
        k.axpy("MINUS", p, beta, AMp, p)                   # :259 p = p - beta AMp
