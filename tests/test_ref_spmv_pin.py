"""The oracle's SpMV restatement (src/tests/test-blas2.cpp:146-163 FP32,
:231-252 FP64) pinned to the reference's OWN kernels: the outputs of
csrmv_adaptive and csrmv_general (src/library/kernels/csrmv_adaptive.cl,
csrmv_general.cl), compiled from the reference sources and run on the host,
stored in tests/golden/spmv_ref.npz. CPU only.

Bars (relative to the row's absolute scale |alpha| sum_j |a_ij x_j| +
|beta y_i|): FP64 1e-12, FP32 1e-5 -- the library's parity bars -- and,
between the compensated (EXTENDED_PRECISION) reference kernels and the
compensated FP64 oracle, 1e-15."""
from __future__ import annotations

import numpy as np
import pytest

import spmv_golden as G

D = G.load()
COEFS = [tuple(c) for c in D["coefs"]]
TOL = {"d": 1e-12, "s": 1e-5}


def oracle_y(orc, t, rp, col, val, x, y0, alpha, beta):
    if t == "d":
        return orc.dcsrmv(rp, col, val, alpha, x, beta, y0)
    return orc.scsrmv(rp, col, np.asarray(val, np.float32), np.float32(alpha), np.asarray(x, np.float32),
                      np.float32(beta), np.asarray(y0, np.float32)).astype(np.float64)


def scale_of(orc, t, rp, col, val, x, y0, alpha, beta):
    dt = np.float64 if t == "d" else np.float32
    return orc.dcsrmv_absscale(rp, col, np.asarray(val, dt).astype(np.float64), float(dt(alpha)),
                               np.asarray(x, dt).astype(np.float64), float(dt(beta)),
                               np.asarray(y0, dt).astype(np.float64))


@pytest.mark.parametrize("t", ["d", "s"])
@pytest.mark.parametrize("name", G.names(D))
def test_oracle_spmv_matches_reference_kernels(orc, name, t):
    rp, col, val, x, y0 = G.case(D, name)
    for k, (alpha, beta) in enumerate(COEFS):
        ref_o = oracle_y(orc, t, rp, col, val, x, y0, alpha, beta)
        sc = scale_of(orc, t, rp, col, val, x, y0, alpha, beta)
        tiny = np.finfo(np.float64 if t == "d" else np.float32).tiny
        for kind in ("adaptive", "general"):
            for ext in (False, True):
                if kind == "general" and t == "s" and ext:
                    continue
                y = G.reference(D, name, kind, t, ext, k).astype(np.float64)
                tol = 1e-15 if (ext and t == "d") else TOL[t]
                err = np.abs(y - ref_o)
                assert np.all(err <= tol * sc + tiny), (kind, ext, k, float((err / (sc + tiny)).max()))


def test_reference_build_reproduces_fixture(orc):
    """Where oracle/_ref was built here, the reference kernels give the
    stored outputs bit for bit (the recipe is deterministic)."""
    if orc.ref_spmv_lib() is None or orc.ref_lib() is None:
        pytest.skip("oracle/_ref not built on this machine")
    name = "threshold_rows"
    rp, col, val, x, y0 = G.case(D, name)
    alpha, beta = COEFS[1]
    y = orc.ref_csrmv_adaptive(rp, col, val, x, y0, alpha, beta, np.float64, False)
    np.testing.assert_array_equal(y, G.reference(D, name, "adaptive", "d", False, 1))
