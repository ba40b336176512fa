"""clsparse{S,D}csrmv (through the C ABI) against the outputs of the
reference's OWN kernels for the same inputs (tests/golden/spmv_ref.npz, made
by compiling src/library/kernels/csrmv_adaptive.cl and csrmv_general.cl from
the reference sources and running them on the host).

With a meta the library's adaptive path is compared with the reference's
csrmv_adaptive, without one its vector path with csrmv_general, each plain
and in extended precision. Bars relative to the row's absolute scale:
FP64 1e-12, FP32 1e-5 (plain), FP64 1e-14 and FP32 1e-6 (extended: both
sides compensated)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import spmv_golden as G
from clsparse_b200 import api

pytestmark = pytest.mark.gpu

D = G.load()
COEFS = [tuple(c) for c in D["coefs"]]
DT = {"d": torch.float64, "s": torch.float32}
NPT = {"d": np.float64, "s": np.float32}
TOL = {("d", False): 1e-12, ("s", False): 1e-5, ("d", True): 1e-14, ("s", True): 1e-6}


# (FP32 extended precision of the vector path is not in the fixture)
MODES = [(t, meta, ext) for t in ("d", "s") for meta in (True, False) for ext in (False, True)
         if not (t == "s" and not meta and ext)]


@pytest.mark.parametrize("t,meta,ext", MODES,
                         ids=[f"{t}-{'adaptive' if m else 'vector'}-{'ext' if e else 'plain'}" for t, m, e in MODES])
@pytest.mark.parametrize("name", G.names(D))
def test_library_spmv_matches_reference_kernels(ctrl, orc, name, t, meta, ext):
    kind = "adaptive" if meta else "general"
    rp, col, val, x, y0 = G.case(D, name)
    dt, npt = DT[t], NPT[t]
    A = api.CsrMatrix.from_numpy(rp, col, val, num_cols=len(x), dtype=dt)
    if meta:
        A.create_meta(ctrl)
    ctrl.enable_extended_precision(ext)
    try:
        for k, (alpha, beta) in enumerate(COEFS):
            xt = torch.tensor(np.asarray(x, npt), device="cuda")
            yt = torch.tensor(np.asarray(y0, npt), device="cuda")
            at = torch.tensor([alpha], dtype=dt, device="cuda")
            bt = torch.tensor([beta], dtype=dt, device="cuda")
            api.csrmv(at, A, xt, bt, yt, ctrl)
            out = yt.cpu().numpy().astype(np.float64)
            ref = G.reference(D, name, kind, t, ext, k).astype(np.float64)
            sc = orc.dcsrmv_absscale(rp, col, np.asarray(val, npt).astype(np.float64), float(npt(alpha)),
                                     np.asarray(x, npt).astype(np.float64), float(npt(beta)),
                                     np.asarray(y0, npt).astype(np.float64))
            tiny = np.finfo(npt).tiny
            err = np.abs(out - ref)
            assert np.all(err <= TOL[(t, ext)] * sc + tiny), (k, float((err / (sc + tiny)).max()))
    finally:
        ctrl.enable_extended_precision(False)
