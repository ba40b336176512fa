"""The library's CG / BiCGStab (clsparse{S,D}csr{cg,bicgStab} through the
C ABI) against runs of the reference's host solver code over the
reference's OWN kernels (tests/golden/solvers_ref.npz): the reference's
solver-test settings (src/tests/test-solvers.cpp:267-277) and a tighter set,
FP64 and FP32, Jacobi and no preconditioner, a matrix without a meta
(the reference test's csrmv_general path) and with one (csrmv_adaptive).
Every run also goes through the persistent engine. The bars are stated in
tests/solver_golden.py; the library's reductions sum in a different order
from the reference's, as two GPUs would."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import solver_golden as G
from clsparse_b200 import api

pytestmark = pytest.mark.gpu

D = G.load()
RUNS = G.runs()
TORCH = {"d": torch.float64, "s": torch.float32}


def lib_solve(ctrl, run, loop_mode):
    name, setting, method, t, pre, path = run
    rp, col, val, x0, b, rel, abs_, max_it = G.inputs(run)
    dt = TORCH[t]
    ctrl.set_solver_loop_mode(loop_mode)
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=dt)
    if path == "adaptive":
        A.create_meta(ctrl)
    x = torch.tensor(x0, dtype=dt, device="cuda")
    bt = torch.tensor(b, dtype=dt, device="cuda")
    sc = api.SolverControl(G.PRECONDS[pre], max_it, rel, abs_)
    info = api.solve(method, x, A, bt, sc, ctrl)
    sc.release()
    return x.cpu().numpy().astype(np.float64), info, (rel, abs_, max_it)


@pytest.mark.parametrize("loop_mode", [0, 2], ids=["graph", "persistent"])
@pytest.mark.parametrize("run", RUNS, ids=[G.run_id(r) for r in RUNS])
def test_library_solver_matches_reference_run(ctrl, run, loop_mode):
    name, setting, method, t, pre, path = run
    xr, it, init, cur, hist = G.reference(D, run)
    x, info, (rel, abs_, max_it) = lib_solve(ctrl, run, loop_mode)
    assert abs(info["nIters"] - it) <= G.iter_slack(method, t, it), (info, it)
    assert info["initialResidual"] == pytest.approx(init, rel=1e-12 if t == "d" else 1e-6)
    c = info["currentResidual"]
    assert c <= rel or c <= abs_ * init or info["nIters"] >= max_it
    dx = np.max(np.abs(x - xr.astype(np.float64))) / np.max(np.abs(xr))
    assert dx <= G.X_TOL[t], dx
