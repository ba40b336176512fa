"""The oracle's CG / BiCGStab restatements (oracle/oracle.c, following
src/library/solvers/conjugate-gradients.hpp:47-228 and
biconjugate-gradients-stabilized.hpp:41-268) pinned to runs of the
reference's host solver code over the reference's OWN kernels
(tests/golden/solvers_ref.npz). CPU only; the bars are stated in
tests/solver_golden.py."""
from __future__ import annotations

import numpy as np
import pytest

import solver_golden as G

D = G.load()
RUNS = G.runs()


@pytest.mark.parametrize("run", RUNS, ids=[G.run_id(r) for r in RUNS])
def test_oracle_solver_matches_reference_run(orc, run):
    name, setting, method, t, pre, path = run
    rp, col, val, x0, b, rel, abs_, max_it = G.inputs(run)
    dt = G.TYPES[t]
    x, it, init, cur, hist = G.reference(D, run)
    xo, info = orc.solve(method, dt, rp, col, np.asarray(val, dt), np.asarray(x0, dt), np.asarray(b, dt),
                         G.PRECONDS[pre], max_it, rel, abs_)
    assert abs(info.nIters - it) <= G.iter_slack(method, t, it), (info.nIters, it)
    assert info.initialResidual == pytest.approx(init, rel=1e-12 if t == "d" else 1e-6)
    assert hist[0] == init and hist[-1] == cur
    # both stopped on the reference's criterion (solver-control.hpp:47-64)
    for c in (cur, info.currentResidual):
        assert c <= rel or c <= abs_ * init or it >= max_it
    dx = np.max(np.abs(xo - x.astype(np.float64))) / np.max(np.abs(x))
    assert dx <= G.X_TOL[t], dx


def test_fixture_covers_reference_test_settings():
    """The reference's solver test settings (src/tests/test-solvers.cpp:
    267-277) are among the runs, for both methods, types and
    preconditioners."""
    have = {(m, t, p) for (_, s, m, t, p, _) in RUNS if s == "reftest"}
    assert have == {(m, t, p) for m in ("cg", "bicgstab") for t in ("d", "s") for p in ("jacobi", "none")}


def test_reference_build_reproduces_solver_fixture(orc):
    """Where oracle/_ref was built here, the reference's kernels reproduce
    stored runs bit for bit (the host emulation is deterministic)."""
    from oracle import ref_solvers
    if ref_solvers.lib() is None or orc.ref_spmv_lib() is None:
        pytest.skip("oracle/_ref not built on this machine")
    for run in [("poisson20", "reftest", "cg", "d", "jacobi", "general"),
                ("convdiff20", "reftest", "bicgstab", "s", "none", "general"),
                ("diffusion3d_8", "tight", "cg", "d", "jacobi", "adaptive")]:
        name, setting, method, t, pre, path = run
        rp, col, val, x0, b, rel, abs_, max_it = G.inputs(run)
        x, it, init, cur, hist = getattr(ref_solvers, method)(rp, col, val, x0, b, G.TYPES[t], G.PRECONDS[pre],
                                                              max_it, rel, abs_, meta=(path == "adaptive"))
        xr, itr, initr, curr, histr = G.reference(D, run)
        assert it == itr and init == initr and cur == curr
        assert np.array_equal(np.asarray(x, G.TYPES[t]), xr)
        assert np.array_equal(np.asarray(hist), histr)
