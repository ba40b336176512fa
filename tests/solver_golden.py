"""Shared loader of tests/golden/solvers_ref.npz: CG and BiCGStab runs of
the reference's host solver code over its OWN kernels (compiled from its
sources and run on the host; see tests/golden/make_solver_golden.py), with
the run parameters regenerated here."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GOLD = HERE / "golden" / "solvers_ref.npz"
sys.path.insert(0, str(HERE / "golden"))

import make_solver_golden as mk  # noqa: E402

TYPES = mk.TYPES
PRECONDS = mk.PRECONDS


def load():
    return np.load(GOLD)


def runs():
    return mk.runs()


def run_id(run):
    return mk.key(*run)


def inputs(run):
    """(rp, col, val, x0, b, rel, abs, max_iters) of a run, FP64 values."""
    name, setting, method, t, pre, path = run
    rp, col, val = mk.matrix(name)
    x0, b, rel_d, rel_s, abs_, max_it = mk.run_inputs(name, setting, len(rp) - 1)
    return rp, col, val, x0, b, (rel_d if t == "d" else rel_s), abs_, max_it


def reference(d, run):
    """(x, nIters, initialResidual, currentResidual, history) of the
    reference's run."""
    k = mk.key(*run)
    it, init, cur = d[k + "__stats"]
    return d[k + "__x"], int(it), float(init), float(cur), d[k + "__hist"]


# Parity bars against the reference's runs, from the spread between two
# faithful implementations (the oracle and the reference kernels agree on
# every initial residual bit for bit; their reductions sum in different
# orders): iteration counts -- CG exactly in FP64, within 1 in FP32;
# BiCGStab within max(2, 5%), its convergence being irregular (the
# reference's own csrmv_general and csrmv_adaptive runs of poisson20 tight
# FP64 take 46 and 44 iterations) -- and x relative to max|x|: 1e-6 in FP64
# (observed up to 1.5e-7 on the unpreconditioned lognormal diffusion
# matrix), 1e-2 in FP32 (the reference test's own relative tolerance;
# observed up to 2.1e-3).
# The banded loop mode's BiCGStab sums its dot products in yet another order
# and crosses the tolerance of that irregular history up to 3 iterations
# from the reference's run (poisson20 tight FP64 Jacobi, adaptive: 47
# against 44; the reference's own general-path run takes 46): its bar is
# max(3, 7%). Its CG keeps the exact bar.
def iter_slack(method, t, n_ref, banded=False):
    if method == "cg":
        return 0 if t == "d" else 1
    if banded:
        return max(3, int(0.07 * n_ref))
    return max(2, int(0.05 * n_ref))


X_TOL = {"d": 1e-6, "s": 1e-2}
