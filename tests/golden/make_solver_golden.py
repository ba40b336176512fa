"""Generates tests/golden/solvers_ref.npz: CG and BiCGStab runs of the
reference's host solver code (src/library/solvers/conjugate-gradients.hpp:
47-228, biconjugate-gradients-stabilized.hpp:41-268) issued by
oracle/ref_solvers.py over the reference's OWN kernels (SpMV, dot, reduce,
atomic_reduce, blas1, elementwise_transform, matrix_utils), which
oracle/Makefile compiles from the reference sources into oracle/_ref and runs
on the host (oracle/clc_shim.h). Per run it stores x, nIters, the initial
and final relative residual and the residual history.

Runs: the reference's solver-test settings (src/tests/test-solvers.cpp:
267-277: x0 = 0, b = 1, relative 1e-2, absolute 1e-5, 100 iterations,
Diagonal or Void preconditioner) and a tighter set (seeded b, relative 1e-8
FP64 / 1e-4 FP32, no absolute tolerance, 1000 iterations), FP64 and FP32,
on SPD matrices (CG and BiCGStab) and a nonsymmetric convection-diffusion
matrix (BiCGStab). The SpMV is csrmv_general (a matrix without a meta, as in
the reference's solver test) and, for a few runs, csrmv_adaptive.

Run where the reference tree exists:  python tests/golden/make_solver_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from clsparse_b200 import matgen  # noqa: E402

# (name, iteration methods)
MATRICES = {
    "poisson20": ("cg", "bicgstab"),
    "diffusion3d_8": ("cg", "bicgstab"),
    "random_spd_600": ("cg", "bicgstab"),
    "convdiff20": ("bicgstab",),
}
TYPES = {"d": np.float64, "s": np.float32}
PRECONDS = {"jacobi": 1, "none": 0}
# settings: (x0 kind, b kind, rel FP64, rel FP32, abs, max iters)
SETTINGS = {
    "reftest": ("zero", "one", 1e-2, 1e-2, 1e-5, 100),
    "tight": ("zero", "seeded", 1e-8, 1e-4, 0.0, 1000),
}
ADAPTIVE = [("poisson20", "tight"), ("diffusion3d_8", "tight")]


def convdiff(m: int, wind: float = 0.4):
    """Upwind convection-diffusion on an m x m grid: the 5-point Laplacian
    plus wind * (u_i - u_{i-1}) in x, nonsymmetric and diagonally dominant."""
    rp, col, val = matgen.poisson2d(m)
    n = m * m
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    col = col.astype(np.int64)
    val = val.copy()
    val[rows == col] += wind
    west = (col == rows - 1) & (rows % m != 0)
    val[west] -= wind
    return rp, col.astype(np.uint32), val


def matrix(name):
    if name == "poisson20":
        return matgen.poisson2d(20)
    if name == "diffusion3d_8":
        return matgen.diffusion3d_lognormal(8, sigma=1.0, seed=2)
    if name == "random_spd_600":
        return matgen.random_spd(600, seed=3)
    if name == "convdiff20":
        return convdiff(20)
    raise KeyError(name)


def run_inputs(name, setting, n):
    """x0, b and tolerances of one run (FP64 values; the run casts)."""
    x0k, bk, rel_d, rel_s, abs_, max_it = SETTINGS[setting]
    x0 = np.zeros(n)
    b = np.ones(n) if bk == "one" else np.random.default_rng(n + 7).uniform(-1, 1, n)
    return x0, b, rel_d, rel_s, abs_, max_it


def runs():
    """Every run key with its parameters."""
    out = []
    for name, methods in MATRICES.items():
        for setting in SETTINGS:
            for method in methods:
                for t in TYPES:
                    for pre in PRECONDS:
                        paths = ["general"] + (["adaptive"] if (name, setting) in ADAPTIVE and pre == "jacobi" else [])
                        for path in paths:
                            out.append((name, setting, method, t, pre, path))
    return out


def key(name, setting, method, t, pre, path):
    return f"{name}__{setting}__{method}_{t}_{pre}_{path}"


def main():
    from oracle import ref_solvers
    if ref_solvers.lib() is None:
        raise SystemExit("oracle/_ref/librefblas1.so missing: run make -C oracle where the reference tree exists")
    arrays = {}
    for name, setting, method, t, pre, path in runs():
        rp, col, val = matrix(name)
        n = len(rp) - 1
        x0, b, rel_d, rel_s, abs_, max_it = run_inputs(name, setting, n)
        rel = rel_d if t == "d" else rel_s
        fn = getattr(ref_solvers, method)
        x, it, init, cur, hist = fn(rp, col, val, x0, b, TYPES[t], PRECONDS[pre], max_it, rel, abs_,
                                    meta=(path == "adaptive"))
        k = key(name, setting, method, t, pre, path)
        arrays[k + "__x"] = np.asarray(x, TYPES[t])
        arrays[k + "__stats"] = np.array([it, init, cur], np.float64)
        arrays[k + "__hist"] = np.asarray(hist, np.float64)
        print(k, it, f"{cur:.3e}", flush=True)
    dst = Path(__file__).resolve().parent / "solvers_ref.npz"
    np.savez_compressed(dst, **arrays)
    print(f"wrote {dst} ({len(runs())} runs)")


if __name__ == "__main__":
    main()
