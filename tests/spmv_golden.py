"""Shared loader of tests/golden/spmv_ref.npz: the outputs of the reference's
own SpMV kernels (csrmv_adaptive / csrmv_general, compiled from its sources
and run on the host; see tests/golden/make_spmv_golden.py) for seeded
matrices whose inputs are regenerated here and checked against the stored
digest."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GOLD = HERE / "golden" / "spmv_ref.npz"
sys.path.insert(0, str(HERE / "golden"))

import make_spmv_golden as mk  # noqa: E402


def load():
    return np.load(GOLD)


def names(d=None):
    d = load() if d is None else d
    return sorted({k.split("__")[0] for k in d.files if "__" in k})


def case(d, name):
    """(rp, col, val, x, y0) of a case, after checking the digest."""
    lens = [int(v) for v in d[f"{name}__lens"]]
    rp, col, val, x, y0 = mk.case_inputs(name, lens)
    assert mk.digest(rp, col, val, x, y0) == str(d[f"{name}__digest"]), f"{name}: inputs no longer match"
    return rp, col, val, x, y0


def reference(d, name, kind, t, ext, k):
    return d[f"{name}__{kind}_{t}_{'ext' if ext else 'plain'}_{k}"]
