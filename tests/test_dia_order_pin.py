"""The row order of the banded drop-in engine (solver loop mode 3) against the
reference's own csrmv_adaptive kernel (src/library/kernels/csrmv_adaptive.cl,
built here from the reference sources into oracle/_ref).

The engine forms row i of A x as: products rounded, summed one by one in
increasing column order from zero -- except in the CSR-Adaptive STREAM blocks
that reduce a row over g > 1 lanes, whose rows it forms as lane l summing
the products l, l + g, ... one by one and the lanes combined pairwise at
distances g/2, ..., 1 (g from the block's row-block word). This restates that
order in numpy and checks it bit for bit against the reference kernel on the
stencil matrices of the solver pins, FP64 and FP32. No GPU; skipped where
oracle/_ref was not built."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from clsparse_b200 import matgen

WG_BITS = 24


def lanes_per_row(rp):
    """g per row from the row-block words (the kernel's LaneRange table)."""
    words = oracle.row_blocks(rp)[0]
    n = len(rp) - 1
    g = np.ones(n, np.int64)
    rows = (words >> np.uint64(32)).astype(np.int64)
    low = (words & np.uint64((1 << WG_BITS) - 1)).astype(np.int64)
    for w in range(len(words) - 1):
        g[rows[w]:rows[w + 1]] = 1 if low[w] == 0 else min(int(low[w]), 32)
    return g


def banded_order_spmv(rp, col, val, x, t):
    n = len(rp) - 1
    g = lanes_per_row(rp)
    y = np.zeros(n, t)
    for i in range(n):
        gi = min(int(g[i]), 16)
        v = [t(0)] * 16
        for k in range(int(rp[i]), int(rp[i + 1])):
            ln = (k - int(rp[i])) & (gi - 1)
            v[ln] = t(v[ln] + t(val[k] * x[col[k]]))
        off = gi // 2
        while off > 0:
            for ln in range(off):
                v[ln] = t(v[ln] + v[ln + off])
            off //= 2
        y[i] = v[0]
    return y


MATRICES = {
    "poisson20": lambda: matgen.poisson2d(20),
    "poisson_37x91": lambda: matgen.poisson2d(37, 91),
    "diffusion3d_8": lambda: matgen.diffusion3d_lognormal(8, sigma=1.0, seed=2),
    "diffusion3d_20": lambda: matgen.diffusion3d_lognormal(20, sigma=1.0, seed=9),
}


@pytest.mark.parametrize("dtype", [np.float64, np.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("name", sorted(MATRICES))
def test_banded_row_order_equals_reference_adaptive_kernel(name, dtype):
    if oracle.ref_spmv_lib() is None or oracle.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    rp, col, val = MATRICES[name]()
    n = len(rp) - 1
    t = np.dtype(dtype).type
    x = np.random.default_rng(0).uniform(-1, 1, n).astype(t)
    v = np.asarray(val, t)
    ref = oracle.ref_csrmv_adaptive(rp, col, v, x, np.zeros(n, t), 1.0, 0.0, dtype=t)
    ours = banded_order_spmv(rp, col, v, x, t)
    assert np.array_equal(ref, ours), int((ref != ours).sum())
    # the matrices exercise blocks reduced over several lanes
    assert name.startswith("poisson20") or (lanes_per_row(rp) > 1).any()
