"""cldenseDdotNoAlloc, the dot product for callers that cannot allocate device
memory (no control object, scratch in a fixed device array of the library).

Checked through the C ABI against an exactly rounded host sum (math.fsum of
the products) and against the regular cldenseDdot on the same inputs, twice
in a row (the shared scratch keeps the previous call's contents, so the
second call shows it is cleared correctly), within the FP64 BLAS-1 tolerance
of the other tests: 1e-12 relative to sum |x_i y_i|. The sizes include a
length whose grid fills every scratch slot (the last slot and the arrival
ticket right after it), the maximum length, offsets into the buffers, and a
small call right after a large one. This file is named to be collected last
and passes alone or after the rest of the suite."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CHUNK = 16384
MAX_ELEMENTS = 2048 * CHUNK


def _noalloc_dot(lib, L, s, x, y, off=0):
    stream = torch.cuda.current_stream().cuda_stream
    sv = L.clsparseScalar(C.c_void_p(s.data_ptr()), 0)
    xv = L.cldenseVector(x.numel() - off, C.c_void_p(x.data_ptr()), off)
    yv = L.cldenseVector(y.numel() - off, C.c_void_p(y.data_ptr()), off)
    st = lib.cldenseDdotNoAlloc(C.byref(sv), C.byref(xv), C.byref(yv), C.c_void_p(stream))
    torch.cuda.current_stream().synchronize()
    return st


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)


def _check(libso, L, xh, yh, off=0):
    """Two calls in a row on the same inputs, each against math.fsum."""
    x = torch.tensor(xh, dtype=torch.float64, device="cuda")
    y = torch.tensor(yh, dtype=torch.float64, device="cuda")
    prod = xh[off:] * yh[off:]
    exact = math.fsum(prod.tolist()) if len(prod) else 0.0
    scale = float(np.abs(prod).sum())
    got = None
    for _ in range(2):
        out = torch.full((1,), 123.0, dtype=torch.float64, device="cuda")
        assert _noalloc_dot(libso, L, out, x, y, off) == 0
        got = float(out)
        assert abs(got - exact) <= 1e-12 * scale + 1e-300, (got, exact)
    return got


@pytest.mark.parametrize("n", [0, 1, 1000, 16384, 16385, 3_000_001])
def test_noalloc_dot_matches_fsum_and_cldenseDdot_twice(libso, n):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from clsparse_b200 import _lib as L
    from clsparse_b200 import api
    libso.clsparseSetup()
    xh, yh = _inputs(n, n + 7)
    got = _check(libso, L, xh, yh)
    x = torch.tensor(xh, dtype=torch.float64, device="cuda")
    y = torch.tensor(yh, dtype=torch.float64, device="cuda")
    scale = float(np.abs(xh * yh).sum()) if n else 0.0
    with api.Control() as ctrl:
        ref = torch.zeros(1, dtype=torch.float64, device="cuda")
        api.blas1("cldenseDdot", ("s", ref), x, y, ctrl=ctrl)
        assert abs(got - float(ref)) <= 1e-12 * scale + 1e-300


@pytest.mark.parametrize("n", [2047 * CHUNK + 1, MAX_ELEMENTS], ids=["grid_2048", "max_elements"])
def test_noalloc_dot_full_grid_then_small(libso, n):
    """A length whose grid is 2048 CTAs writes every scratch slot and the
    ticket word after them; the small call that follows must not see any of
    it."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from clsparse_b200 import _lib as L
    libso.clsparseSetup()
    xh, yh = _inputs(n, 11)
    _check(libso, L, xh, yh)
    del xh, yh
    xs, ys = _inputs(777, 12)
    _check(libso, L, xs, ys)


def test_noalloc_dot_honours_offsets(libso):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from clsparse_b200 import _lib as L
    libso.clsparseSetup()
    xh, yh = _inputs(50_003, 13)
    _check(libso, L, xh, yh, off=3)


def test_noalloc_dot_rejects_oversize(libso):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from clsparse_b200 import _lib as L
    libso.clsparseSetup()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    small = torch.zeros(4, dtype=torch.float64, device="cuda")
    sv = L.clsparseScalar(C.c_void_p(out.data_ptr()), 0)
    # only the sizes are inspected before the rejection; nothing is read
    big = L.cldenseVector(MAX_ELEMENTS + 1, C.c_void_p(small.data_ptr()), 0)
    st = libso.cldenseDdotNoAlloc(C.byref(sv), C.byref(big), C.byref(big),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == L.clsparseInvalidSize
