"""cldenseDdotNoAlloc, the dot product for callers that cannot allocate device
memory (no control object, scratch in a fixed device array of the library).

Checked through the C ABI against the regular cldenseDdot on the same inputs,
twice in a row (the shared scratch keeps the previous call's contents, so the
second call shows it is cleared correctly), within the FP64 BLAS-1 tolerance
of the other tests: 1e-12 relative to sum |x_i y_i|. This file is named to
be collected last and passes alone or after the rest of the suite."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 2048 * 16384


def _noalloc_dot(lib, L, s, x, y):
    stream = torch.cuda.current_stream().cuda_stream
    sv = L.clsparseScalar(C.c_void_p(s.data_ptr()), 0)
    xv = L.cldenseVector(x.numel(), C.c_void_p(x.data_ptr()), 0)
    yv = L.cldenseVector(y.numel(), C.c_void_p(y.data_ptr()), 0)
    st = lib.cldenseDdotNoAlloc(C.byref(sv), C.byref(xv), C.byref(yv), C.c_void_p(stream))
    torch.cuda.current_stream().synchronize()
    return st


@pytest.mark.parametrize("n", [0, 1, 1000, 16384, 16385, 3_000_001])
def test_noalloc_dot_matches_cldenseDdot_twice(libso, n):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from clsparse_b200 import _lib as L
    from clsparse_b200 import api
    libso.clsparseSetup()
    rng = np.random.default_rng(n + 7)
    x = torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, device="cuda")
    y = torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, device="cuda")
    scale = float((x * y).abs().sum()) if n else 0.0
    with api.Control() as ctrl:
        ref = torch.zeros(1, dtype=torch.float64, device="cuda")
        api.blas1("cldenseDdot", ("s", ref), x, y, ctrl=ctrl)
        expect = float(ref)
    for _ in range(2):
        out = torch.full((1,), 123.0, dtype=torch.float64, device="cuda")
        assert _noalloc_dot(libso, L, out, x, y) == 0
        assert abs(float(out) - expect) <= 1e-12 * scale + 1e-300


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
