"""cldense* BLAS-1 entry points through the C ABI against numpy (float64
references), the semantics of src/library/blas1/*.cpp. Tolerances: FP64 1e-12
relative, FP32 1e-5 relative (the reference's own test uses absolute 1e-14 /
1e-7 on constant vectors, src/tests/test-blas1.cpp:146-148)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from clsparse_b200 import api

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.float32: 1e-5}
SIZES = [1, 7, 1000, 1_048_579]


def t(a, dtype):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("n", SIZES)
def test_reductions(ctrl, dtype, n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(-1, 1, n)
    p = "D" if dtype == torch.float64 else "S"
    xt, yt = t(x, dtype), t(y, dtype)
    xd = xt.double().cpu().numpy()
    yd = yt.double().cpu().numpy()
    s = torch.zeros(1, dtype=dtype, device="cuda")
    cases = {
        f"cldense{p}reduce": (xd.sum(), np.abs(xd).sum()),
        f"cldense{p}nrm1": (np.abs(xd).sum(), np.abs(xd).sum()),
        f"cldense{p}nrm2": (np.sqrt((xd * xd).sum()), np.sqrt((xd * xd).sum())),
    }
    for name, (ref, scale) in cases.items():
        api.blas1(name, ("s", s), xt, ctrl=ctrl)
        assert abs(float(s) - ref) <= TOL[dtype] * scale + 1e-300, name
    api.blas1(f"cldense{p}dot", ("s", s), xt, yt, ctrl=ctrl)
    assert abs(float(s) - (xd * yd).sum()) <= TOL[dtype] * np.abs(xd * yd).sum() + 1e-300


def test_int_reduce(ctrl):
    x = torch.arange(-500, 100_000, dtype=torch.int32, device="cuda")
    s = torch.zeros(1, dtype=torch.int32, device="cuda")
    api.blas1("cldenseIreduce", ("s", s), x, ctrl=ctrl)
    # 32-bit two's-complement wraparound, as an int accumulation would give
    total = int(np.arange(-500, 100_000, dtype=np.int64).sum())
    assert int(s) == ((total + 2 ** 31) % 2 ** 32) - 2 ** 31


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("n", SIZES)
def test_elementwise_and_axpy(ctrl, dtype, n):
    rng = np.random.default_rng(n + 1)
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(0.5, 1.5, n)
    p = "D" if dtype == torch.float64 else "S"
    xt, yt = t(x, dtype), t(y, dtype)
    xd, yd = xt.double().cpu().numpy(), yt.double().cpu().numpy()
    r = torch.empty(n, dtype=dtype, device="cuda")
    for name, ref in (("add", xd + yd), ("sub", xd - yd), ("mul", xd * yd), ("div", xd / yd)):
        api.blas1(f"cldense{p}{name}", r, xt, yt, ctrl=ctrl)
        np.testing.assert_allclose(r.double().cpu().numpy(), ref, rtol=TOL[dtype] * 10, atol=1e-30)
    a = t([1.75], dtype)
    bb = t([-0.5], dtype)
    api.blas1(f"cldense{p}scale", r, ("s", a), yt, ctrl=ctrl)
    np.testing.assert_allclose(r.double().cpu().numpy(), 1.75 * yd, rtol=TOL[dtype] * 10)
    api.blas1(f"cldense{p}axpy", r, ("s", a), xt, yt, ctrl=ctrl)
    np.testing.assert_allclose(r.double().cpu().numpy(), yd + 1.75 * xd, rtol=TOL[dtype] * 10, atol=TOL[dtype])
    api.blas1(f"cldense{p}axpby", r, ("s", a), xt, ("s", bb), yt, ctrl=ctrl)
    np.testing.assert_allclose(r.double().cpu().numpy(), 1.75 * xd - 0.5 * yd, rtol=TOL[dtype] * 10,
                               atol=TOL[dtype])


def test_alpha_zero_shortcuts(ctrl):
    """alpha == 0: scale fills zeros, axpy copies y (cldense-scale.cpp:41-53,
    cldense-axpy.cpp:50-63) -- even when x holds NaN."""
    n = 1000
    x = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    y = torch.arange(n, dtype=torch.float64, device="cuda")
    r = torch.empty(n, dtype=torch.float64, device="cuda")
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    api.blas1("cldenseDscale", r, ("s", z), x, ctrl=ctrl)
    assert float(r.abs().sum()) == 0.0
    api.blas1("cldenseDaxpy", r, ("s", z), x, y, ctrl=ctrl)
    assert torch.equal(r, y)


def test_empty_vectors(ctrl):
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    s = torch.full((1,), 5.0, dtype=torch.float64, device="cuda")
    api.blas1("cldenseDnrm1", ("s", s), e, ctrl=ctrl)
    assert float(s) == 0.0
    api.blas1("cldenseDadd", e, e, e, ctrl=ctrl)


def test_size_mismatch(ctrl):
    a = torch.zeros(5, dtype=torch.float64, device="cuda")
    b = torch.zeros(6, dtype=torch.float64, device="cuda")
    with pytest.raises(api.ClsparseError):
        api.blas1("cldenseDadd", a, a, b, ctrl=ctrl)


def test_async_mode_and_event(ctrl):
    ctrl.enable_async(True)
    n = 1 << 20
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    s = torch.zeros(1, dtype=torch.float64, device="cuda")
    api.blas1("cldenseDnrm1", ("s", s), x, ctrl=ctrl)
    ev = api.lib().clsparseGetEvent(ctrl.handle)
    assert ev.status == 0 and ev.event
    torch.cuda.synchronize()
    assert float(s) == n
