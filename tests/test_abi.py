"""The C ABI library: it loads, exports every function the headers declare,
and the host-only entry points behave as the reference's do. CPU only."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
        for m in re.finditer(r"CLSPARSE_EXPORT[^;(]*?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_reference_surface():
    names = declared_functions()
    for must in ("clsparseSetup", "clsparseCreateControl", "clsparseCsrMetaCreate", "clsparseCsrMetaCompute",
                 "clsparseScsrmv", "clsparseDcsrmv", "clsparseScsrcg", "clsparseDcsrcg",
                 "clsparseScsrbicgStab", "clsparseDcsrbicgStab", "cldenseDdot", "cldenseSnrm2"):
        assert must in names
    assert len(names) >= 70


def test_library_exports_every_declared_symbol(libso):
    from clsparse_b200 import _lib as L
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    # and the ctypes binding covers them all
    assert set(declared_functions()) <= set(L.SIGNATURES)


def test_setup_version_init(libso):
    from clsparse_b200 import _lib as L
    assert libso.clsparseSetup() == 0
    v = [L.cl_uint() for _ in range(4)]
    assert libso.clsparseGetVersion(*[C.byref(x) for x in v]) == 0
    assert [x.value for x in v] == [0, 10, 2, 0]
    m = L.clsparseCsrMatrix(num_rows=5, meta=C.c_void_p(1234))
    assert libso.clsparseInitCsrMatrix(C.byref(m)) == 0
    assert m.num_rows == 0 and not m.meta
    s = L.clsparseScalar(C.c_void_p(99), 3)
    assert libso.clsparseInitScalar(C.byref(s)) == 0 and s.off_value == 0


def test_struct_layouts_match_reference_field_order():
    from clsparse_b200 import _lib as L
    # clSPARSE-1x.h:60-90 field order
    assert [f[0] for f in L.clsparseCsrMatrix._fields_] == [
        "num_rows", "num_cols", "num_nonzeros", "values", "col_indices", "row_pointer",
        "off_values", "off_col_indices", "off_row_pointer", "meta"]
    assert C.sizeof(L.clsparseCsrMatrix) == 4 * 3 + 4 + 8 * 3 + 4 * 3 + 4 + 8


def test_status_values(libso):
    from clsparse_b200 import _lib as L
    assert L.clsparseNotImplemented == -1024 and L.clsparseNotInitialized == -1023
    assert L.clsparseInvalidSolverControlObject == -2048 and L.clsparseIterationsExceeded == -2046


def test_uninitialised_and_null_control(libso):
    from clsparse_b200 import _lib as L
    libso.clsparseTeardown()
    a = L.clsparseScalar()
    m = L.clsparseCsrMatrix()
    v = L.cldenseVector()
    assert libso.clsparseDcsrmv(C.byref(a), C.byref(m), C.byref(v), C.byref(a), C.byref(v), None) == \
        L.clsparseNotInitialized
    libso.clsparseSetup()
    assert libso.clsparseDcsrmv(C.byref(a), C.byref(m), C.byref(v), C.byref(a), C.byref(v), None) == \
        L.clsparseInvalidControlObject
    assert libso.clsparseScsrcg(C.byref(v), C.byref(m), C.byref(v), None, None) == \
        L.clsparseInvalidControlObject
    assert libso.cldenseDnrm2(C.byref(a), C.byref(v), None) == L.clsparseInvalidControlObject
    assert libso.clsparseEnableAsync(None, 1) == L.clsparseInvalidControlObject


def test_solver_control_lifecycle(libso):
    from clsparse_b200 import _lib as L
    r = libso.clsparseCreateSolverControl(L.DIAGONAL, 100, 1e-2, 1e-5)
    assert r.status == 0 and r.control
    assert libso.clsparseSetSolverParams(r.control, L.NOPRECOND, 7, 1e-3, 1e-6) == 0
    assert libso.clsparseSolverPrintMode(r.control, L.QUIET) == 0
    it = L.cl_int()
    r0 = C.c_double()
    r1 = C.c_double()
    assert libso.clsparseB200SolverGetInfo(r.control, C.byref(it), C.byref(r0), C.byref(r1)) == 0
    assert it.value == 0
    assert libso.clsparseReleaseSolverControl(r.control) == 0
    assert libso.clsparseReleaseSolverControl(None) == L.clsparseInvalidSolverControlObject
    assert libso.clsparseSetSolverParams(None, 0, 1, 1.0, 1.0) == L.clsparseInvalidSolverControlObject


def test_out_of_path_entries_not_implemented(libso):
    from clsparse_b200 import _lib as L
    libso.clsparseSetup()
    assert libso.clsparseScsrSpGemm(None, None, None, None) == L.clsparseNotImplemented
    assert libso.clsparseHeaderfromFile(None, None, None, b"x.mtx") == L.clsparseInvalidValue


def test_meta_delete_without_meta(libso):
    from clsparse_b200 import _lib as L
    m = L.clsparseCsrMatrix()
    assert libso.clsparseCsrMetaDelete(C.byref(m)) == 0


def test_host_binning_rejects_decreasing_row_pointer(libso):
    import numpy as np
    from clsparse_b200 import _lib as L
    rp = np.array([0, 5, 3], dtype=np.uint32)
    s = L.clsparseIdx_t()
    assert libso.clsparseB200ComputeRowBlocksHost(rp.ctypes.data_as(C.POINTER(L.clsparseIdx_t)), 2, None, 0,
                                                  C.byref(s)) == L.clsparseInvalidValue


def test_create_control_without_device_fails_cleanly(libso):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    r = libso.clsparseCreateControl(None)
    assert r.status != 0 and not r.control
