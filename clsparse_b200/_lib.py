"""ctypes binding of libclsparse_b200.so (the C ABI of include/clSPARSE.h and
include/clSPARSE-b200.h).

The structs mirror include/clSPARSE-1x.h field for field. `load()` opens the
in-tree library and fails loudly if it has not been built: there is no
fallback implementation behind this module.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(os.environ.get("CLSPARSE_B200_LIB", Path(__file__).resolve().parent / "libclsparse_b200.so"))

cl_uint = C.c_uint32
cl_int = C.c_int32
cl_bool = C.c_uint32
cl_ulong = C.c_uint64
cl_mem = C.c_void_p
clsparseIdx_t = cl_uint
clsparseStatus = C.c_int

# clsparseStatus values (include/clSPARSE.h)
clsparseSuccess = 0
clsparseInvalidValue = -30
clsparseInvalidMemObject = -38
clsparseInvalidDevice = -33
clsparseOutOfResources = -5
clsparseNotImplemented = -1024
clsparseNotInitialized = -1023
clsparseStructInvalid = -1022
clsparseInvalidSize = -1021
clsparseInvalidMemObj = -1020
clsparseInsufficientMemory = -1019
clsparseInvalidControlObject = -1018
clsparseInvalidFile = -1017
clsparseInvalidFileFormat = -1016
clsparseInvalidKernelExecution = -1015
clsparseInvalidSolverControlObject = -2048
clsparseInvalidSystemSize = -2047
clsparseIterationsExceeded = -2046

NOPRECOND = 0
DIAGONAL = 1
QUIET, NORMAL, VERBOSE = 0, 1, 2


class clsparseScalar(C.Structure):
    _fields_ = [("value", cl_mem), ("off_value", clsparseIdx_t)]


class cldenseVector(C.Structure):
    _fields_ = [("num_values", clsparseIdx_t), ("values", cl_mem), ("off_values", clsparseIdx_t)]


class clsparseCsrMatrix(C.Structure):
    _fields_ = [
        ("num_rows", clsparseIdx_t), ("num_cols", clsparseIdx_t), ("num_nonzeros", clsparseIdx_t),
        ("values", cl_mem), ("col_indices", cl_mem), ("row_pointer", cl_mem),
        ("off_values", clsparseIdx_t), ("off_col_indices", clsparseIdx_t),
        ("off_row_pointer", clsparseIdx_t), ("meta", C.c_void_p),
    ]


class clsparseCooMatrix(C.Structure):
    _fields_ = [
        ("num_rows", clsparseIdx_t), ("num_cols", clsparseIdx_t), ("num_nonzeros", clsparseIdx_t),
        ("values", cl_mem), ("col_indices", cl_mem), ("row_indices", cl_mem),
        ("off_values", clsparseIdx_t), ("off_col_indices", clsparseIdx_t),
        ("off_row_indices", clsparseIdx_t),
    ]


# cldenseMajor (clSPARSE-xx.h)
rowMajor = 1
columnMajor = 2


class cldenseMatrix(C.Structure):
    _fields_ = [
        ("num_rows", clsparseIdx_t), ("num_cols", clsparseIdx_t), ("lead_dim", clsparseIdx_t),
        ("major", C.c_int), ("values", cl_mem), ("off_values", clsparseIdx_t),
    ]


class clsparseCreateResult(C.Structure):
    _fields_ = [("status", clsparseStatus), ("control", C.c_void_p)]


class clsparseEventResult(C.Structure):
    _fields_ = [("status", clsparseStatus), ("event", C.c_void_p)]


class clsparseCreateSolverResult(C.Structure):
    _fields_ = [("status", clsparseStatus), ("control", C.c_void_p)]


class clsparseMetaSizeResult(C.Structure):
    _fields_ = [("status", clsparseStatus), ("metaSize", clsparseIdx_t)]


class clsparseB200MixedInfo(C.Structure):
    _fields_ = [("outerIterations", cl_int), ("innerIterations", cl_int),
                ("initialTrueResidual", C.c_double), ("trueResidual", C.c_double), ("converged", cl_int)]


P = C.POINTER
_V = C.c_void_p
_S = P(clsparseScalar)
_D = P(cldenseVector)
_M = P(clsparseCsrMatrix)

# name -> (restype, argtypes); every symbol a header declares
SIGNATURES = {
    "clsparseSetup": (clsparseStatus, []),
    "clsparseTeardown": (clsparseStatus, []),
    "clsparseGetVersion": (clsparseStatus, [P(cl_uint)] * 4),
    "clsparseInitScalar": (clsparseStatus, [_S]),
    "clsparseInitVector": (clsparseStatus, [_D]),
    "clsparseInitCooMatrix": (clsparseStatus, [P(clsparseCooMatrix)]),
    "clsparseInitCsrMatrix": (clsparseStatus, [_M]),
    "cldenseInitMatrix": (clsparseStatus, [P(cldenseMatrix)]),
    "clsparseCreateControl": (clsparseCreateResult, [_V]),
    "clsparseEnableAsync": (clsparseStatus, [_V, cl_bool]),
    "clsparseEnableExtendedPrecision": (clsparseStatus, [_V, cl_bool]),
    "clsparseGetEvent": (clsparseEventResult, [_V]),
    "clsparseReleaseControl": (clsparseStatus, [_V]),
    "clsparseCreateSolverControl": (clsparseCreateSolverResult, [C.c_int, cl_int, C.c_double, C.c_double]),
    "clsparseReleaseSolverControl": (clsparseStatus, [_V]),
    "clsparseSetSolverParams": (clsparseStatus, [_V, C.c_int, cl_int, C.c_double, C.c_double]),
    "clsparseSolverPrintMode": (clsparseStatus, [_V, C.c_int]),
    "clsparseScsrcg": (clsparseStatus, [_D, _M, _D, _V, _V]),
    "clsparseDcsrcg": (clsparseStatus, [_D, _M, _D, _V, _V]),
    "clsparseScsrbicgStab": (clsparseStatus, [_D, _M, _D, _V, _V]),
    "clsparseDcsrbicgStab": (clsparseStatus, [_D, _M, _D, _V, _V]),
    "clsparseHeaderfromFile": (clsparseStatus, [P(clsparseIdx_t)] * 3 + [C.c_char_p]),
    "clsparseSCooMatrixfromFile": (clsparseStatus, [P(clsparseCooMatrix), C.c_char_p, _V, cl_bool]),
    "clsparseDCooMatrixfromFile": (clsparseStatus, [P(clsparseCooMatrix), C.c_char_p, _V, cl_bool]),
    "clsparseSCsrMatrixfromFile": (clsparseStatus, [_M, C.c_char_p, _V, cl_bool]),
    "clsparseDCsrMatrixfromFile": (clsparseStatus, [_M, C.c_char_p, _V, cl_bool]),
    "clsparseB200ReadMatrixMarketHost": (clsparseStatus, [C.c_char_p, cl_bool, P(clsparseIdx_t), P(clsparseIdx_t),
                                                          P(clsparseIdx_t), P(clsparseIdx_t), P(clsparseIdx_t),
                                                          P(C.c_double), C.c_size_t]),
    "clsparseCsrMetaSize": (clsparseMetaSizeResult, [_M, _V]),
    "clsparseCsrMetaCreate": (clsparseStatus, [_M, _V]),
    "clsparseCsrMetaDelete": (clsparseStatus, [_M]),
    "clsparseCsrMetaCompute": (clsparseStatus, [_M, _V]),
    "cldenseSscale": (clsparseStatus, [_D, _S, _D, _V]),
    "cldenseDscale": (clsparseStatus, [_D, _S, _D, _V]),
    "cldenseSaxpy": (clsparseStatus, [_D, _S, _D, _D, _V]),
    "cldenseDaxpy": (clsparseStatus, [_D, _S, _D, _D, _V]),
    "cldenseSaxpby": (clsparseStatus, [_D, _S, _D, _S, _D, _V]),
    "cldenseDaxpby": (clsparseStatus, [_D, _S, _D, _S, _D, _V]),
    "cldenseIreduce": (clsparseStatus, [_S, _D, _V]),
    "cldenseSreduce": (clsparseStatus, [_S, _D, _V]),
    "cldenseDreduce": (clsparseStatus, [_S, _D, _V]),
    "cldenseSnrm1": (clsparseStatus, [_S, _D, _V]),
    "cldenseDnrm1": (clsparseStatus, [_S, _D, _V]),
    "cldenseSnrm2": (clsparseStatus, [_S, _D, _V]),
    "cldenseDnrm2": (clsparseStatus, [_S, _D, _V]),
    "cldenseSdot": (clsparseStatus, [_S, _D, _D, _V]),
    "cldenseDdot": (clsparseStatus, [_S, _D, _D, _V]),
    "cldenseSadd": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseDadd": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseSsub": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseDsub": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseSmul": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseDmul": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseSdiv": (clsparseStatus, [_D, _D, _D, _V]),
    "cldenseDdiv": (clsparseStatus, [_D, _D, _D, _V]),
    "clsparseScsrmv": (clsparseStatus, [_S, _M, _D, _S, _D, _V]),
    "clsparseDcsrmv": (clsparseStatus, [_S, _M, _D, _S, _D, _V]),
    "clsparseScoomv": (clsparseStatus, [_S, P(clsparseCooMatrix), _D, _S, _D, _V]),
    "clsparseDcoomv": (clsparseStatus, [_S, P(clsparseCooMatrix), _D, _S, _D, _V]),
    "clsparseScsrmm": (clsparseStatus, [_S, _M, P(cldenseMatrix), _S, P(cldenseMatrix), _V]),
    "clsparseDcsrmm": (clsparseStatus, [_S, _M, P(cldenseMatrix), _S, P(cldenseMatrix), _V]),
    "clsparseScsrSpGemm": (clsparseStatus, [_M, _M, _M, _V]),
    "clsparseScsr2coo": (clsparseStatus, [_M, P(clsparseCooMatrix), _V]),
    "clsparseDcsr2coo": (clsparseStatus, [_M, P(clsparseCooMatrix), _V]),
    "clsparseScoo2csr": (clsparseStatus, [P(clsparseCooMatrix), _M, _V]),
    "clsparseDcoo2csr": (clsparseStatus, [P(clsparseCooMatrix), _M, _V]),
    "clsparseScsr2dense": (clsparseStatus, [_M, P(cldenseMatrix), _V]),
    "clsparseDcsr2dense": (clsparseStatus, [_M, P(cldenseMatrix), _V]),
    "clsparseSdense2csr": (clsparseStatus, [P(cldenseMatrix), _M, _V]),
    "clsparseDdense2csr": (clsparseStatus, [P(cldenseMatrix), _M, _V]),
    # project extensions (include/clSPARSE-b200.h)
    "clsparseB200ComputeRowBlocksHost": (clsparseStatus, [P(clsparseIdx_t), clsparseIdx_t, P(cl_ulong),
                                                          C.c_size_t, P(clsparseIdx_t)]),
    "clsparseB200CsrMetaGetRowBlocks": (clsparseStatus, [_M, P(cl_ulong), C.c_size_t, P(C.c_size_t)]),
    "clsparseB200CsrMetaCreateTuned": (clsparseStatus, [_M, cl_uint, cl_uint, cl_uint, cl_uint, _V]),
    "clsparseB200SolverGetInfo": (clsparseStatus, [_V, P(cl_int), P(C.c_double), P(C.c_double)]),
    "clsparseB200SolverGetDeviceStatus": (clsparseStatus, [_V, P(cl_uint)]),
    "clsparseB200SetSolverLoopMode": (clsparseStatus, [_V, cl_int]),
    "clsparseB200SolverSetNormType": (clsparseStatus, [_V, cl_int]),
    "clsparseDcsrcgMixed": (clsparseStatus, [_D, _M, _D, _V, cl_int, C.c_double, P(clsparseB200MixedInfo), _V]),
    "clsparseDcsrbicgStabMixed": (clsparseStatus, [_D, _M, _D, _V, cl_int, C.c_double, P(clsparseB200MixedInfo), _V]),
}

_lib = None


def load() -> C.CDLL:
    """Opens libclsparse_b200.so once and binds every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m clsparse_b200.build` "
            "(there is no fallback implementation)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class clsparseB200BatchResult(C.Structure):
    _fields_ = [("iterations", C.POINTER(cl_int)), ("residuals", C.POINTER(C.c_double)),
                ("systemsConverged", cl_int), ("maxIterations", cl_int), ("worstResidual", C.c_double)]


SIGNATURES["cldenseDdotNoAlloc"] = (clsparseStatus, [P(clsparseScalar), P(cldenseVector), P(cldenseVector),
                                                     C.c_void_p])

SIGNATURES["clsparseScsrcgBatched"] = (
    clsparseStatus, [P(cldenseVector), P(clsparseCsrMatrix), P(cldenseVector), P(clsparseIdx_t), cl_int,
                     P(cl_int), C.c_void_p, P(clsparseB200BatchResult), C.c_void_p])

SIGNATURES.update({
    "clsparseB200SpaiCreate": (clsparseStatus, [P(C.c_void_p), cl_ulong]),
    "clsparseB200SpaiRelease": (clsparseStatus, [C.c_void_p]),
    "clsparseB200SpaiSetMatrix": (clsparseStatus, [C.c_void_p, P(clsparseCsrMatrix), C.c_void_p]),
    "clsparseB200SpaiParams": (clsparseStatus, [C.c_void_p, P(C.c_float), C.c_size_t, P(C.c_size_t), cl_int]),
    "clsparseB200SpaiLossGrad": (clsparseStatus, [C.c_void_p, P(cldenseVector), cl_int, C.c_double, cl_int,
                                                  P(C.c_double), P(C.c_float), C.c_size_t, C.c_void_p]),
    "clsparseB200SpaiTrainStep": (clsparseStatus, [C.c_void_p, P(cldenseVector), cl_int, C.c_double, C.c_double,
                                                   P(C.c_double), C.c_void_p]),
    "clsparseB200SpaiBuild": (clsparseStatus, [C.c_void_p, C.c_void_p]),
    "clsparseB200SpaiGetFactor": (clsparseStatus, [C.c_void_p, P(clsparseIdx_t), P(clsparseIdx_t), P(C.c_double),
                                                   C.c_size_t, P(C.c_size_t)]),
    "clsparseB200SpaiSave": (clsparseStatus, [C.c_void_p, C.c_char_p]),
    "clsparseB200SpaiLoad": (clsparseStatus, [C.c_void_p, C.c_char_p]),
    "clsparseDcsrcgLearned": (clsparseStatus, [P(cldenseVector), P(clsparseCsrMatrix), P(cldenseVector), C.c_void_p,
                                               C.c_void_p, cl_int, C.c_double, P(clsparseB200MixedInfo), P(cl_int),
                                               C.c_void_p]),
})

SIGNATURES.update({
    "clsparseB200DistCgCreate": (clsparseStatus, [P(C.c_void_p), P(clsparseCsrMatrix), cl_uint, cl_uint, cl_int,
                                                  C.c_void_p]),
    "clsparseB200DistCgRelease": (clsparseStatus, [C.c_void_p]),
    "clsparseB200DistCgBuffers": (clsparseStatus, [C.c_void_p, P(P(C.c_double)), P(P(C.c_double)),
                                                   P(P(C.c_double))]),
    "clsparseB200DistCgStart": (clsparseStatus, [C.c_void_p, P(cldenseVector), P(cldenseVector), C.c_void_p]),
    "clsparseB200DistCgResidual": (clsparseStatus, [C.c_void_p, C.c_void_p]),
    "clsparseB200DistCgProduct": (clsparseStatus, [C.c_void_p, C.c_void_p]),
    "clsparseB200DistCgUpdate": (clsparseStatus, [C.c_void_p, cl_int, C.c_void_p, C.c_void_p]),
    "clsparseB200DistCgState": (clsparseStatus, [C.c_void_p, P(cl_int), C.c_void_p, C.c_void_p]),
    "clsparseB200DistCgGather": (clsparseStatus, [C.c_void_p, C.c_void_p, C.c_void_p, cl_uint, C.c_void_p]),
})

SIGNATURES.update({
    "clsparseB200SolverSetHistory": (clsparseStatus, [C.c_void_p, C.c_void_p, cl_uint]),
    "clsparseB200SolverGetHistoryLength": (clsparseStatus, [C.c_void_p, P(cl_uint)]),
    "clsparseB200SolverSetSnapshots": (clsparseStatus, [C.c_void_p, P(cl_int), cl_int, C.c_void_p]),
})

SIGNATURES.update({
    "clsparseB200SpaiGradient": (clsparseStatus, [C.c_void_p, P(P(C.c_float)), P(C.c_size_t)]),
    "clsparseB200SpaiAdamStep": (clsparseStatus, [C.c_void_p, C.c_double, C.c_double, C.c_void_p]),
})
