"""The public headers compile for C (C99) and C++ callers, and a program using
the reference's own call sequence (sample-spmv.cpp's setup, control, meta,
csrmv, teardown) links against libclsparse_b200.so. CPU only: the program's
main makes no GPU call."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")

SRC = r"""
#include <cuda_runtime.h>
#include "clSPARSE.h"
#include "clSPARSE-b200.h"

int run_spmv(size_t n, size_t nnz) {
    clsparseSetup();
    cudaStream_t stream;
    cudaStreamCreate(&stream);
    clsparseCreateResult cr = clsparseCreateControl(stream);
    clsparseCsrMatrix A;
    clsparseInitCsrMatrix(&A);
    A.num_rows = n;
    A.num_cols = n;
    A.num_nonzeros = nnz;
    cudaMalloc(&A.values, nnz * sizeof(double));
    cudaMalloc(&A.col_indices, nnz * sizeof(clsparseIdx_t));
    cudaMalloc(&A.row_pointer, (n + 1) * sizeof(clsparseIdx_t));
    clsparseCsrMetaCreate(&A, cr.control);
    clsparseScalar alpha, beta;
    cldenseVector x, y;
    clsparseInitScalar(&alpha);
    clsparseInitScalar(&beta);
    clsparseInitVector(&x);
    clsparseInitVector(&y);
    clsparseStatus st = clsparseDcsrmv(&alpha, &A, &x, &beta, &y, cr.control);
    clsparseCsrMetaDelete(&A);
    clsparseReleaseControl(cr.control);
    clsparseTeardown();
    return st == clsparseSuccess ? 0 : 1;
}

int main(void) { return 0; }
"""


@pytest.mark.parametrize("compiler,std,suffix", [("gcc", "-std=c99", ".c"), ("g++", "-std=c++17", ".cpp")])
def test_headers_compile_and_link(tmp_path, compiler, std, suffix):
    if shutil.which(compiler) is None or not (CUDA / "include" / "cuda_runtime.h").exists():
        pytest.skip(f"{compiler} or the CUDA headers are not available")
    lib = ROOT / "clsparse_b200" / "libclsparse_b200.so"
    if not lib.exists():
        pytest.skip("libclsparse_b200.so is not built")
    src = tmp_path / ("prog" + suffix)
    src.write_text(SRC)
    exe = tmp_path / "prog"
    cmd = [compiler, std, "-Wall", "-Werror", f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(src),
           f"-L{lib.parent}", "-lclsparse_b200", f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{lib.parent}", f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
