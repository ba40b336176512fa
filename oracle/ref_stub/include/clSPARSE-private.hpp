// Stand-in for the reference's src/library/include/clSPARSE-private.hpp, just
// enough for its csr-meta.hpp to compile without OpenCL headers: the index and
// word types and the five CSR-Adaptive constants of clSPARSE-private.hpp:46-50.
// Test infrastructure only (see oracle/Makefile).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstddef>
typedef uint32_t cl_uint;
typedef uint64_t cl_ulong;
typedef cl_uint clsparseIdx_t;
const cl_uint WG_BITS = 24;
const cl_uint ROW_BITS = 32;
const cl_uint BLKSIZE = 1024;
const cl_uint BLOCK_MULTIPLIER = 3;
const cl_uint ROWS_FOR_VECTOR = 1;
