/*
 * clSPARSE-xx.h -- scalar and handle types of the clSPARSE C ABI, defined for a
 * CUDA (sm_100a) implementation without any OpenCL header.
 *
 * Replaces the reference's src/include/clSPARSE-xx.h:25-50, which pulls the
 * cl_* scalar types from <CL/cl.h>. Here every cl_* scalar type is a
 * fixed-width C type of the same size, so structs keep their reference
 * layout:
 *
 *   cl_mem            -> void*         a CUDA device pointer (byte address of the
 *                                      first element of the user's allocation;
 *                                      the off_* fields of the structs are
 *                                      added to it in ELEMENTS, as in the
 *                                      reference)
 *   cl_command_queue  -> cudaStream_t  (struct CUstream_st*); NULL = legacy
 *                                      default stream
 *   cl_event          -> cudaEvent_t   (struct CUevent_st*)
 *
 * clsparseIdx_t stays a 32-bit unsigned index (clSPARSE-xx.h:45-50); the
 * reference refuses 64-bit indices with #error, and so does this header.
 */
#ifndef CLSPARSE_B200_XX_H_
#define CLSPARSE_B200_XX_H_

#include <stdint.h>

#ifndef CLSPARSE_CL_TYPES_DEFINED
#define CLSPARSE_CL_TYPES_DEFINED
typedef int32_t  cl_int;
typedef uint32_t cl_uint;
typedef int64_t  cl_long;
typedef uint64_t cl_ulong;
typedef uint32_t cl_bool;
typedef float    cl_float;
typedef double   cl_double;
typedef void*    cl_mem;
typedef struct CUstream_st* cl_command_queue;
typedef struct CUevent_st*  cl_event;
#endif

#ifndef CL_TRUE
#define CL_TRUE  1u
#define CL_FALSE 0u
#endif

/* Public Khronos status numbers the clsparseStatus enum is built from
 * (reference clSPARSE.h:51-66 takes them from <CL/cl.h>). */
#ifndef CL_SUCCESS
#define CL_SUCCESS                    0
#define CL_COMPILER_NOT_AVAILABLE    -3
#define CL_OUT_OF_RESOURCES          -5
#define CL_OUT_OF_HOST_MEMORY        -6
#define CL_BUILD_PROGRAM_FAILURE    -11
#define CL_INVALID_VALUE            -30
#define CL_INVALID_DEVICE           -33
#define CL_INVALID_CONTEXT          -34
#define CL_INVALID_COMMAND_QUEUE    -36
#define CL_INVALID_MEM_OBJECT       -38
#define CL_INVALID_KERNEL_ARGS      -52
#define CL_INVALID_EVENT_WAIT_LIST  -57
#define CL_INVALID_EVENT            -58
#define CL_INVALID_OPERATION        -59
#endif

/* Memory layout of a dense matrix (reference clSPARSE-xx.h:32-41). */
typedef enum _cldenseMajor
{
    rowMajor = 1,
    columnMajor
} cldenseMajor;

#if defined(CLSPARSE_INDEX_SIZEOF) && (CLSPARSE_INDEX_SIZEOF == 8)
#error clsparse-b200 implements 32-bit indices only, as the reference does
#endif
typedef cl_uint clsparseIdx_t;

#endif /* CLSPARSE_B200_XX_H_ */
