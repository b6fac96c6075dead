/*
 * cann_ops_solver_common.h -- ABI types of the B200 build of the aclsolver C API.
 *
 * Replaces the reference's include/cann_ops_solver_common.h (status codes :36-50,
 * handle type :52, complex types :58-69, fill mode :72-76).  The numeric values of
 * every enumerator are kept so that a program compiled against the reference header
 * links against libops_solver.so unchanged.
 *
 * The Ascend runtime types the reference takes from <acl/acl.h> are mapped onto CUDA:
 *   aclrtStream  -> cudaStream_t (the handle stream every compute entry enqueues on)
 *   aclError     -> int, with ACL_SUCCESS = 0 and ACL_ERROR_INVALID_PARAM = 100000
 *                   (the CANN runtime values; only aclsolverSgetrs returns aclError).
 */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C"
{
#endif

    /* The CUDA stream type, declared without pulling in cuda_runtime.h so that plain C
     * callers (and ctypes) need no CUDA headers. */
    struct CUstream_st;
    typedef struct CUstream_st *aclrtStream;
    typedef int aclError;

#ifndef ACL_SUCCESS
#define ACL_SUCCESS 0
#endif
#ifndef ACL_ERROR_INVALID_PARAM
#define ACL_ERROR_INVALID_PARAM 100000
#endif

    /* Status codes, values identical to the reference enumeration. */
    typedef enum aclsolverStatus
    {
        ACLSOLVER_STATUS_SUCCESS = 0,
        ACLSOLVER_STATUS_NOT_INITIALIZED = 1,
        ACLSOLVER_STATUS_ALLOC_FAILED = 2,
        ACLSOLVER_STATUS_INVALID_VALUE = 3,
        ACLSOLVER_STATUS_MAPPING_ERROR = 4,
        ACLSOLVER_STATUS_EXECUTION_FAILED = 5,
        ACLSOLVER_STATUS_INTERNAL_ERROR = 6,
        ACLSOLVER_STATUS_NOT_SUPPORTED = 7,
        ACLSOLVER_STATUS_ARCH_MISMATCH = 8,
        ACLSOLVER_STATUS_HANDLE_IS_NULLPTR = 9,
        ACLSOLVER_STATUS_INVALID_ENUM = 10,
        ACLSOLVER_STATUS_UNKNOWN = 11
    } aclsolverStatus_t;

    /* Opaque solver handle (a heap object owned by the library). */
    typedef void *aclsolverHandle_t;

    /* complex64: two consecutive IEEE float32 values (real, imag); layout-equal to
     * std::complex<float> and cuComplex. */
    typedef struct
    {
        float real;
        float imag;
    } aclsolverFloatComplex;

    typedef struct
    {
        float real;
        float imag;
    } aclFloatComplex;

    typedef enum
    {
        ACLSOLVER_FILL_MODE_LOWER = 0,
        ACLSOLVER_FILL_MODE_UPPER = 1
    } aclsolverFillMode_t;

    typedef enum
    {
        ACLSOLVER_OP_N = 0,
        ACLSOLVER_OP_T = 1,
        ACLSOLVER_OP_C = 2
    } aclsolverOperation_t;

    /* Parameter object of the generic (X-prefixed) entries; this build ships none, so it must
     * be NULL (reference cann_ops_solver_common.h:83). */
    typedef void *aclsolverParams_t;

    /* Order of the elementary reflectors of a block reflector (reference :101-105). */
    typedef enum
    {
        ACLSOLVER_DIRECT_FORWARD = 0,
        ACLSOLVER_DIRECT_BACKWARD = 1
    } aclsolverDirectMode_t;

    /* Storage of the reflector vectors (reference :108-111). */
    typedef enum
    {
        ACLSOLVER_STOREV_COLUMNWISE = 0
    } aclsolverStorevMode_t;

    /* Element type of a generic entry (reference :114-118). */
    typedef enum
    {
        ACLSOLVER_R_32F = 0,
        ACLSOLVER_C_32F = 1
    } aclsolverDataType_t;

    /* Side from which an orthogonal factor is applied (reference cann_ops_solver_common.h:93-98). */
    typedef enum
    {
        ACLSOLVER_SIDE_LEFT = 0,
        ACLSOLVER_SIDE_RIGHT = 1
    } aclsolverSideMode_t;

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
static_assert(sizeof(aclsolverFloatComplex) == 2 * sizeof(float), "complex64 is two float32 values");
static_assert(offsetof(aclsolverFloatComplex, imag) == sizeof(float), "imag follows real");
#endif
