/*
 * cann_ops_solver_b200.h -- entry points this build adds beside the reference C ABI.
 *
 * None of these names exists in the reference; the existing entry points of
 * cann_ops_solver.h keep their reference contracts unchanged.  Each addition states the
 * reference call sequence it stands in for.  All of them are asynchronous on the handle
 * stream (no host synchronisation inside), so they can be captured in a CUDA graph, except
 * where an entry's comment says otherwise (aclsolverSgesvIrBatched above order 512).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "cann_ops_solver_common.h"

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
#ifdef __cplusplus
extern "C"
{
#endif

    /* Switches the synchronous device-data checks of the real LU family on the handle:
     * the non-finite scan (src/utils/real_lu_common.h:90, CheckFinite), the pivot-range
     * read-back (:134, CheckPivots) and the pointer-table validation (:196, ArrayValidation)
     * of aclsolverSgetrf, aclsolverSgetri, aclsolverSgetriBatched and aclsolverSmatinvBatched.
     * enabled = 1 (the default) keeps the reference contract: those entries copy metadata
     * back and synchronise the handle stream.  enabled = 0 skips them, which makes the
     * entries asynchronous and capturable in a CUDA graph; argument checks stay, and the
     * caller becomes responsible for finite inputs, valid pivots and disjoint outputs. */
    aclsolverStatus_t aclsolverSetDeviceChecks(aclsolverHandle_t handle, int enabled);
    aclsolverStatus_t aclsolverGetDeviceChecks(aclsolverHandle_t handle, int *enabled);

    /* Batched P*A = L*U of square n x n matrices, the arithmetic of aclsolverSgetrf applied to
     * every slot (first-maximum |a| pivot with the earliest row on ties, IEEE division of the
     * column, FMA rank-1 updates).  PivotArray holds n pivots per matrix, 1-based (NULL = no
     * pivoting).  infoArray[b] = first zero U(k,k) of matrix b, or -2 for a null slot.
     * The reference exposes no batched getrf: its callers issue one aclsolverSgetrf
     * (include/cann_ops_solver.h:101) per matrix, each with a synchronous finite check.
     * This entry does not scan for non-finite values (they propagate, as in LAPACK).
     * 0 <= n <= 4096.  Argument errors: INVALID_VALUE, infoArray filled with -i.  A null
     * matrix slot sets its info to -2. */
    aclsolverStatus_t aclsolverSgetrfBatched(aclsolverHandle_t handle, int n, float *const Aarray[], int lda,
                                             int *PivotArray, int *infoArray, int batchSize);

    /* Batched solve op(A_b) X_b = B_b from the factors of aclsolverSgetrfBatched, device
     * column-major buffers (the reference aclsolverSgetrs, include/cann_ops_solver.h:1011, is
     * host-buffer, row-major and synchronous).  trans: ACLSOLVER_OP_N or ACLSOLVER_OP_T.
     * PivotArray n per matrix (NULL = no pivoting).  infoArray[b] = 0, or -i argument error,
     * or -6 when matrix b's pivot k lies outside [k+1, n] (that slot is left unsolved).
     * 0 <= n <= 8192, 0 <= nrhs (both trans codes at every order). */
    aclsolverStatus_t aclsolverSgetrsBatched(aclsolverHandle_t handle, aclsolverOperation_t trans, int n, int nrhs,
                                             const float *const Aarray[], int lda, const int *PivotArray,
                                             float *const Barray[], int ldb, int *infoArray, int batchSize);

    /* aclsolverCpotrsBatched without its one-right-hand-side restriction: 0 <= nrhs <= 128
     * columns per matrix, same arguments, info (device scalar) and argument-error rules.  The
     * reference requires nrhs == 1 for non-empty batches (src/cpotrs_batched/arch35/
     * cpotrs_batched.cpp:19-21), so a caller with k right-hand sides issues k calls there. */
    aclsolverStatus_t aclsolverCpotrsBatchedMultiRhs(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                                     int nrhs, const aclsolverFloatComplex *const Aarray[], int lda,
                                                     aclsolverFloatComplex *Barray[], int ldb, int *info,
                                                     int batchSize);

    /* Uneven-order batches: factor A_b = L_b L_b^H (or U^H U) and solve A_b X_b = B_b for
     * matrices of different orders in one persistent launch captured in a CUDA graph.  The
     * reference factors one uniform order per call (aclsolverCpotrfBatched,
     * include/cann_ops_solver.h:224) and solves one right-hand side per call
     * (aclsolverCpotrsBatched, :244), so an uneven batch takes it one pair of calls per
     * distinct order and right-hand side.
     *
     * Create: nArray, ldaArray, ldbArray are HOST arrays of batchSize entries (0 <= n <= 160,
     * lda, ldb >= max(1, n)); 0 <= nrhs <= 128.  The plan sorts the matrices by order into
     * size buckets, and with autotune = 1 times candidate launch shapes (warp-path cutoff,
     * threads per matrix, persistent blocks per SM) on scratch matrices of the same orders,
     * keeping the fastest; choices are cached in the file named by OPS_SOLVER_TUNE_CACHE
     * (default $HOME/.cache/ops_solver_b200_vbatched_tune.txt).
     * Execute: Aarray / Barray are device tables of device matrix pointers; infoArray
     * (device, batchSize entries) receives each matrix's factor info (first non-positive
     * pivot, or -3 for a null slot); a failed matrix keeps its completed columns and its B
     * is left unsolved.  Asynchronous on the handle stream; the graph is instantiated on
     * the first execution with a given set of tables and replayed afterwards.
     * Argument errors return INVALID_VALUE (no device write at plan creation). */
    typedef struct aclsolverVbatchedPlan_st *aclsolverVbatchedPlan_t;
    aclsolverStatus_t aclsolverCposvVbatchedPlanCreate(aclsolverHandle_t handle, aclsolverFillMode_t uplo,
                                                       const int *nArray, const int *ldaArray, const int *ldbArray,
                                                       int nrhs, int batchSize, int autotune,
                                                       aclsolverVbatchedPlan_t *plan);
    aclsolverStatus_t aclsolverCposvVbatched(aclsolverHandle_t handle, aclsolverVbatchedPlan_t plan,
                                             aclsolverFloatComplex *const Aarray[], aclsolverFloatComplex *const Barray[],
                                             int *infoArray);
    aclsolverStatus_t aclsolverVbatchedPlanDestroy(aclsolverVbatchedPlan_t plan);

    /* aclsolverSmatinvBatched for callers that cannot let the library allocate device memory
     * (hosts that hand out all device memory from their own pool and forbid allocations after
     * start-up, and latency-critical loops where an allocation's implicit device
     * synchronisation is not acceptable).  No counterpart in the reference: there the call
     * takes its pivot scratch from the handle, which allocates it.  This variant keeps the
     * LU pivots in an array compiled into the library (2^20 ints, 4 MiB, held by every GPU
     * that loads the library until the process exits) and calls no allocator; n * batchSize
     * above 2^20 is rejected with INVALID_VALUE and info = -7 (split the batch).  Same
     * arguments, arithmetic, info and argument-error rules as aclsolverSmatinvBatched, except
     * that the synchronous device-data checks (finite scan, pointer-table validation) are not
     * run, since they need staging buffers.  The first call on each device resolves the
     * array's device address and should come before any stream capture; so should the first
     * call after the device's context was reset (cudaDeviceReset or a released primary
     * context), which resolves it again.  The current device must be the handle's device
     * (EXECUTION_FAILED otherwise).  All calls share the array: calls whose executions
     * overlap on the GPU race on it and must be serialised. */
    aclsolverStatus_t aclsolverSmatinvBatchedNoAlloc(aclsolverHandle_t handle, int n, const float *const A[], int lda,
                                                     float *const Ainv[], int lda_inv, int *info, int batchSize);

    /* Precision of the LU factorisation behind aclsolverSgesvIrBatched. */
    typedef enum
    {
        ACLSOLVER_FACTOR_FP32 = 0,   /* plain FP32: the factors of aclsolverSgetrfBatched, bit for bit */
        ACLSOLVER_FACTOR_BF16 = 1,   /* trailing update on the BF16 tensor cores, FP32 accumulation */
        ACLSOLVER_FACTOR_BF16X3 = 3, /* split BF16 (a = hi + lo): hi*hi + hi*lo + lo*hi on the tensor
                                        cores, FP32 accumulation, about FP32-level factors */
    } aclsolverFactorPrecision_t;

    /* Solve A_b X_b = B_b by an LU factorisation of the chosen precision plus iterative
     * refinement whose residual r = B - A X and solution update run in FP64.  The reference
     * solves with aclsolverSgetrf (include/cann_ops_solver.h:101) then aclsolverSgetrs
     * (:1011), FP32 throughout and one matrix per call; this entry batches the pair and adds
     * the refinement.  A (lda) and B (ldb) are read only; X (ldx) receives the FP32 solution
     * and may be the same buffers as B.  Column-major, device pointer tables.
     * Per right-hand side the loop stops when the normwise backward error
     * berr = max|r| / (||A||_inf max|x| + max|b|) reaches tol, when it stops halving (the
     * better of the last two iterates is kept) or after maxIter corrections.
     * iterArray (device, may be NULL): corrections kept per matrix (maximum over its
     * right-hand sides).  berrArray (device doubles, may be NULL): final berr per matrix
     * (maximum over its right-hand sides; NaN when the factorisation failed).
     * infoArray (device): the factorisation's info (first zero U(k,k), -2 for a null slot); a
     * matrix with info != 0 is not solved and its X is left unchanged.
     * 0 <= n <= 8192, 0 <= nrhs, 0 <= maxIter, tol >= 0.  Up to n = 512 the batch is refined
     * together, asynchronously on the handle stream, with workspace from the handle (about
     * 4 n^2 + 12 n nrhs bytes per matrix).  Above 512 the systems are refined one after another
     * over the whole GPU, each with at most 16 right-hand sides (NOT_SUPPORTED beyond), and the
     * call reads one status word back per correction (it returns after its work).  Argument
     * errors: INVALID_VALUE, infoArray filled with -i (precision is argument 1). */
    aclsolverStatus_t aclsolverSgesvIrBatched(aclsolverHandle_t handle, aclsolverFactorPrecision_t precision, int n,
                                              int nrhs, const float *const Aarray[], int lda,
                                              const float *const Barray[], int ldb, float *const Xarray[], int ldx,
                                              int maxIter, double tol, int *iterArray, double *berrArray,
                                              int *infoArray, int batchSize);

    /* aclsolverSgetrfBatched with a choice of precision for the trailing updates, for callers
     * that run their own refinement or reuse the factors: ACLSOLVER_FACTOR_FP32 gives exactly
     * the factors, pivots and info of aclsolverSgetrfBatched; the BF16 precisions form the
     * trailing products on the tensor cores (the panels, pivot search and triangular solves
     * stay FP32).  Orders n <= 64 always factor in plain FP32.  0 <= n <= 512; arguments,
     * info and errors as aclsolverSgetrfBatched (precision is argument 1, the others shift
     * by one).  No counterpart in the reference, whose factorisations are FP32 only. */
    aclsolverStatus_t aclsolverSgetrfBatchedMixed(aclsolverHandle_t handle, aclsolverFactorPrecision_t precision,
                                                  int n, float *const Aarray[], int lda, int *PivotArray,
                                                  int *infoArray, int batchSize);

#ifdef __cplusplus
}
#endif
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
