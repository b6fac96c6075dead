/*
 * cann_ops_solver.h -- drop-in C ABI of the B200 (sm_100a) factor-and-solve library.
 *
 * Every declaration below keeps the name, argument order, argument meaning, status codes
 * and info conventions of the reference entry point cited beside it (paths are relative
 * to the reference project root).  Matrices are column major, A[i + j*lda]; matrices,
 * pointer tables, pivots and info live in device memory unless stated otherwise.  All
 * compute entries enqueue on the handle stream and return without synchronising, except
 * where the reference contract itself synchronises (the finite/pivot checks of the real
 * LU family and the host-buffer aclsolverSgetrs).
 *
 * Argument-error info values are -i, i the 1-based argument position excluding handle.
 */
#pragma once
#include <stdint.h>

#include "cann_ops_solver_common.h"

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
#ifdef __cplusplus
extern "C"
{
#endif

    /* ---- handle and stream; reference include/cann_ops_solver.h:50,61,70,80 ----------- */

    /* Creates a handle bound to the current CUDA device.  *handle must be NULL on entry. */
    aclsolverStatus_t aclsolverCreate(aclsolverHandle_t *handle);
    /* Waits for the handle's scratch users, frees scratch, frees the handle. */
    aclsolverStatus_t aclsolverDestroy(aclsolverHandle_t handle);
    /* Binds a stream (NULL = legacy default stream) to the handle. */
    aclsolverStatus_t aclsolverSetStream(aclsolverHandle_t handle, aclrtStream stream);
    aclsolverStatus_t aclsolverGetStream(aclsolverHandle_t handle, aclrtStream *stream);

    /* ---- real LU family; reference include/cann_ops_solver.h:100-110 -------------------- */

    /* Lwork in float elements; replaces cann_ops_solver.h:100 (src/sgetrf/sgetrf_host.cpp:24). */
    aclsolverStatus_t aclsolverSgetrf_bufferSize(aclsolverHandle_t handle, int m, int n, float *A, int lda, int *Lwork);
    /* P*A = L*U in place, 1-based devIpiv (NULL = no pivoting), devInfo = first zero U(k,k);
     * replaces cann_ops_solver.h:101 (src/sgetrf/sgetrf_host.cpp:96).  Non-finite input gives
     * INVALID_VALUE with devInfo=-3 after a synchronous check, as in the reference. */
    aclsolverStatus_t aclsolverSgetrf(aclsolverHandle_t handle, int m, int n, float *A, int lda, float *Workspace,
                                      int *devIpiv, int *devInfo);
    /* replaces cann_ops_solver.h:103 (src/sgetri/sgetri_host.cpp:59). */
    aclsolverStatus_t aclsolverSgetri_bufferSize(aclsolverHandle_t handle, int n, float *A, int lda, int *Lwork);
    /* In-place inverse from packed LU + pivots; replaces cann_ops_solver.h:104 (src/sgetri/sgetri_host.cpp:86). */
    aclsolverStatus_t aclsolverSgetri(aclsolverHandle_t handle, int n, float *A, int lda, int *devIpiv,
                                      float *Workspace, int Lwork, int *devInfo);
    /* Out-of-place inverse of a batch of LU factors, PivotArray n*batchSize (NULL = none);
     * replaces cann_ops_solver.h:106 (src/sgetri_batched/sgetri_batched_host.cpp:86). */
    aclsolverStatus_t aclsolverSgetriBatched(aclsolverHandle_t handle, int n, const float *const Aarray[], int lda,
                                             const int *PivotArray, float *const Carray[], int ldc, int *infoArray,
                                             int batchSize);
    /* Inverse of original matrices, 0 <= n <= 32; replaces cann_ops_solver.h:109
     * (src/smatinv_batched/smatinv_batched_host.cpp:11). */
    aclsolverStatus_t aclsolverSmatinvBatched(aclsolverHandle_t handle, int n, const float *const A[], int lda,
                                              float *const Ainv[], int lda_inv, int *info, int batchSize);

    /* ---- complex Cholesky family; reference include/cann_ops_solver.h:135-247 ----------- */

    /* replaces cann_ops_solver.h:135 (src/cpotrf/arch35). Lwork in complex elements. */
    aclsolverStatus_t aclsolverCpotrf_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                                 aclsolverFloatComplex *A, int lda, int *Lwork);
    /* A = L*L^H (LOWER) or U^H*U (UPPER) in place; replaces cann_ops_solver.h:152. */
    aclsolverStatus_t aclsolverCpotrf(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                      aclsolverFloatComplex *A, int lda, aclsolverFloatComplex *Workspace, int Lwork,
                                      int *devInfo);
    /* Solve from a complex Cholesky factor, 0 <= nrhs <= 128; replaces cann_ops_solver.h:171. */
    aclsolverStatus_t aclsolverCpotrs(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                      const aclsolverFloatComplex *A, int lda, aclsolverFloatComplex *B, int ldb,
                                      int *devInfo);
    /* replaces cann_ops_solver.h:185 (src/cpotri/arch35/cpotri.cpp). Lwork = n*n complex. */
    aclsolverStatus_t aclsolverCpotri_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                                 aclsolverFloatComplex *A, int lda, int *Lwork);
    /* The selected triangle of A^-1 from a complex Cholesky factor, in place; devInfo = first
     * invalid factor diagonal (real part <= 0, imaginary part != 0 or non-finite), 1-based,
     * with A unchanged; replaces cann_ops_solver.h:203 (src/cpotri/arch35/cpotri.cpp). */
    aclsolverStatus_t aclsolverCpotri(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                      aclsolverFloatComplex *A, int lda, aclsolverFloatComplex *Workspace, int Lwork,
                                      int *devInfo);
    /* Batched complex Cholesky, uniform n; argument errors use infoArray[0];
     * replaces cann_ops_solver.h:224 (src/cpotrf_batched/arch35/cpotrf_batched.cpp:14). */
    aclsolverStatus_t aclsolverCpotrfBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                             aclsolverFloatComplex *Aarray[], int lda, int *infoArray, int batchSize);
    /* Batched complex solve, nrhs must be 1 for non-empty problems; info is a device scalar;
     * replaces cann_ops_solver.h:244 (src/cpotrs_batched/arch35/cpotrs_batched.cpp:14). */
    aclsolverStatus_t aclsolverCpotrsBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                             const aclsolverFloatComplex *const Aarray[], int lda,
                                             aclsolverFloatComplex *Barray[], int ldb, int *info, int batchSize);


    /* ---- real Cholesky family; reference include/cann_ops_solver.h:433-547 -------------- */

    /* replaces cann_ops_solver.h:433 (src/cholesky/arch35/cholesky_host.cpp:236). */
    aclsolverStatus_t aclsolverSpotrf_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A,
                                                 int lda, int *Lwork);
    /* replaces cann_ops_solver.h:451 (src/cholesky/arch35/cholesky_host.cpp:246). */
    aclsolverStatus_t aclsolverSpotrf(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A, int lda,
                                      float *Workspace, int Lwork, int *devInfo);
    /* 0 <= nrhs <= 128; replaces cann_ops_solver.h:470 (src/cholesky/arch35/cholesky_host.cpp:331). */
    aclsolverStatus_t aclsolverSpotrs(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                      const float *A, int lda, float *B, int ldb, int *devInfo);
    /* replaces cann_ops_solver.h:484 (src/cholesky/arch35/cholesky_host.cpp:241). */
    aclsolverStatus_t aclsolverSpotri_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A,
                                                 int lda, int *Lwork);
    /* The selected triangle of A^-1 from a real Cholesky factor, in place (Lwork = n*n);
     * devInfo = first non-positive or non-finite factor diagonal, 1-based, with A unchanged;
     * replaces cann_ops_solver.h:504 (src/cholesky/arch35/cholesky_host.cpp:277). */
    aclsolverStatus_t aclsolverSpotri(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A, int lda,
                                      float *Workspace, int Lwork, int *devInfo);
    /* Batched in-place Cholesky; a null slot sets only its info to -3; host argument errors
     * fill every info entry; replaces cann_ops_solver.h:524 (cholesky_host.cpp:283). */
    aclsolverStatus_t aclsolverSpotrfBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *Aarray[],
                                             int lda, int *infoArray, int batchSize);
    /* Batched solve, nrhs must be 1 for non-empty problems; info is a device scalar set to -4
     * (null A slot) or -6 (null B slot); replaces cann_ops_solver.h:545 (cholesky_host.cpp:363). */
    aclsolverStatus_t aclsolverSpotrsBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                             float *Aarray[], int lda, float *Barray[], int ldb, int *info,
                                             int batchSize);

    /* ---- host-buffer LU solve; reference include/cann_ops_solver.h:1011 ----------------- */

    /* A (packed LU), ipiv, B and info are HOST buffers in ROW-major order: A(r,c) = A[r*lda+c],
     * B(r,c) = B[r*ldb+c].  trans 0 solves A X = B, 1 solves A^T X = B.  Synchronous.  An ipiv
     * entry outside [1,n] sets *info = -4.  Returns ACL_SUCCESS or ACL_ERROR_INVALID_PARAM;
     * replaces cann_ops_solver.h:1011 (src/sgetrs/sgetrs_host.cpp:131). */
    aclError aclsolverSgetrs(aclsolverHandle_t handle, const uint64_t trans, const int64_t n, const int64_t nrhs,
                             float *A, const int64_t lda, int32_t *ipiv, float *B, const int64_t ldb, int32_t *info);

    /* ---- complex LU family; reference include/cann_ops_solver.h:882-921 and :1042 ---------- */

    /* Lwork (complex elements) for Cgetrf: 0, the panels factor in shared memory.
     * m <= 4096, n <= 8192, lda >= max(1, m); an invalid shape or a null Lwork returns
     * INVALID_VALUE and writes nothing; replaces cann_ops_solver.h:882 (cgetrf_host.cpp:34). */
    aclsolverStatus_t aclsolverCgetrf_bufferSize(aclsolverHandle_t handle, int m, int n, aclFloatComplex *A, int lda,
                                                 int *Lwork);
    /* In-place complex LU with partial pivoting by the L1 magnitude (earliest row on ties);
     * devIpiv null selects no pivoting; Workspace may be null.  devInfo = 0, the first exactly
     * zero pivot (1-based), or -i for invalid argument i (1 m, 2 n, 3 A, 4 lda, 5 Workspace,
     * 6 devIpiv); replaces cann_ops_solver.h:890 (cgetrf_host.cpp:54). */
    aclsolverStatus_t aclsolverCgetrf(aclsolverHandle_t handle, int m, int n, aclFloatComplex *A, int lda,
                                      aclFloatComplex *Workspace, int *devIpiv, int *devInfo);
    /* Lwork = n * n for Cgetri (n <= 4096); A may be null; replaces cann_ops_solver.h:896
     * (cgetri_host.cpp:78). */
    aclsolverStatus_t aclsolverCgetri_bufferSize(aclsolverHandle_t handle, int n, aclFloatComplex *A, int lda,
                                                 int *Lwork);
    /* In-place inverse from Cgetrf's LU and pivots (null = no pivoting).  devInfo = -4 for a
     * pivot outside [row+1, n] (the call then returns INVALID_VALUE), else the first zero
     * diagonal with A unchanged, else 0.  Workspace (n*n) must not overlap A, devIpiv or
     * devInfo; replaces cann_ops_solver.h:903 (cgetri_host.cpp:95). */
    aclsolverStatus_t aclsolverCgetri(aclsolverHandle_t handle, int n, aclFloatComplex *A, int lda, int *devIpiv,
                                      aclFloatComplex *Workspace, int Lwork, int *devInfo);
    /* Out-of-place inverses from LU factors: Aarray / Carray device tables, PivotArray n per
     * matrix or null; per-matrix infoArray as for Cgetri, failed outputs left unwritten;
     * batchSize <= 1,000,000; replaces cann_ops_solver.h:911 (cgetri_batched_host.cpp:33). */
    aclsolverStatus_t aclsolverCgetriBatched(aclsolverHandle_t handle, int n, const aclFloatComplex *const Aarray[],
                                             int lda, const int *PivotArray, aclFloatComplex *const Carray[], int ldc,
                                             int *infoArray, int batchSize);
    /* Direct out-of-place inverses (Gauss-Jordan, partial pivoting) of n <= 32 matrices;
     * info per matrix = the first zero pivot (output unwritten) or 0; batchSize <=
     * 10,000,000; replaces cann_ops_solver.h:919 (cmatinv_batched_host.cpp:33). */
    aclsolverStatus_t aclsolverCmatinvBatched(aclsolverHandle_t handle, int n, const aclFloatComplex *const A[],
                                              int lda, aclFloatComplex *const Ainv[], int lda_inv, int *info,
                                              int batchSize);
    /* Host-buffer complex LU solve, ROW-major like aclsolverSgetrs: trans 0 A X = B, 1 A^T X = B,
     * 2 A^H X = B; n, nrhs in [1, 8192]; an ipiv entry outside [1, n] sets *info = -4.
     * Synchronous; returns ACL_SUCCESS or ACL_ERROR_INVALID_PARAM; replaces
     * cann_ops_solver.h:1042 (src/cgetrs/cgetrs_host.cpp:172). */
    aclError aclsolverCgetrs(aclsolverHandle_t handle, const uint64_t trans, const int64_t n, const int64_t nrhs,
                             aclFloatComplex *A, const int64_t lda, int32_t *ipiv, aclFloatComplex *B,
                             const int64_t ldb, int32_t *info);

    /* ---- real QR family; reference include/cann_ops_solver.h:566-861 --------------------- */

    /* Lwork (floats) for Sgeqrf: 0 for an empty problem, else two 32 x 32 block factors;
     * m <= 8192 (NOT_SUPPORTED above); replaces cann_ops_solver.h:566 (sgeqrf_host.cpp:173). */
    aclsolverStatus_t aclsolverSgeqrf_bufferSize(aclsolverHandle_t handle, int m, int n, float *A, int lda, int *Lwork);
    /* Householder QR in place (LAPACK sign convention): R on and above the diagonal, the
     * reflectors below it, TAU[min(m, n)]; devInfo 0 or -i (1 m, 2 n, 3 A, 4 lda, 5 TAU,
     * 6 Workspace, 7 Lwork); replaces cann_ops_solver.h:598 (sgeqrf_host.cpp:204). */
    aclsolverStatus_t aclsolverSgeqrf(aclsolverHandle_t handle, int m, int n, float *A, int lda, float *TAU,
                                      float *Workspace, int Lwork, int *devInfo);
    /* lwork (floats) for Sorgqr: m * k + 1024; m <= 4096; replaces cann_ops_solver.h:619
     * (sorgqr_host.cpp:142). */
    aclsolverStatus_t aclsolverSorgqr_bufferSize(aclsolverHandle_t handle, int m, int n, int k, const float *A,
                                                 int lda, const float *tau, int *lwork);
    /* The first n columns of Q = H(1) ... H(k), overwriting A; replaces cann_ops_solver.h:645
     * (sorgqr_host.cpp:181). */
    aclsolverStatus_t aclsolverSorgqr(aclsolverHandle_t handle, int m, int n, int k, float *A, int lda,
                                      const float *tau, float *work, int lwork, int *devInfo);
    /* lwork (floats) for Sormqr: one 32 x 32 block factor; nq <= 4096; replaces
     * cann_ops_solver.h:675 (sormqr_host.cpp:149). */
    aclsolverStatus_t aclsolverSormqr_bufferSize(aclsolverHandle_t handle, aclsolverSideMode_t side,
                                                 aclsolverOperation_t trans, int m, int n, int k, const float *A,
                                                 int lda, const float *tau, const float *C, int ldc, int *lwork);
    /* op(Q) C (LEFT) or C op(Q) (RIGHT), OP_T / OP_C apply Q^T; replaces cann_ops_solver.h:708
     * (sormqr_host.cpp:254). */
    aclsolverStatus_t aclsolverSormqr(aclsolverHandle_t handle, aclsolverSideMode_t side, aclsolverOperation_t trans,
                                      int m, int n, int k, const float *A, int lda, const float *tau, float *C,
                                      int ldc, float *work, int lwork, int *devInfo);
    /* Workspace bytes for Xlarft: k * k floats on the device, 0 on the host; params must be
     * NULL, storev COLUMNWISE, all types ACLSOLVER_R_32F (else NOT_SUPPORTED), n <= 4096 and
     * k <= 256 (else NOT_SUPPORTED); replaces cann_ops_solver.h:742 (xlarft_host.cpp:117). */
    aclsolverStatus_t aclsolverXlarft_bufferSize(aclsolverHandle_t handle, aclsolverParams_t params,
                                                 aclsolverDirectMode_t direct, aclsolverStorevMode_t storev, int64_t n,
                                                 int64_t k, aclsolverDataType_t dataTypeV, const void *V, int64_t ldv,
                                                 aclsolverDataType_t dataTypeTau, const void *tau,
                                                 aclsolverDataType_t dataTypeT, void *T, int64_t ldt,
                                                 aclsolverDataType_t computeType, size_t *workspaceInBytesOnDevice,
                                                 size_t *workspaceInBytesOnHost);
    /* The triangular factor T of the block reflector (slarft, columnwise): FORWARD T upper for
     * H(1)...H(k), BACKWARD T lower for H(k)...H(1); only that triangle is written; no devInfo;
     * replaces cann_ops_solver.h:784 (xlarft_host.cpp:190). */
    aclsolverStatus_t aclsolverXlarft(aclsolverHandle_t handle, aclsolverParams_t params, aclsolverDirectMode_t direct,
                                      aclsolverStorevMode_t storev, int64_t n, int64_t k, aclsolverDataType_t dataTypeV,
                                      const void *V, int64_t ldv, aclsolverDataType_t dataTypeTau, const void *tau,
                                      aclsolverDataType_t dataTypeT, void *T, int64_t ldt,
                                      aclsolverDataType_t computeType, void *bufferOnDevice,
                                      size_t workspaceInBytesOnDevice, void *bufferOnHost,
                                      size_t workspaceInBytesOnHost);
    /* Bytes for SSgels: tau, Q^T B and two block factors; m >= n, m, n <= 4096, nrhs <= 128;
     * replaces cann_ops_solver.h:815 (sgels_host.cpp:149). */
    aclsolverStatus_t aclsolverSSgels_bufferSize(aclsolverHandle_t handle, int m, int n, int nrhs, float *dA, int ldda,
                                                 float *dB, int lddb, float *dX, int lddx, void *dwork,
                                                 size_t *lwork_bytes);
    /* Least squares by QR: X = R^-1 (Q^T B)(1:n, :); dA overwritten, dB read only, dX must
     * overlap neither; *niter = 0; a zero diagonal of R propagates Inf/NaN (not reported);
     * replaces cann_ops_solver.h:859 (sgels_host.cpp:285). */
    aclsolverStatus_t aclsolverSSgels(aclsolverHandle_t handle, int m, int n, int nrhs, float *dA, int ldda, float *dB,
                                      int lddb, float *dX, int lddx, void *dWorkspace, size_t lwork_bytes, int *niter,
                                      int *dinfo);

    /* ---- complex QR family; reference include/cann_ops_solver.h:259-424 ------------------- *
     * complex64, column-major; reflectors in the clarfg convention (H = I - tau v v^H, beta
     * real); padding rows are preserved.  Each execute call screens its inputs for NaN / Inf
     * first (one stream synchronisation and a four-byte read-back, as the reference does):
     * INVALID_VALUE with info -i for the first such argument. */

    /* Lwork (complex elements) for Cgeqrf: 0 for an empty problem, else two 32 x 32 block
     * factors; replaces cann_ops_solver.h:259 (cgeqrf_host.cpp:45). */
    aclsolverStatus_t aclsolverCgeqrf_bufferSize(aclsolverHandle_t handle, int m, int n, aclsolverFloatComplex *A,
                                                 int lda, int *Lwork);
    /* A = Q R in place, TAU[min(m, n)]; devInfo 0 or -i (1 m, 2 n, 3 A, 4 lda, 5 TAU,
     * 6 Workspace, 7 Lwork); replaces cann_ops_solver.h:277 (cgeqrf_host.cpp:51). */
    aclsolverStatus_t aclsolverCgeqrf(aclsolverHandle_t handle, int m, int n, aclsolverFloatComplex *A, int lda,
                                      aclsolverFloatComplex *TAU, aclsolverFloatComplex *Workspace, int Lwork,
                                      int *devInfo);
    /* lwork (complex elements) for Cungqr: m * k + 1024 (0 when empty); replaces
     * cann_ops_solver.h:292 (cungqr_host.cpp:47). */
    aclsolverStatus_t aclsolverCungqr_bufferSize(aclsolverHandle_t handle, int m, int n, int k,
                                                 const aclsolverFloatComplex *A, int lda,
                                                 const aclsolverFloatComplex *tau, int *lwork);
    /* The first n columns of Q = H(1) ... H(k) (k = 0: identity columns), overwriting A;
     * replaces cann_ops_solver.h:310 (cungqr_host.cpp:54). */
    aclsolverStatus_t aclsolverCungqr(aclsolverHandle_t handle, int m, int n, int k, aclsolverFloatComplex *A, int lda,
                                      const aclsolverFloatComplex *tau, aclsolverFloatComplex *work, int lwork,
                                      int *devInfo);
    /* lwork (complex elements) for Cunmqr: one 32 x 32 block factor (0 when empty); trans N or
     * C; replaces cann_ops_solver.h:329 (cunmqr_host.cpp:55). */
    aclsolverStatus_t aclsolverCunmqr_bufferSize(aclsolverHandle_t handle, aclsolverSideMode_t side,
                                                 aclsolverOperation_t trans, int m, int n, int k,
                                                 const aclsolverFloatComplex *A, int lda,
                                                 const aclsolverFloatComplex *tau, const aclsolverFloatComplex *C,
                                                 int ldc, int *lwork);
    /* op(Q) C (LEFT) or C op(Q) (RIGHT), op(Q) = Q (OP_N) or Q^H (OP_C; OP_T is rejected as
     * argument 2); replaces cann_ops_solver.h:353 (cunmqr_host.cpp:65). */
    aclsolverStatus_t aclsolverCunmqr(aclsolverHandle_t handle, aclsolverSideMode_t side, aclsolverOperation_t trans,
                                      int m, int n, int k, const aclsolverFloatComplex *A, int lda,
                                      const aclsolverFloatComplex *tau, aclsolverFloatComplex *C, int ldc,
                                      aclsolverFloatComplex *work, int lwork, int *devInfo);
    /* Bytes for CCgels: tau, Q^H B and two block factors; m >= n, m, n <= 4096, nrhs <= 128;
     * replaces cann_ops_solver.h:376 (ccgels_host.cpp:68). */
    aclsolverStatus_t aclsolverCCgels_bufferSize(aclsolverHandle_t handle, int m, int n, int nrhs,
                                                 aclsolverFloatComplex *dA, int ldda, aclsolverFloatComplex *dB,
                                                 int lddb, aclsolverFloatComplex *dX, int lddx, void *dwork,
                                                 size_t *lwork_bytes);
    /* Least squares by QR: X = R^-1 (Q^H B)(1:n, :); dA overwritten, dB read only, dX must
     * overlap neither; *niter = 0; a zero diagonal entry of R sets dinfo to its one-based
     * position and leaves dX untouched; replaces cann_ops_solver.h:408 (ccgels_host.cpp:77). */
    aclsolverStatus_t aclsolverCCgels(aclsolverHandle_t handle, int m, int n, int nrhs, aclsolverFloatComplex *dA,
                                      int ldda, aclsolverFloatComplex *dB, int lddb, aclsolverFloatComplex *dX,
                                      int lddx, void *dWorkspace, size_t lwork_bytes, int *niter, int *dinfo);

#ifdef __cplusplus
}
#endif
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#include "cann_ops_solver_b200.h"
