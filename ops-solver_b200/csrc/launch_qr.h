// launch_qr.h -- launchers of the real QR family (qr.cu) and the complex QR family (cqr.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ops_solver
{
constexpr int QR_BLOCK = 32;                    // reflectors per panel / block factor
constexpr int QR_T_FLOATS = QR_BLOCK * QR_BLOCK;  // one block factor T
// The factorisations keep two block factors: with look-ahead, consecutive panels' T overlap.
constexpr int QR_GEQRF_T_FLOATS = 2 * QR_T_FLOATS;
// In-place Householder QR of one m x n matrix; tau gets min(m, n) scalars; T holds two
// 32 x 32 block factors (QR_GEQRF_T_FLOATS floats of workspace).
cudaError_t launch_sgeqrf(float *A, int lda, int m, int n, float *tau, float *T, cudaStream_t stream);
// op(Q) C (side 0) or C op(Q) (side 1), trans 0 = Q, else Q^T; Q from k reflectors of A.
cudaError_t launch_sormqr(int side, int trans, int m, int n, int k, const float *A, int lda, const float *tau,
                          float *C, int ldc, float *T, cudaStream_t stream);
// The first n columns of Q from k reflectors, overwriting A; work holds m * k + QR_T_FLOATS floats.
cudaError_t launch_sorgqr(int m, int n, int k, float *A, int lda, const float *tau, float *work, cudaStream_t stream);
// Least squares (m >= n): A overwritten by its QR, B read only, X = n x nrhs solution;
// work holds sgels_work_floats(m, n, nrhs) floats.
size_t sgels_work_floats(int m, int n, int nrhs);
cudaError_t launch_sgels(int m, int n, int nrhs, float *A, int lda, const float *B, int ldb, float *X, int ldx,
                         float *work, cudaStream_t stream);
// T (k x k, ld ldt) of k <= 256 reflectors (backward: units at rows n-k+i), columnwise; G
// holds xlarft_work_bytes(k) of workspace.  Only the referenced triangle of T is written.
size_t xlarft_work_bytes(int k);
cudaError_t launch_xlarft(int backward, int n, int k, const float *V, int ldv, const float *tau, float *T, int ldt,
                          float *G, cudaStream_t stream);

// ---- complex QR family (cqr.cu), complex64 as float2, column-major -------------------------
// In-place Householder QR (clarfg convention); tau gets min(m, n) scalars; T holds
// QR_GEQRF_T_FLOATS complex elements of workspace.
cudaError_t launch_cgeqrf(float2 *A, int lda, int m, int n, float2 *tau, float2 *T, cudaStream_t stream);
// op(Q) C (side 0) or C op(Q) (side 1), herm 0 = Q, else Q^H; Q from k reflectors of A.
cudaError_t launch_cunmqr(int side, int herm, int m, int n, int k, const float2 *A, int lda, const float2 *tau,
                          float2 *C, int ldc, float2 *T, cudaStream_t stream);
// The first n columns of Q from k reflectors, overwriting A; work holds m * k + QR_T_FLOATS elements.
cudaError_t launch_cungqr(int m, int n, int k, float2 *A, int lda, const float2 *tau, float2 *work,
                          cudaStream_t stream);
// Least squares (m >= n): A overwritten by its QR, B read only, X = n x nrhs solution; a zero
// diagonal entry of R sets *info to its one-based position and leaves X untouched; work holds
// cgels_work_elems(m, n, nrhs) complex elements.
size_t cgels_work_elems(int m, int n, int nrhs);
cudaError_t launch_cgels(int m, int n, int nrhs, float2 *A, int lda, const float2 *B, int ldb, float2 *X, int ldx,
                         float2 *work, int *info, cudaStream_t stream);
// A complex64 region screened for NaN and infinity (strict: entries below the diagonal only).
struct CqRegion
{
    const void *p;
    int rows, cols;
    int64_t ld;
    int strict, code;
};
// *flag = min(*flag, code of each region holding a non-finite entry); up to three regions.
cudaError_t launch_cq_finite(const CqRegion *regions, int count, int *flag, cudaStream_t stream);
}  // namespace ops_solver
