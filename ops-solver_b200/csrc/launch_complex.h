// launch_complex.h -- launchers of the complex64 Cholesky kernels (float2 = (re, im)).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ops_solver
{
// Largest order factored and solved by one block per matrix over a packed shared-memory
// triangle; above it launch_cpotrf_large factors one matrix at a time over the whole GPU.
constexpr int CPOTRF_PACKED_MAX = 240;
// In-place complex Cholesky of `count` n x n matrices (table slot q, or `single`), per-slot
// info (first non-positive pivot, -3 for a null slot); n <= CPOTRF_PACKED_MAX.
cudaError_t launch_cpotrf(float2 *single, float2 *const *table, int n, int lda, int upper, int count, int *info,
                          cudaStream_t stream);
// Solve L L^H X = B (or U^H U) for nrhs columns per matrix; skipped when info && info[0] != 0.
cudaError_t launch_cpotrs(const float2 *a_single, const float2 *const *a_table, float2 *b_single,
                          float2 *const *b_table, int n, int lda, int ldb, int nrhs, int upper, int count,
                          const int *info, cudaStream_t stream);
// One n x n matrix (n > CPOTRF_PACKED_MAX) over the whole GPU; info is this matrix's entry;
// scratch holds cpotrf_large_scratch_bytes(n) (the backup for the failure contract).
size_t cpotrf_large_scratch_bytes(int n);
cudaError_t launch_cpotrf_large(float2 *A, int lda, int upper, int n, int *info, void *scratch, cudaStream_t stream);
}  // namespace ops_solver

namespace ops_solver
{
// ---- complex LU family (complex_lu.cu) ----
// Largest order whose inverse keeps each column's state in registers (one block per 8
// columns); above it the state lives in launch_cgetri's scratch and the GPU sweeps one
// matrix at a time.
constexpr int CGETRI_RESIDENT_MAX = 256;
// In-place LU of one m x n matrix; ipiv null selects no pivoting; info must hold 0 on entry
// and receives the first zero pivot (1-based).
cudaError_t launch_cgetrf(float2 *A, int lda, int m, int n, int *ipiv, int *info, cudaStream_t stream);
// Solve with the n x n working matrix M (M = A for trans 0; op(A) for trans 1 and 2),
// X (n x nrhs, ld ldx) overwritten.  Pivots are applied before (trans 0) or after the sweeps.
cudaError_t launch_cgetrs(const float2 *M, int ldm, const int *ipiv, float2 *X, int ldx, int n, int nrhs, int trans,
                          cudaStream_t stream);
// Inverse from LU factors for `count` matrices (pointer tables or strided single buffers),
// per-matrix info (-4 bad pivot, first zero diagonal, or 0); outputs of failed matrices are
// left unwritten.  Orders above CGETRI_RESIDENT_MAX need cgetri_scratch_bytes(n) of scratch.
size_t cgetri_scratch_bytes(int n);
cudaError_t launch_cgetri(const float2 *a_single, const float2 *const *a_table, int lda, int64_t a_stride,
                          const int *ipiv, float2 *c_single, float2 *const *c_table, int ldc, int64_t c_stride, int n,
                          int count, int *info, void *scratch, cudaStream_t stream);
// Gauss-Jordan inverse of `count` matrices of order n <= 32 (pointer tables); info per matrix.
cudaError_t launch_cmatinv(const float2 *const *a_table, float2 *const *c_table, int n, int lda, int ldc, int *info,
                           int count, cudaStream_t stream);
// dst (n x n, ld ldd) = src (n x n, ld n) when *info == 0.
cudaError_t launch_ccopy_ok(const float2 *src, int n, float2 *dst, int ldd, const int *info, cudaStream_t stream);
// Negates the imaginary part of `count` consecutive elements.
cudaError_t launch_cconj(float2 *p, int64_t count, cudaStream_t stream);
// dst (column-major, ld ldd) = transpose of the `rows` x `cols` row-major src (row stride
// lds), conjugated when conj.
cudaError_t launch_ctranspose(const float2 *src, int64_t lds, float2 *dst, int64_t ldd, int rows, int cols, bool conj,
                              cudaStream_t stream);
}  // namespace ops_solver
