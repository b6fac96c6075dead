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
