// refine.h -- FP64 iterative-refinement kernels (refine.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ops_solver
{

// Refinement state.  A "job" is one (matrix, right-hand side) pair, job = matrix * nrhs +
// rhs; vectors are n long and packed by job.  All device memory.
struct IrState
{
    double *x64;   // per job: the solution in FP64
    float *r32;    // per job: FP32 right-hand side of the next solve (b, then residuals)
    double *berr;  // per job: backward error of the current x64
    int *state;    // per job: IR_RUNNING, IR_CONVERGED, IR_STALLED or IR_FAILED
    int *iters;    // per job: corrections applied (a correction taken back is not counted)
};

enum
{
    IR_RUNNING = 0,
    IR_CONVERGED = 1,  // berr <= tol
    IR_STALLED = 2,    // berr stopped halving; the better of the last two iterates is kept
    IR_FAILED = 3,     // the factorisation reported info != 0: nothing is solved
};

// r32 <- b; state from the factor info; berr <- huge; iters <- 0.
cudaError_t launch_ir_init(const IrState &s, const float *const *b, int ldb, const int *factor_info, int n, int nrhs,
                           int count, cudaStream_t stream);
// Running jobs: x64 <- r32 (assign = 1, the first solve) or x64 += r32 (a correction,
// counted in iters).
cudaError_t launch_ir_update(const IrState &s, int assign, int n, int nrhs, int count, cudaStream_t stream);
// Running jobs: r = b - A x in FP64 from the original FP32 A and b, the normwise backward
// error berr = max|r| / (||A||_inf max|x| + max|b|) and the next state; r goes to r32.  A
// job whose berr did not fall below its previous value takes its last correction back.
cudaError_t launch_ir_residual(const IrState &s, const float *const *a, int lda, const float *const *b, int ldb, int n,
                               int nrhs, int count, double tol, cudaStream_t stream);
// X <- (float) x64 for solved jobs; per matrix, the maximum over its right-hand sides of the
// backward error (NaN for a failed matrix) and of the corrections applied (either output may
// be null).
cudaError_t launch_ir_finish(const IrState &s, float *const *x, int ldx, int n, int nrhs, int count, double *berr,
                             int *iters, cudaStream_t stream);

}  // namespace ops_solver
