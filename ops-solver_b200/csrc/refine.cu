// refine.cu -- FP64 iterative refinement around an LU factorisation of any precision.
//
// For each system A x = b (A and b the caller's FP32 data, never modified):
//   x0 = solve(LU, b) in FP32, kept in FP64
//   repeat: r = b - A x with FP64 fused multiply-adds, berr = max|r| / (||A||_inf max|x| + max|b|)
//           stop when berr <= tol, or when berr stops halving (then the better iterate stays)
//           d = solve(LU, r) in FP32;  x = x + d in FP64
// The residual and the update are the only FP64 steps.  The scheme is classic mixed-
// precision refinement (Wilkinson; Moler 1967; Langou et al. 2006): it converges to FP32
// backward error while kappa(A) times the factorisation's unit roundoff stays below one.
#include <math.h>

#include "common.cuh"
#include "refine.h"

namespace ops_solver
{
namespace
{
constexpr int RT = 256;  // residual block: 64 rows x 4 column quarters
constexpr int RQ = 4;

__device__ __forceinline__ double warp_max_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block maximum of four values at once (one barrier pair).
__device__ void block_max4(double (&v)[4], double *red)
{
#pragma unroll
    for (int e = 0; e < 4; ++e) v[e] = warp_max_d(v[e]);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int e = 0; e < 4; ++e) red[e * (RT / 32) + (threadIdx.x >> 5)] = v[e];
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 4; ++e)
    {
        double r = red[e * (RT / 32)];
        for (int w = 1; w < RT / 32; ++w) r = fmax(r, red[e * (RT / 32) + w]);
        v[e] = r;
    }
    __syncthreads();
}

__global__ void ir_init_kernel(const IrState s, const float *const *b, int ldb, const int *factor_info, int n,
                               int nrhs, int count)
{
    for (int64_t job = blockIdx.x; job < (int64_t)count * nrhs; job += gridDim.x)
    {
        const int64_t q = job / nrhs;
        const int r = (int)(job % nrhs);
        const float *bq = slot(b, q) + (int64_t)r * ldb;
        float *dst = s.r32 + job * (int64_t)n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = bq[i];
        if (threadIdx.x == 0)
        {
            s.berr[job] = HUGE_VAL;
            s.state[job] = factor_info[q] != 0 ? IR_FAILED : IR_RUNNING;
            s.iters[job] = 0;
        }
    }
}

__global__ void ir_update_kernel(const IrState s, int assign, int n, int nrhs, int count)
{
    for (int64_t job = blockIdx.x; job < (int64_t)count * nrhs; job += gridDim.x)
    {
        if (s.state[job] != IR_RUNNING) continue;
        double *x = s.x64 + job * (int64_t)n;
        const float *d = s.r32 + job * (int64_t)n;
        if (assign)
            for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (double)d[i];
        else
            for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] += (double)d[i];
        if (!assign && threadIdx.x == 0) s.iters[job] += 1;
    }
}

// One block per running job; rows go in chunks of 64.  Thread (g = t % 64, c = t / 64)
// forms the partial sum of row i0 + g over column quarter c; the four partials are added in
// a fixed order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(RT) ir_residual_kernel(const IrState s, const float *const *a, int lda,
                                                          const float *const *b, int ldb, int n, int nrhs, int count,
                                                          double tol)
{
    extern __shared__ double xs[];  // n
    __shared__ double part[RQ][RT / RQ], rowsum[RQ][RT / RQ];
    __shared__ double red[4 * (RT / 32)];
    const int t = threadIdx.x;
    const int g = t % (RT / RQ), c = t / (RT / RQ);
    const int span = (n + RQ - 1) / RQ;
    const int j0 = min(n, c * span), j1 = min(n, j0 + span);
    for (int64_t job = blockIdx.x; job < (int64_t)count * nrhs; job += gridDim.x)
    {
        if (s.state[job] != IR_RUNNING) continue;  // uniform
        const int64_t q = job / nrhs;
        const int r = (int)(job % nrhs);
        const float *A = slot(a, q);
        const float *bq = slot(b, q) + (int64_t)r * ldb;
        double *x = s.x64 + job * (int64_t)n;
        float *rv = s.r32 + job * (int64_t)n;
        double m[4] = {0.0, 0.0, 0.0, 0.0};  // max |r|, ||A||_inf, max |b|, max |x|
        for (int i = t; i < n; i += RT)
        {
            xs[i] = x[i];
            m[3] = fmax(m[3], fabs(xs[i]));
        }
        __syncthreads();
        const double prev = s.berr[job];
        for (int i0 = 0; i0 < n; i0 += RT / RQ)
        {
            const int i = i0 + g;
            double acc = 0.0, arow = 0.0;
            if (i < n)
            {
                const float *col = A + i;
#pragma unroll 8
                for (int j = j0; j < j1; ++j)
                {
                    const double aij = (double)col[(int64_t)j * lda];
                    acc = fma(aij, xs[j], acc);
                    arow += fabs(aij);
                }
            }
            part[c][g] = acc;
            rowsum[c][g] = arow;
            __syncthreads();
            if (c == 0 && i < n)
            {
                const double ax = ((part[0][g] + part[1][g]) + part[2][g]) + part[3][g];
                const double as = ((rowsum[0][g] + rowsum[1][g]) + rowsum[2][g]) + rowsum[3][g];
                const double bi = (double)bq[i];
                const double ri = bi - ax;
                m[0] = fmax(m[0], fabs(ri));
                m[1] = fmax(m[1], as);
                m[2] = fmax(m[2], fabs(bi));
                x[i] = ri;  // x64 holds r until the decision below (xs keeps x)
            }
            __syncthreads();
        }
        block_max4(m, red);
        const double den = m[1] * m[3] + m[2];
        const double berr = den > 0.0 ? m[0] / den : 0.0;
        const bool better = berr < prev;        // false for a NaN berr
        const bool first = !(prev < HUGE_VAL);  // x is the first solve: nothing to take back
        for (int i = t; i < n; i += RT)
        {
            const double ri = x[i];
            if (better) rv[i] = (float)ri;
            x[i] = better || first ? xs[i] : xs[i] - (double)rv[i];  // else: the last correction back
        }
        if (t == 0)
        {
            if (better || first) s.berr[job] = berr;
            if (!better && !first) s.iters[job] -= 1;
            s.state[job] = !better ? IR_STALLED
                                   : (berr <= tol ? IR_CONVERGED : (berr > 0.5 * prev ? IR_STALLED : IR_RUNNING));
        }
        __syncthreads();
    }
}

__global__ void ir_finish_kernel(const IrState s, float *const *xout, int ldx, int n, int nrhs, int count,
                                 double *berr_out, int *iter_out)
{
    for (int64_t job = blockIdx.x; job < (int64_t)count * nrhs; job += gridDim.x)
    {
        const int64_t q = job / nrhs;
        const int r = (int)(job % nrhs);
        const bool failed = s.state[job] == IR_FAILED;
        if (!failed)
        {
            float *X = slot(xout, q) + (int64_t)r * ldx;
            const double *x = s.x64 + job * (int64_t)n;
            for (int i = threadIdx.x; i < n; i += blockDim.x) X[i] = (float)x[i];
        }
        if (threadIdx.x == 0 && r == 0)
        {
            double mx = 0.0;
            int it = 0;
            for (int k = 0; k < nrhs; ++k)
            {
                const double e = s.berr[q * nrhs + k];
                mx = e != e ? e : (mx != mx ? mx : fmax(mx, e));  // a NaN propagates
                it = max(it, s.iters[q * nrhs + k]);
            }
            if (berr_out) berr_out[q] = failed ? NAN : mx;
            if (iter_out) iter_out[q] = it;
        }
    }
}

unsigned grid(int64_t jobs) { return (unsigned)(jobs < 148 * 8 ? (jobs < 1 ? 1 : jobs) : 148 * 8); }
}  // namespace

size_t ir_residual_smem(int n) { return (size_t)n * sizeof(double); }

cudaError_t launch_ir_init(const IrState &s, const float *const *b, int ldb, const int *factor_info, int n, int nrhs,
                           int count, cudaStream_t stream)
{
    ir_init_kernel<<<grid((int64_t)count * nrhs), 128, 0, stream>>>(s, b, ldb, factor_info, n, nrhs, count);
    return cudaGetLastError();
}

cudaError_t launch_ir_update(const IrState &s, int assign, int n, int nrhs, int count, cudaStream_t stream)
{
    ir_update_kernel<<<grid((int64_t)count * nrhs), 128, 0, stream>>>(s, assign, n, nrhs, count);
    return cudaGetLastError();
}

cudaError_t launch_ir_residual(const IrState &s, const float *const *a, int lda, const float *const *b, int ldb, int n,
                               int nrhs, int count, double tol, cudaStream_t stream)
{
    const size_t smem = ir_residual_smem(n);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaFuncSetAttribute(ir_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ir_residual_kernel<<<grid((int64_t)count * nrhs), RT, smem, stream>>>(s, a, lda, b, ldb, n, nrhs, count, tol);
    return cudaGetLastError();
}

cudaError_t launch_ir_finish(const IrState &s, float *const *x, int ldx, int n, int nrhs, int count, double *berr,
                             int *iters, cudaStream_t stream)
{
    ir_finish_kernel<<<grid((int64_t)count * nrhs), 128, 0, stream>>>(s, x, ldx, n, nrhs, count, berr, iters);
    return cudaGetLastError();
}

}  // namespace ops_solver
