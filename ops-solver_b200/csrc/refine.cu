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
constexpr int RT = 256;  // residual block

__device__ __forceinline__ double warp_max_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
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

// One block per (matrix, group of up to RG right-hand sides), so A is read once per group.
// Thread (g = t % 128, c = t / 128) owns rows i0 + 4g .. +3 of a 512-row pass and column half
// c; its four row chains are independent FP64 fused multiply-adds over ascending columns, the
// loads are 16-byte vectors when the layout allows.  The two halves are added in a fixed
// order (c = 0 then c = 1), so the result does not depend on scheduling.
constexpr int RG = 4;
__global__ void __launch_bounds__(RT) ir_residual_kernel(const IrState s, const float *const *a, int lda,
                                                          const float *const *b, int ldb, int n, int nrhs, int count,
                                                          double tol)
{
    extern __shared__ double xs[];               // RG x n
    __shared__ double part[RG][512], rsum[512];  // the c = 1 half's partial sums
    __shared__ double red[(2 + 3 * RG) * (RT / 32)];
    __shared__ int decide[RG];                   // per right-hand side: 1 accept, 2 first, 0 take back, 3 idle
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int g = t & 127, c = t >> 7;
    const int groups = (nrhs + RG - 1) / RG;
    const int half = (n + 1) / 2;
    const int jb = c == 0 ? 0 : half, je = c == 0 ? half : n;
    for (int64_t job = blockIdx.x; job < (int64_t)count * groups; job += gridDim.x)
    {
        const int64_t q = job / groups;
        const int r0 = (int)(job % groups) * RG;
        const int nr = min(RG, nrhs - r0);
        bool any = false;
        for (int r = 0; r < nr; ++r) any = any || s.state[q * nrhs + r0 + r] == IR_RUNNING;
        if (!any) continue;  // uniform
        const float *A = slot(a, q);
        const float *B = slot(b, q);
        const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0;
        double mx[RG];
#pragma unroll
        for (int r = 0; r < RG; ++r) mx[r] = 0.0;
        for (int e = t; e < nr * n; e += RT)
        {
            const int r = e / n, i = e % n;
            const double v = s.x64[(q * nrhs + r0 + r) * (int64_t)n + i];
            xs[e] = v;
#pragma unroll
            for (int rr = 0; rr < RG; ++rr)
                if (rr == r) mx[rr] = fmax(mx[rr], fabs(v));
        }
        __syncthreads();
        double mr[RG], mb[RG], ma = 0.0;
#pragma unroll
        for (int r = 0; r < RG; ++r) mr[r] = mb[r] = 0.0;
        for (int i0 = 0; i0 < n; i0 += 512)
        {
            const int ib = i0 + 4 * g;
            double acc[RG][4], arow[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int r = 0; r < RG; ++r)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[r][e] = 0.0;
            if (ib < n)
            {
                const float *base = A + ib;
                auto column = [&](int j, const float (&v)[4]) {
#pragma unroll
                    for (int e = 0; e < 4; ++e) arow[e] += fabs((double)v[e]);
#pragma unroll
                    for (int r = 0; r < RG; ++r)
                    {
                        if (r < nr)
                        {
                            const double xj = xs[r * n + j];
#pragma unroll
                            for (int e = 0; e < 4; ++e) acc[r][e] = fma((double)v[e], xj, acc[r][e]);
                        }
                    }
                };
                if (vec && ib + 3 < n)
                {
                    // 16-byte loads, eight columns in flight before their products (same order)
                    int j = jb;
                    for (; j + 8 <= je; j += 8)
                    {
                        float4 f[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                            f[u] = __ldg(reinterpret_cast<const float4 *>(base + (int64_t)(j + u) * lda));
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                        {
                            const float v[4] = {f[u].x, f[u].y, f[u].z, f[u].w};
                            column(j + u, v);
                        }
                    }
                    for (; j < je; ++j)
                    {
                        const float4 f = __ldg(reinterpret_cast<const float4 *>(base + (int64_t)j * lda));
                        const float v[4] = {f.x, f.y, f.z, f.w};
                        column(j, v);
                    }
                }
                else
                {
                    for (int j = jb; j < je; ++j)
                    {
                        float v[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) v[e] = ib + e < n ? base[(int64_t)j * lda + e] : 0.0f;
                        column(j, v);
                    }
                }
            }
            if (c == 1)
            {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                {
                    rsum[4 * g + e] = arow[e];
#pragma unroll
                    for (int r = 0; r < RG; ++r) part[r][4 * g + e] = acc[r][e];
                }
            }
            __syncthreads();
            if (c == 0)
            {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                {
                    const int i = ib + e;
                    if (i < n)
                    {
                        ma = fmax(ma, arow[e] + rsum[4 * g + e]);
#pragma unroll
                        for (int r = 0; r < RG; ++r)
                        {
                            if (r < nr)
                            {
                                const double bi = (double)B[(int64_t)(r0 + r) * ldb + i];
                                const double ri = bi - (acc[r][e] + part[r][4 * g + e]);
                                mr[r] = fmax(mr[r], fabs(ri));
                                mb[r] = fmax(mb[r], fabs(bi));
                                // x64 holds r until the decision below (xs keeps x)
                                s.x64[(q * nrhs + r0 + r) * (int64_t)n + i] = ri;
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
        // block maxima: ||A||_inf, then max |r|, max |b|, max |x| per right-hand side
        {
            double v[2 + 3 * RG];
            v[0] = ma;
            v[1] = 0.0;
#pragma unroll
            for (int r = 0; r < RG; ++r)
            {
                v[2 + r] = mr[r];
                v[2 + RG + r] = mb[r];
                v[2 + 2 * RG + r] = mx[r];
            }
#pragma unroll
            for (int e = 0; e < 2 + 3 * RG; ++e)
            {
                const double x = warp_max_d(v[e]);
                if (lane == 0) red[e * (RT / 32) + warp] = x;
            }
            __syncthreads();
            if (t < nr)
            {
                double m4[4];
                const int idx[4] = {2 + t, 0, 2 + RG + t, 2 + 2 * RG + t};
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    double x = red[idx[k] * (RT / 32)];
                    for (int w = 1; w < RT / 32; ++w) x = fmax(x, red[idx[k] * (RT / 32) + w]);
                    m4[k] = x;
                }
                const int64_t job_r = q * nrhs + r0 + t;
                const double den = m4[1] * m4[3] + m4[2];
                const double berr = den > 0.0 ? m4[0] / den : 0.0;
                const double prev = s.berr[job_r];
                const bool better = berr < prev;        // false for a NaN berr
                const bool first = !(prev < HUGE_VAL);  // x is the first solve: nothing to take back
                if (s.state[job_r] != IR_RUNNING)
                    decide[t] = 3;  // not refined in this pass: x stays as it was
                else
                {
                    decide[t] = better ? 1 : (first ? 2 : 0);
                    if (better || first) s.berr[job_r] = berr;
                    if (!better && !first) s.iters[job_r] -= 1;
                    s.state[job_r] = !better ? IR_STALLED
                                             : (berr <= tol ? IR_CONVERGED
                                                            : (berr > 0.5 * prev ? IR_STALLED : IR_RUNNING));
                }
            }
            __syncthreads();
        }
        for (int e = t; e < nr * n; e += RT)
        {
            const int r = e / n, i = e % n;
            const int64_t off = (q * nrhs + r0 + r) * (int64_t)n + i;
            const int d = decide[r];
            if (d == 1) s.r32[off] = (float)s.x64[off];
            // accept, first or idle: x stays; take back: x minus the last correction
            s.x64[off] = d == 0 ? xs[e] - (double)s.r32[off] : xs[e];
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

size_t ir_residual_smem(int n) { return (size_t)RG * n * sizeof(double); }

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
    const int64_t groups = (nrhs + RG - 1) / RG;
    ir_residual_kernel<<<grid((int64_t)count * groups), RT, smem, stream>>>(s, a, lda, b, ldb, n, nrhs, count, tol);
    return cudaGetLastError();
}

cudaError_t launch_ir_finish(const IrState &s, float *const *x, int ldx, int n, int nrhs, int count, double *berr,
                             int *iters, cudaStream_t stream)
{
    ir_finish_kernel<<<grid((int64_t)count * nrhs), 128, 0, stream>>>(s, x, ldx, n, nrhs, count, berr, iters);
    return cudaGetLastError();
}

}  // namespace ops_solver
