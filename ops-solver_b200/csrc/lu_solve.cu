// lu_solve.cu -- LU solve P A X = B for orders above the register-resident kernels
// (64 < n <= 8192), one block per (matrix, group of up to 8 right-hand sides).
//
// Order (the oracle's orc_sgetrs, trans 0): row interchanges applied in sequence, then the
// unit-lower forward sweep x_i = fma(-l_ik, x_k, x_i) in ascending k, then the upper sweep
// x_k = x_k / u_kk, x_i = fma(-u_ik, x_k, x_i) in descending k.  Blocking keeps every
// element's sequence: columns go in blocks of 32; the 32 x 32 diagonal triangle is solved by
// one warp with shuffles, then every other row of the block column takes its 32 updates in
// order (rows staged in chunks of 512 through shared memory).
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int ST = 256;     // threads per block
constexpr int KB = 32;      // column block
constexpr int RC = 512;     // staged rows per chunk
constexpr int MAX_RHS_PER_BLOCK = 8;

__global__ void __launch_bounds__(ST) getrs_blocked_kernel(float *a_single, float *const *a_table, int a_first,
                                                            const int *ipiv, float *b_single, float *const *b_table,
                                                            int b_first, int n, int lda,
                                                            int ldb, int nrhs, int count, int RHS, int *info,
                                                            const int *skip)
{
    extern __shared__ float sm[];
    float *x = sm;                        // RHS x n  (RHS = right-hand sides per block)
    float *lt = sm + (size_t)RHS * n;     // KB x (RC + 1) staged block column (column-major)
    __shared__ int bad;
    const int groups = (nrhs + RHS - 1) / RHS;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int64_t job = blockIdx.x; job < (int64_t)count * groups; job += gridDim.x)
    {
        const int64_t q = job / groups;
        const int r0 = (int)(job % groups) * RHS;
        const int nr = min(RHS, nrhs - r0);
        if (skip)
        {
            bool all_done = true;
            for (int r = 0; r < nr; ++r) all_done = all_done && skip[q * nrhs + r0 + r] != 0;
            if (all_done) continue;  // uniform across the block
        }
        const float *A = a_table ? slot(a_table, a_first + q) : a_single;
        float *B = b_table ? slot(b_table, b_first + q) : b_single;
        const int *piv = ipiv ? ipiv + q * n : nullptr;
        if (!A || !B)
        {
            if (t == 0 && info && r0 == 0) info[q] = !A ? -4 : -7;
            continue;
        }
        if (t == 0) bad = 0;
        __syncthreads();
        if (piv)
            for (int k = t; k < n; k += ST)
                if (piv[k] < k + 1 || piv[k] > n) bad = 1;
        for (int e = t; e < RHS * n; e += ST)
        {
            const int r = e / n, i = e % n;
            x[e] = r < nr ? B[(int64_t)(r0 + r) * ldb + i] : 0.0f;
        }
        __syncthreads();
        if (bad)
        {
            if (t == 0 && info && r0 == 0) info[q] = -6;
            __syncthreads();
            continue;
        }
        // interchanges, in order: one thread per right-hand side
        if (piv && t < nr)
            for (int k = 0; k < n; ++k)
            {
                const int p = piv[k] - 1;
                if (p != k)
                {
                    const float v = x[t * n + k];
                    x[t * n + k] = x[t * n + p];
                    x[t * n + p] = v;
                }
            }
        __syncthreads();
        // forward, unit lower
        for (int kb = 0; kb < n; kb += KB)
        {
            const int w = min(KB, n - kb);
            // diagonal triangle: warp r solves right-hand side r
            if (warp < nr)
            {
                float xv = lane < w ? x[warp * n + kb + lane] : 0.0f;
                for (int k = 0; k < w; ++k)
                {
                    const float xk = __shfl_sync(0xffffffffu, xv, k);
                    const float l = lane < w ? A[(int64_t)(kb + k) * lda + kb + lane] : 0.0f;
                    if (lane > k && lane < w) xv = fma_rn(-l, xk, xv);
                }
                if (lane < w) x[warp * n + kb + lane] = xv;
            }
            __syncthreads();
            // rows below the block, staged in chunks
            for (int c0 = kb + w; c0 < n; c0 += RC)
            {
                const int rows = min(RC, n - c0);
                for (int e = t; e < w * rows; e += ST)
                {
                    const int k = e / rows, i = e % rows;
                    lt[k * (RC + 1) + i] = A[(int64_t)(kb + k) * lda + c0 + i];
                }
                __syncthreads();
                for (int e = t; e < nr * rows; e += ST)
                {
                    const int r = e / rows, i = e % rows;
                    float v = x[r * n + c0 + i];
                    for (int k = 0; k < w; ++k) v = fma_rn(-lt[k * (RC + 1) + i], x[r * n + kb + k], v);
                    x[r * n + c0 + i] = v;
                }
                __syncthreads();
            }
        }
        // backward, upper
        for (int ke = n; ke > 0; ke -= KB)
        {
            const int kb = max(0, ke - KB);
            const int w = ke - kb;
            if (warp < nr)
            {
                float xv = lane < w ? x[warp * n + kb + lane] : 0.0f;
                for (int k = w - 1; k >= 0; --k)
                {
                    const float dk = A[(int64_t)(kb + k) * lda + kb + k];
                    if (lane == k) xv = div_rn(xv, dk);
                    const float xk = __shfl_sync(0xffffffffu, xv, k);
                    const float u = lane < w ? A[(int64_t)(kb + k) * lda + kb + lane] : 0.0f;
                    if (lane < k) xv = fma_rn(-u, xk, xv);
                }
                if (lane < w) x[warp * n + kb + lane] = xv;
            }
            __syncthreads();
            for (int c0 = 0; c0 < kb; c0 += RC)
            {
                const int rows = min(RC, kb - c0);
                for (int e = t; e < w * rows; e += ST)
                {
                    const int k = e / rows, i = e % rows;
                    lt[k * (RC + 1) + i] = A[(int64_t)(kb + k) * lda + c0 + i];
                }
                __syncthreads();
                for (int e = t; e < nr * rows; e += ST)
                {
                    const int r = e / rows, i = e % rows;
                    float v = x[r * n + c0 + i];
                    for (int k = w - 1; k >= 0; --k) v = fma_rn(-lt[k * (RC + 1) + i], x[r * n + kb + k], v);
                    x[r * n + c0 + i] = v;
                }
                __syncthreads();
            }
        }
        for (int e = t; e < nr * n; e += ST)
        {
            const int r = e / n, i = e % n;
            B[(int64_t)(r0 + r) * ldb + i] = x[e];
        }
        if (t == 0 && info && r0 == 0) info[q] = 0;
        __syncthreads();
    }
}
}  // namespace

cudaError_t launch_getrs_blocked(const RealBatch &a, const int *ipiv, const RealBatch &b, int nrhs, int *info,
                                 const int *skip, cudaStream_t stream)
{
    const size_t budget = 220 * 1024 / sizeof(float) - (size_t)KB * (RC + 1);
    int rpb = (int)(budget / (size_t)a.n);
    if (rpb > MAX_RHS_PER_BLOCK) rpb = MAX_RHS_PER_BLOCK;
    if (rpb > nrhs) rpb = nrhs;
    if (rpb < 1) return cudaErrorInvalidValue;
    const size_t smem = ((size_t)rpb * a.n + (size_t)KB * (RC + 1)) * sizeof(float);
    cudaFuncSetAttribute(getrs_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int groups = (nrhs + rpb - 1) / rpb;
    int64_t jobs = (int64_t)a.count * groups;
    int64_t blocks = jobs < 148 * 8 ? jobs : 148 * 8;
    if (blocks < 1) blocks = 1;
    getrs_blocked_kernel<<<(unsigned)blocks, ST, smem, stream>>>(a.single, a.table, a.first, ipiv, b.single,
                                                                 b.table, b.first, a.n,
                                                                 a.ld, b.ld, nrhs, a.count, rpb, info, skip);
    return cudaGetLastError();
}

}  // namespace ops_solver
