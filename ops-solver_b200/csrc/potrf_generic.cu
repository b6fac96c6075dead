// potrf_generic.cu -- real Cholesky solve for 32 < n <= 4096, any batch (the factorisation
// above order 32 is in potrf_blocked.cu).
//
// Solve orders (the parity contract, oracle orc_spotrs):
//   DOT   (33..128): dot accumulators, x_k = (b_k - dot_k) / l_kk   (cholesky_vector.cpp:30-122)
//   RIGHT (> 128):   right-looking sweeps in 64-row blocks, fma inside a block and one
//                    partial sum per block for the rows outside it (this build's order)
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int GT = 256;

__device__ __forceinline__ int64_t tri(int lda, int upper, int i, int j)
{
    return upper ? (int64_t)i * lda + j : (int64_t)j * lda + i;
}

constexpr int ORDER_DOT = 1;
constexpr int ORDER_RIGHT = 2;

// The right-looking sweeps of one right-hand side in blocks of SB rows (orc_spotrs_right):
// inside a block the unknowns are finished one at a time and taken into the block's other
// rows by fma; the rows outside the block take the whole block as one partial sum
// t = fma(l, x_k, t) from zero (ascending k), then x_i - t -- the rounding of a blocked
// solve, which the reference's residual gate asks for at large orders.  x in shared memory.
constexpr int SB = 64;
__device__ __forceinline__ void blocked_sweeps(const float *pa, int lda, int upper, int n, float *x)
{
    // forward: L y = b
    for (int K0 = 0; K0 < n; K0 += SB)
    {
        const int kend = min(K0 + SB, n);
        for (int k = K0; k < kend; ++k)
        {
            const float xk = div_rn(x[k], pa[(int64_t)k * (lda + 1)]);
            for (int i = k + 1 + threadIdx.x; i < kend; i += GT) x[i] = fma_rn(-pa[tri(lda, upper, i, k)], xk, x[i]);
            __syncthreads();
            if (threadIdx.x == 0) x[k] = xk;
            __syncthreads();
        }
        for (int i = kend + threadIdx.x; i < n; i += GT)
        {
            float t = 0.0f;
            for (int k = K0; k < kend; ++k) t = fma_rn(pa[tri(lda, upper, i, k)], x[k], t);
            x[i] = sub_rn(x[i], t);
        }
        __syncthreads();
    }
    // backward: L^T x = y, blocks in descending order
    for (int K0 = ((n - 1) / SB) * SB; n > 0 && K0 >= 0; K0 -= SB)
    {
        const int kend = min(K0 + SB, n);
        for (int k = kend - 1; k >= K0; --k)
        {
            const float xk = div_rn(x[k], pa[(int64_t)k * (lda + 1)]);
            for (int i = K0 + threadIdx.x; i < k; i += GT) x[i] = fma_rn(-pa[tri(lda, upper, k, i)], xk, x[i]);
            __syncthreads();
            if (threadIdx.x == 0) x[k] = xk;
            __syncthreads();
        }
        for (int i = threadIdx.x; i < K0; i += GT)
        {
            float t = 0.0f;
            for (int k = K0; k < kend; ++k) t = fma_rn(pa[tri(lda, upper, k, i)], x[k], t);
            x[i] = sub_rn(x[i], t);
        }
        __syncthreads();
    }
}

// One block per (matrix); right-hand sides one after another; x and the accumulators in
// shared memory, rows spread over the threads.
template <int ORDER>
__global__ void __launch_bounds__(GT) potrs_generic_kernel(float *a_single, float *const *a_table, int a_first,
                                                           float *b_single, float *const *b_table, int b_first, int n,
                                                           int lda, int ldb, int nrhs, int upper, int count,
                                                           const int *info)
{
    extern __shared__ float sm[];
    float *x = sm;       // n
    float *dot = sm + n; // n
    if (info[0] != 0) return;
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        const float *pa = a_table ? slot(a_table, a_first + q) : a_single;
        float *pb = b_table ? slot(b_table, b_first + q) : b_single;
        if (!pa || !pb) continue;
        for (int r = 0; r < nrhs; ++r)
        {
            float *xb = pb + (int64_t)r * ldb;
            for (int i = threadIdx.x; i < n; i += GT)
            {
                x[i] = xb[i];
                dot[i] = 0.0f;
            }
            __syncthreads();
            if constexpr (ORDER == ORDER_RIGHT)
            {
                blocked_sweeps(pa, lda, upper, n, x);
                for (int i = threadIdx.x; i < n; i += GT) xb[i] = x[i];
                __syncthreads();
                continue;
            }
            else
            {
            // forward: L x = b
            for (int k = 0; k < n; ++k)
            {
                if (ORDER == ORDER_DOT)
                {
                    const float xk = div_rn(sub_rn(x[k], dot[k]), pa[(int64_t)k * (lda + 1)]);
                    for (int i = k + 1 + threadIdx.x; i < n; i += GT)
                        dot[i] = fma_rn(pa[tri(lda, upper, i, k)], xk, dot[i]);
                    __syncthreads();
                    if (threadIdx.x == 0) x[k] = xk;
                }
                else
                {
                    const float xk = div_rn(x[k], pa[(int64_t)k * (lda + 1)]);
                    for (int i = k + 1 + threadIdx.x; i < n; i += GT) x[i] = fma_rn(-pa[tri(lda, upper, i, k)], xk, x[i]);
                    __syncthreads();
                    if (threadIdx.x == 0) x[k] = xk;
                }
                __syncthreads();
            }
            for (int i = threadIdx.x; i < n; i += GT) dot[i] = 0.0f;
            __syncthreads();
            // backward: L^T x = y
            for (int k = n - 1; k >= 0; --k)
            {
                if (ORDER == ORDER_DOT)
                {
                    const float xk = div_rn(sub_rn(x[k], dot[k]), pa[(int64_t)k * (lda + 1)]);
                    for (int i = threadIdx.x; i < k; i += GT) dot[i] = fma_rn(pa[tri(lda, upper, k, i)], xk, dot[i]);
                    __syncthreads();
                    if (threadIdx.x == 0) x[k] = xk;
                }
                else
                {
                    const float xk = div_rn(x[k], pa[(int64_t)k * (lda + 1)]);
                    for (int i = threadIdx.x; i < k; i += GT) x[i] = fma_rn(-pa[tri(lda, upper, k, i)], xk, x[i]);
                    __syncthreads();
                    if (threadIdx.x == 0) x[k] = xk;
                }
                __syncthreads();
            }
            for (int i = threadIdx.x; i < n; i += GT) xb[i] = x[i];
            __syncthreads();
            }
        }
    }
}

unsigned grid_for(int count)
{
    int64_t g = count;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return (unsigned)g;
}
}  // namespace

cudaError_t launch_potrs_generic(const RealBatch &a, const RealBatch &b, int nrhs, int upper, int dot_order,
                                 const int *info, cudaStream_t stream)
{
    size_t smem = 2 * (size_t)a.n * sizeof(float);
    if (dot_order)
    {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(potrs_generic_kernel<ORDER_DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        potrs_generic_kernel<ORDER_DOT><<<grid_for(a.count), GT, smem, stream>>>(
            a.single, a.table, a.first, b.single, b.table, b.first, a.n, a.ld, b.ld, nrhs, upper, a.count, info);
    }
    else
    {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(potrs_generic_kernel<ORDER_RIGHT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        potrs_generic_kernel<ORDER_RIGHT><<<grid_for(a.count), GT, smem, stream>>>(
            a.single, a.table, a.first, b.single, b.table, b.first, a.n, a.ld, b.ld, nrhs, upper, a.count, info);
    }
    return cudaGetLastError();
}

}  // namespace ops_solver
