// complex_chol.cu -- batched complex64 Cholesky factor and solve (uniform order per call)
// and the uneven-order persistent kernel, sm_100a.
//
// Arithmetic (restated in oracle/oracle.c, orc_cpotrf / orc_cpotrs):
//   factor, right-looking: d = Re(a_kk) must satisfy d > 0 and d <= FLT_MAX, s = sqrt(d)
//   (IEEE), l_kk = (s, 0), l_ik = (Re a_ik / s, Im a_ik / s) (IEEE), and every trailing
//   a_ij -= l_ik * conj(l_jk) as four FMAs in ascending k:
//       re = fma(-ar, cr, re); re = fma(-ai, ci, re); im = fma(-ai, cr, im); im = fma(ar, ci, im)
//   with l_ik = (ar, ai), l_jk = (cr, ci).  A failed matrix keeps its completed columns.
//   solve: forward z_i -= l_ik * y_k (y_k = z_k / l_kk) and backward z_i -= conj(l_ki) * x_k,
//   both right-looking, the complex products again as two FMAs per component; above order
//   240 in blocks of 64 rows, the rows outside a block taking it as one partial sum from
//   zero and one subtraction (orc_cpotrs_blocked).
// The reference's own kernels (src/cpotrf/arch35) keep a compensated double-float first
// column and diagonal and hand n > 64 to a CATLASS complex GEMM, so parity with them is
// held to the 1e-5 relative tolerance and the reference's complex128 residual gate.
//
// Layouts: n <= 16 -- a width-N sub-warp per matrix, lane i holds row i (re[], im[]) and the
// finished column is broadcast through shared memory; 17..240 -- one block per matrix (64, 128
// or 256 threads), the lower triangle packed in shared memory (n = 240: 226 KB), factored
// left-looking in blocks of 16 columns and solved a warp per right-hand side
// (complex_block.cuh); above 240 the factor runs one matrix at a time over the whole GPU
// (cpotrf_large.cu) and the solve one block per matrix from global memory.
// (A 32-lane register version needs more than 255 registers per lane for the complex rows.)
#include "common.cuh"
#include "complex_block.cuh"
#include "launch_complex.h"

namespace ops_solver
{
namespace
{
constexpr float FLT_MAX_VALUE = 3.402823466e38F;
constexpr int CW_THREADS = 128;

// z -= l * conj(c)
__device__ __forceinline__ void sub_lconj(float &re, float &im, float ar, float ai, float cr, float ci)
{
    re = fma_rn(-ar, cr, re);
    re = fma_rn(-ai, ci, re);
    im = fma_rn(-ai, cr, im);
    im = fma_rn(ar, ci, im);
}
// t += l * y, a block's partial sum in the large-order solve:
//   tr = fma(lr, yr, tr); tr = fma(-li, yi, tr); ti = fma(lr, yi, ti); ti = fma(li, yr, ti)
__device__ __forceinline__ void add_prod(float2 &t, float2 l, float2 y)
{
    t.x = fma_rn(l.x, y.x, t.x);
    t.x = fma_rn(-l.y, y.y, t.x);
    t.y = fma_rn(l.x, y.y, t.y);
    t.y = fma_rn(l.y, y.x, t.y);
}
constexpr int SOLVE_BLOCK = 64;  // rows per block of the large-order solve's partial sums

// z -= l * y
__device__ __forceinline__ void sub_prod(float &re, float &im, float ar, float ai, float yr, float yi)
{
    re = fma_rn(-ar, yr, re);
    re = fma_rn(ai, yi, re);
    im = fma_rn(-ar, yi, im);
    im = fma_rn(-ai, yr, im);
}

// Element (i, j), j <= i, of the lower factor: lower storage reads A[i + j*lda]; upper
// storage reads conj(A[j + i*lda]).
__device__ __forceinline__ float2 load_tri(const float2 *p, int lda, int upper, int i, int j)
{
    if (upper)
    {
        float2 v = p[(int64_t)i * lda + j];
        return make_float2(v.x, -v.y);
    }
    return p[(int64_t)j * lda + i];
}
__device__ __forceinline__ void store_tri(float2 *p, int lda, int upper, int i, int j, float re, float im)
{
    if (upper)
        p[(int64_t)i * lda + j] = make_float2(re, -im);
    else
        p[(int64_t)j * lda + i] = make_float2(re, im);
}

// ---------------------------------------------------------------------------------------
// n <= N <= 32: sub-warp per matrix
// ---------------------------------------------------------------------------------------
// Column K of the right-looking factor, then column K + 1; the recursion keeps every
// register index a compile-time constant.
template <int N, int K>
__device__ __forceinline__ void cfactor_step(float (&re)[N], float (&im)[N], int n, int row, float2 *col,
                                             int &failure)
{
    if constexpr (K < N)
    {
        if (K < n)
        {
            const float d = __shfl_sync(0xffffffffu, re[K], K, N);
            if (!(d > 0.0f && d <= FLT_MAX_VALUE) && failure == 0) failure = K + 1;
            const float s = sqrt_rn(d);
            if (row == K)
            {
                re[K] = s;
                im[K] = 0.0f;
            }
            else
            {
                re[K] = div_rn(re[K], s);
                im[K] = div_rn(im[K], s);
            }
            __syncwarp();
            col[row] = make_float2(re[K], im[K]);
            __syncwarp();
#pragma unroll
            for (int j = K + 1; j < N; ++j)
            {
                if (j < n)
                {
                    const float2 c = col[j];
                    sub_lconj(re[j], im[j], re[K], im[K], c.x, c.y);
                }
            }
            cfactor_step<N, K + 1>(re, im, n, row, col, failure);
        }
    }
}

template <int N>
__device__ __forceinline__ void cpotrf_warp_matrix(float2 *p, int n, int lda, int upper, int row, float2 *col,
                                                   int &failure)
{
    float re[N], im[N];
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
        float2 v = make_float2(0.0f, 0.0f);
        if (p && j < n && row < n && j <= row) v = load_tri(p, lda, upper, row, j);
        re[j] = v.x;
        im[j] = v.y;
    }
    cfactor_step<N, 0>(re, im, n, row, col, failure);
    if (p)
    {
        const int done = failure ? failure - 1 : n;
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (j < done && row < n && j <= row) store_tri(p, lda, upper, row, j, re[j], im[j]);
    }
}

template <int N>
__global__ void __launch_bounds__(CW_THREADS) cpotrf_warp_kernel(float2 *single, float2 *const *table, int n, int lda,
                                                                  int upper, int count, int *info)
{
    constexpr int MPW = 32 / N;
    __shared__ float2 cols[CW_THREADS];
    const int lane = threadIdx.x & 31;
    const int row = lane % N;
    const int sub = lane / N;
    float2 *col = cols + (threadIdx.x & ~31) + sub * N;
    const int warp_global = (blockIdx.x * CW_THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * CW_THREADS) >> 5;
    for (int64_t group = warp_global; group * MPW < count; group += warps_total)
    {
        const int64_t q = group * MPW + sub;
        float2 *p = nullptr;
        if (q < count) p = table ? slot(table, q) : single;
        int failure = 0;
        cpotrf_warp_matrix<N>(p, n, lda, upper, row, col, failure);
        if (q < count && row == 0) info[q] = p ? failure : -3;
    }
}

// ---------------------------------------------------------------------------------------
// 32 < n <= 128: one block per matrix, lower triangle in shared memory
// ---------------------------------------------------------------------------------------
template <int T>
__device__ void cpotrf_block_matrix(float2 *p, int n, int lda, int upper, float2 *sa, int ps, int *flag)
{
    const int t = threadIdx.x;
    for (int j = 0; j < n; ++j)
        for (int i = j + t; i < n; i += T) sa[j * ps + i] = load_tri(p, lda, upper, i, j);
    if (t == 0) *flag = 0;
    __syncthreads();
    int failure = 0;
    for (int k = 0; k < n; ++k)
    {
        const float d = sa[k * ps + k].x;
        if (!(d > 0.0f && d <= FLT_MAX_VALUE))
        {
            failure = k + 1;
            break;  // uniform: every thread read the same d
        }
        const float s = sqrt_rn(d);
        __syncthreads();  // every thread has read d before the column is rewritten
        for (int i = k + t; i < n; i += T)
        {
            float2 v = sa[k * ps + i];
            sa[k * ps + i] = i == k ? make_float2(s, 0.0f) : make_float2(div_rn(v.x, s), div_rn(v.y, s));
        }
        __syncthreads();
        for (int i = k + 1 + t; i < n; i += T)
        {
            const float2 l = sa[k * ps + i];
            for (int j = k + 1; j <= i; ++j)
            {
                const float2 c = sa[k * ps + j];
                float2 z = sa[j * ps + i];
                sub_lconj(z.x, z.y, l.x, l.y, c.x, c.y);
                sa[j * ps + i] = z;
            }
        }
        __syncthreads();
    }
    const int done = failure ? failure - 1 : n;
    for (int j = 0; j < done; ++j)
        for (int i = j + t; i < n; i += T)
        {
            float2 v = sa[j * ps + i];
            store_tri(p, lda, upper, i, j, v.x, v.y);
        }
    if (t == 0) *flag = failure;
    __syncthreads();
}

template <int T>
__global__ void __launch_bounds__(T) cpotrf_block_kernel(float2 *single, float2 *const *table, int n, int lda,
                                                          int upper, int count, int *info)
{
    extern __shared__ float2 sa[];
    __shared__ int flag;
    const int ps = n + 1;
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        float2 *p = table ? slot(table, q) : single;
        if (!p)
        {
            if (threadIdx.x == 0) info[q] = -3;
            continue;
        }
        cpotrf_block_matrix<T>(p, n, lda, upper, sa, ps, &flag);
        if (threadIdx.x == 0) info[q] = flag;
        __syncthreads();
    }
}

// 17..128: the packed-triangle block routine, a matrix per block (grid-stride).
template <int T>
__global__ void __launch_bounds__(T) cpotrf_cb_kernel(float2 *single, float2 *const *table, int n, int lda, int upper,
                                                      int count, int *info)
{
    extern __shared__ __align__(16) float cb_mem[];
    const CbShared s = cb_carve(cb_mem, n);
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        float2 *p = table ? slot(table, q) : single;
        if (!p)
        {
            if (threadIdx.x == 0) info[q] = -3;
            continue;
        }
        cb_load<T>(s, p, lda, upper, n);
        __syncthreads();
        const int failure = cb_factor<T>(s, n);
        cb_store<T>(s, p, lda, upper, n, failure ? failure - 1 : n);
        if (threadIdx.x == 0) info[q] = failure;
        __syncthreads();
    }
}

template <int T>
__global__ void __launch_bounds__(T) cpotrs_cb_kernel(const float2 *a_single, const float2 *const *a_table,
                                                      float2 *b_single, float2 *const *b_table, int n, int lda, int ldb,
                                                      int nrhs, int upper, int count, const int *info)
{
    extern __shared__ __align__(16) float cb_mem[];
    if (info && info[0] != 0) return;
    const CbShared s = cb_carve(cb_mem, n);
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        const float2 *pa = a_table ? slot(a_table, q) : a_single;
        float2 *pb = b_table ? slot(b_table, q) : b_single;
        if (!pa || !pb) continue;
        cb_load<T>(s, pa, lda, upper, n);
        __syncthreads();
        cb_solve<T>(s, n, pb, ldb, nrhs);
    }
}

// ---------------------------------------------------------------------------------------
// solve (any n): one block per matrix, L staged in shared memory when it fits, rows over
// threads, right-looking sweeps; right-hand sides one after another.
// ---------------------------------------------------------------------------------------
template <bool STAGED>
__global__ void __launch_bounds__(128) cpotrs_block_kernel(const float2 *a_single, const float2 *const *a_table,
                                                            float2 *b_single, float2 *const *b_table, int n, int lda,
                                                            int ldb, int nrhs, int upper, int count, const int *info)
{
    extern __shared__ float2 sm[];
    if (info && info[0] != 0) return;
    const int ps = n + 1;
    float2 *sl = sm;                                  // staged L (STAGED)
    float2 *x = STAGED ? sm + (size_t)n * ps : sm;    // n
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        const float2 *pa = a_table ? slot(a_table, q) : a_single;
        float2 *pb = b_table ? slot(b_table, q) : b_single;
        if (!pa || !pb) continue;
        auto L = [&](int i, int j) -> float2
        { return STAGED ? sl[j * ps + i] : load_tri(pa, lda, upper, i, j); };
        if (STAGED)
        {
            for (int j = 0; j < n; ++j)
                for (int i = j + threadIdx.x; i < n; i += 128) sl[j * ps + i] = load_tri(pa, lda, upper, i, j);
        }
        __syncthreads();
        for (int r = 0; r < nrhs; ++r)
        {
            float2 *xb = pb + (int64_t)r * ldb;
            for (int i = threadIdx.x; i < n; i += 128) x[i] = xb[i];
            __syncthreads();
            // forward in blocks of SOLVE_BLOCK rows: inside a block y_k = z_k / l_kk and the
            // block's later rows take z_i -= l_ik y_k; the rows below take the block as one
            // partial sum t = sum_k l_ik y_k from zero (ascending k), then z_i - t
            for (int K0 = 0; K0 < n; K0 += SOLVE_BLOCK)
            {
                const int kend = min(K0 + SOLVE_BLOCK, n);
                for (int k = K0; k < kend; ++k)
                {
                    const float dk = L(k, k).x;
                    const float2 zk = x[k];
                    const float yr = div_rn(zk.x, dk), yi = div_rn(zk.y, dk);
                    for (int i = k + 1 + threadIdx.x; i < kend; i += 128)
                    {
                        const float2 l = L(i, k);
                        float2 z = x[i];
                        sub_prod(z.x, z.y, l.x, l.y, yr, yi);
                        x[i] = z;
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) x[k] = make_float2(yr, yi);
                    __syncthreads();
                }
                for (int i = kend + threadIdx.x; i < n; i += 128)
                {
                    float2 t = make_float2(0.0f, 0.0f);
                    for (int k = K0; k < kend; ++k) add_prod(t, L(i, k), x[k]);
                    x[i] = make_float2(sub_rn(x[i].x, t.x), sub_rn(x[i].y, t.y));
                }
                __syncthreads();
            }
            // backward, blocks in descending order, with conj(l_ki)
            for (int K0 = ((n - 1) / SOLVE_BLOCK) * SOLVE_BLOCK; n > 0 && K0 >= 0; K0 -= SOLVE_BLOCK)
            {
                const int kend = min(K0 + SOLVE_BLOCK, n);
                for (int k = kend - 1; k >= K0; --k)
                {
                    const float dk = L(k, k).x;
                    const float2 zk = x[k];
                    const float yr = div_rn(zk.x, dk), yi = div_rn(zk.y, dk);
                    for (int i = K0 + threadIdx.x; i < k; i += 128)
                    {
                        const float2 l = L(k, i);
                        float2 z = x[i];
                        sub_prod(z.x, z.y, l.x, -l.y, yr, yi);
                        x[i] = z;
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) x[k] = make_float2(yr, yi);
                    __syncthreads();
                }
                for (int i = threadIdx.x; i < K0; i += 128)
                {
                    float2 t = make_float2(0.0f, 0.0f);
                    for (int k = K0; k < kend; ++k)
                    {
                        const float2 l = L(k, i);
                        add_prod(t, make_float2(l.x, -l.y), x[k]);
                    }
                    x[i] = make_float2(sub_rn(x[i].x, t.x), sub_rn(x[i].y, t.y));
                }
                __syncthreads();
            }
            for (int i = threadIdx.x; i < n; i += 128) xb[i] = x[i];
            __syncthreads();
        }
    }
}

unsigned grid_of(int64_t count, int64_t per_block, int64_t cap)
{
    int64_t g = (count + per_block - 1) / per_block;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}
}  // namespace

cudaError_t launch_cpotrf(float2 *single, float2 *const *table, int n, int lda, int upper, int count, int *info,
                          cudaStream_t stream)
{
    if (n <= 8)
        cpotrf_warp_kernel<8><<<grid_of(count, 16, 148 * 64), CW_THREADS, 0, stream>>>(single, table, n, lda, upper,
                                                                                       count, info);
    else if (n <= 16)
        cpotrf_warp_kernel<16><<<grid_of(count, 8, 148 * 64), CW_THREADS, 0, stream>>>(single, table, n, lda, upper,
                                                                                       count, info);
    else if (n <= 64)
    {
        const size_t smem = cb_smem_bytes(n);
        cudaFuncSetAttribute(cpotrf_cb_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cpotrf_cb_kernel<64><<<grid_of(count, 1, 148 * 16), 64, smem, stream>>>(single, table, n, lda, upper, count,
                                                                                info);
    }
    else if (n <= 128)
    {
        const size_t smem = cb_smem_bytes(n);
        cudaFuncSetAttribute(cpotrf_cb_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cpotrf_cb_kernel<128><<<grid_of(count, 1, 148 * 8), 128, smem, stream>>>(single, table, n, lda, upper,
                                                                                count, info);
    }
    else if (n <= CPOTRF_PACKED_MAX)
    {
        const size_t smem = cb_smem_bytes(n);
        cudaFuncSetAttribute(cpotrf_cb_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cpotrf_cb_kernel<256><<<grid_of(count, 1, 148 * 2), 256, smem, stream>>>(single, table, n, lda, upper,
                                                                                count, info);
    }
    else
        return cudaErrorInvalidValue;  // one matrix at a time over the whole GPU: launch_cpotrf_large
    return cudaGetLastError();
}

cudaError_t launch_cpotrs(const float2 *a_single, const float2 *const *a_table, float2 *b_single,
                          float2 *const *b_table, int n, int lda, int ldb, int nrhs, int upper, int count,
                          const int *info, cudaStream_t stream)
{
    if (n > 16 && n <= CPOTRF_PACKED_MAX)
    {
        const size_t smem = cb_smem_bytes(n);
        if (n <= 64)
        {
            cudaFuncSetAttribute(cpotrs_cb_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cpotrs_cb_kernel<64><<<grid_of(count, 1, 148 * 16), 64, smem, stream>>>(
                a_single, a_table, b_single, b_table, n, lda, ldb, nrhs, upper, count, info);
        }
        else if (n <= 128)
        {
            cudaFuncSetAttribute(cpotrs_cb_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cpotrs_cb_kernel<128><<<grid_of(count, 1, 148 * 8), 128, smem, stream>>>(
                a_single, a_table, b_single, b_table, n, lda, ldb, nrhs, upper, count, info);
        }
        else
        {
            cudaFuncSetAttribute(cpotrs_cb_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cpotrs_cb_kernel<256><<<grid_of(count, 1, 148 * 2), 256, smem, stream>>>(
                a_single, a_table, b_single, b_table, n, lda, ldb, nrhs, upper, count, info);
        }
        return cudaGetLastError();
    }
    size_t staged = ((size_t)n * (n + 1) + n) * sizeof(float2);
    if (staged <= 200 * 1024)
    {
        cudaFuncSetAttribute(cpotrs_block_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged);
        cpotrs_block_kernel<true><<<grid_of(count, 1, 148 * 8), 128, staged, stream>>>(
            a_single, a_table, b_single, b_table, n, lda, ldb, nrhs, upper, count, info);
    }
    else
    {
        size_t smem = (size_t)n * sizeof(float2);
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(cpotrs_block_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cpotrs_block_kernel<false><<<grid_of(count, 1, 148 * 8), 128, smem, stream>>>(
            a_single, a_table, b_single, b_table, n, lda, ldb, nrhs, upper, count, info);
    }
    return cudaGetLastError();
}

}  // namespace ops_solver
