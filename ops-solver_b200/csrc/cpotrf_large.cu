// cpotrf_large.cu -- complex64 Cholesky of one matrix above the packed-triangle orders, over
// the whole GPU (aclsolverCpotrf; aclsolverCpotrfBatched takes it one matrix at a time).
//
// Arithmetic (orc_cpotrf_blocked in oracle/oracle.c): inside a 64-column panel every a_ij,
// j <= i, takes the panel's updates a_ij -= l_ik conj(l_jk) as four FMAs in ascending k
// (re = fma(-ar, cr, re); re = fma(-ai, ci, re); im = fma(-ai, cr, im); im = fma(ar, ci, im)
// with l_ik = (ar, ai), l_jk = (cr, ci)); an element right of the panel takes the panel's
// products as one partial sum from zero and one subtraction (see herk below), which keeps
// the rounding at a blocked LAPACK's size, as the reference's residual gate asks.  Then the
// pivot check on d = Re a_jj (d > 0 and d <= FLT_MAX), s = sqrt(d) (IEEE), l_jj = (s, 0),
// and the IEEE division of both components of the column below by s.  The factor is the
// oracle's bit for bit.
//
// Right-looking with 64-column panels; per panel
//   diag:  one block factors the 64 x 64 diagonal block in shared memory;
//   rows:  a thread per row below it forms L21 = A21 L11^-H (ascending k, IEEE divisions),
//          128 rows per block;
//   herk:  the trailing lower triangle takes A22 -= L21 L21^H over 64 x 64 tiles (lower tiles
//          only), both operand panels staged in shared memory, a 4 x 4 tile of complex
//          accumulators per thread: per element the panel's 64 products form one partial
//          sum t from zero (ascending k), then a_ij - t (orc_cpotrf_blocked).
// Failure contract (the reference's): the columns before the failed one keep their factor,
// the failed column and all after it keep the caller's input.  The lower triangle is backed
// up first; every kernel reads info and stops once a pivot has failed, and a restore pass
// copies the backup back into the columns from the failed one on.
// Upper storage (the conjugate transpose) is read and written through the same mapping.
#include "common.cuh"
#include "launch_complex.h"

namespace ops_solver
{
namespace
{
constexpr float FLT_MAX_VALUE = 3.402823466e38F;
constexpr int CPB = 64;       // panel width, herk tile edge
constexpr int CROWS_T = 128;  // panel rows per block of the rows kernel

__device__ __forceinline__ int stopped(const int *info) { return *(volatile const int *)info; }

// Element (i, j), j <= i, of the lower factor: lower storage A[i + j lda], upper storage
// conj(A[j + i lda]).
__device__ __forceinline__ float2 ld(const float2 *A, int lda, int upper, int i, int j)
{
    if (upper)
    {
        const float2 v = A[(int64_t)i * lda + j];
        return make_float2(v.x, -v.y);
    }
    return A[(int64_t)j * lda + i];
}
__device__ __forceinline__ void st(float2 *A, int lda, int upper, int i, int j, float2 v)
{
    if (upper)
        A[(int64_t)i * lda + j] = make_float2(v.x, -v.y);
    else
        A[(int64_t)j * lda + i] = v;
}

// z -= l * conj(c)
__device__ __forceinline__ void sub_lconj(float2 &z, float2 l, float2 c)
{
    z.x = fma_rn(-l.x, c.x, z.x);
    z.x = fma_rn(-l.y, c.y, z.x);
    z.y = fma_rn(-l.y, c.x, z.y);
    z.y = fma_rn(l.x, c.y, z.y);
}

// t += l * conj(c), the partial sum of a panel:
//   tr = fma(ar, cr, tr); tr = fma(ai, ci, tr); ti = fma(ai, cr, ti); ti = fma(-ar, ci, ti)
__device__ __forceinline__ void add_lconj(float2 &t, float2 l, float2 c)
{
    t.x = fma_rn(l.x, c.x, t.x);
    t.x = fma_rn(l.y, c.y, t.x);
    t.y = fma_rn(l.y, c.x, t.y);
    t.y = fma_rn(-l.x, c.y, t.y);
}

__device__ __forceinline__ float2 div2(float2 v, float s, float y, bool ok)
{
    return make_float2(div_by(v.x, s, y, ok), div_by(v.y, s, y, ok));
}

// The 64 x 64 diagonal block at k0, right-looking in shared memory.
__global__ void __launch_bounds__(256) cdiag_kernel(float2 *A, int lda, int upper, int k0, int n, int *info)
{
    __shared__ float2 D[CPB][CPB + 1];  // D[j][i] = element (k0 + i, k0 + j), i >= j
    __shared__ int fail;
    if (stopped(info) != 0) return;
    const int t = threadIdx.x;
    const int w = min(CPB, n - k0);
    for (int e = t; e < CPB * CPB; e += 256)
    {
        const int j = e / CPB, i = e % CPB;
        D[j][i] = (i < w && j < w && i >= j) ? ld(A, lda, upper, k0 + i, k0 + j) : make_float2(0.0f, 0.0f);
    }
    if (t == 0) fail = 0;
    __syncthreads();
    for (int k = 0; k < w; ++k)
    {
        const float d = D[k][k].x;
        if (!(d > 0.0f && d <= FLT_MAX_VALUE))
        {
            if (t == 0) fail = k0 + k + 1;
            break;  // uniform
        }
        const float sq = sqrt_rn(d);
        const float y = div_prepare(sq);
        const bool ok = div_range(sq);
        __syncthreads();  // every thread has read d
        if (t > k && t < w) D[k][t] = div2(D[k][t], sq, y, ok);
        if (t == k) D[k][k] = make_float2(sq, 0.0f);
        __syncthreads();
        for (int e = t; e < CPB * CPB; e += 256)
        {
            const int j = e / CPB, i = e % CPB;
            if (j > k && i >= j && i < w)
            {
                float2 z = D[j][i];
                sub_lconj(z, D[k][i], D[k][j]);
                D[j][i] = z;
            }
        }
        __syncthreads();
    }
    __syncthreads();
    const int done = fail ? fail - 1 - k0 : w;
    for (int e = t; e < CPB * CPB; e += 256)
    {
        const int j = e / CPB, i = e % CPB;
        if (j < done && i >= j && i < w) st(A, lda, upper, k0 + i, k0 + j, D[j][i]);
    }
    if (t == 0 && fail) *info = fail;
}

// L21 of the panel: rows k0 + 64 .. n - 1, a thread per row.  After a failure inside this
// panel the completed columns are still formed.
__global__ void __launch_bounds__(CROWS_T) crows_kernel(float2 *A, int lda, int upper, int k0, int n, int *info)
{
    __shared__ float2 L11[CPB][CPB + 1];  // L11[j][k] = element (k0 + j, k0 + k)
    const int stp = stopped(info);
    int cols = CPB;
    if (stp != 0)
    {
        if (stp < 0 || stp - 1 < k0 || stp - 1 >= k0 + CPB) return;  // stopped before this panel, or an error
        cols = stp - 1 - k0;
        if (cols == 0) return;
    }
    const int t = threadIdx.x;
    for (int e = t; e < CPB * CPB; e += CROWS_T)
    {
        const int j = e / CPB, k = e % CPB;
        L11[j][k] = (k <= j && k0 + j < n) ? ld(A, lda, upper, k0 + j, k0 + k) : make_float2(1.0f, 0.0f);
    }
    __syncthreads();
    const int i = k0 + CPB + blockIdx.x * CROWS_T + t;
    if (i >= n) return;
    float2 z[CPB];
#pragma unroll
    for (int j = 0; j < CPB; ++j) z[j] = j < cols ? ld(A, lda, upper, i, k0 + j) : make_float2(0.0f, 0.0f);
#pragma unroll
    for (int j = 0; j < CPB; ++j)
    {
        if (j < cols)
        {
#pragma unroll
            for (int k = 0; k < j; ++k) sub_lconj(z[j], z[k], L11[j][k]);
            const float d = L11[j][j].x;
            z[j] = div2(z[j], d, div_prepare(d), div_range(d));
        }
    }
#pragma unroll
    for (int j = 0; j < CPB; ++j)
        if (j < cols) st(A, lda, upper, i, k0 + j, z[j]);
}

// The lower tiles of the trailing matrix, tile index -> (tile row ti >= tile column tj).
__device__ __forceinline__ void lower_tile(int idx, int &ti, int &tj)
{
    int r = (int)((sqrtf(8.0f * idx + 1.0f) - 1.0f) * 0.5f);
    while ((r + 1) * (r + 2) / 2 <= idx) ++r;
    while (r * (r + 1) / 2 > idx) --r;
    ti = r;
    tj = idx - r * (r + 1) / 2;
}

struct HerkShared
{
    float2 a[CPB][CPB];  // a[k][r] = element (r0 + r, k0 + k): the tile's rows of L21
    float2 b[CPB][CPB];  // b[k][c] = element (c0 + c, k0 + k): the tile's columns as rows of L21
};

// A22 -= L21 L21^H on the lower tiles; per element the 64 updates in ascending k.
__global__ void __launch_bounds__(256) cherk_kernel(float2 *A, int lda, int upper, int k0, int n, int *info)
{
    extern __shared__ __align__(16) unsigned char herk_mem[];
    HerkShared &sh = *reinterpret_cast<HerkShared *>(herk_mem);
    if (stopped(info) != 0) return;
    const int t = threadIdx.x;
    const int base = k0 + CPB;  // first trailing row / column
    int ti, tj;
    lower_tile(blockIdx.x, ti, tj);
    const int r0 = base + ti * CPB, c0 = base + tj * CPB;
    const float2 zero = make_float2(0.0f, 0.0f);
    for (int e = t; e < CPB * CPB; e += 256)
    {
        const int k = e / CPB, r = e % CPB;
        sh.a[k][r] = r0 + r < n ? ld(A, lda, upper, r0 + r, k0 + k) : zero;
        sh.b[k][r] = c0 + r < n ? ld(A, lda, upper, c0 + r, k0 + k) : zero;
    }
    __syncthreads();
    // thread (tr, tc): rows r0 + 4 tr .. +3, columns c0 + 4 tc .. +3
    const int tr = t & 15, tc = t >> 4;
    const int i0 = r0 + 4 * tr, j0 = c0 + 4 * tc;
    float2 c[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
        {
            const int i = i0 + u, j = j0 + v;
            c[u][v] = (i < n && j <= i) ? ld(A, lda, upper, i, j) : zero;
        }
    // the panel's products as one partial sum per element, t = sum_k l_ik conj(l_jk), then one
    // subtraction per component
    float2 acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = zero;
#pragma unroll 4
    for (int k = 0; k < CPB; ++k)
    {
        const float4 a01 = *reinterpret_cast<const float4 *>(&sh.a[k][4 * tr]);
        const float4 a23 = *reinterpret_cast<const float4 *>(&sh.a[k][4 * tr + 2]);
        const float4 b01 = *reinterpret_cast<const float4 *>(&sh.b[k][4 * tc]);
        const float4 b23 = *reinterpret_cast<const float4 *>(&sh.b[k][4 * tc + 2]);
        const float2 l[4] = {make_float2(a01.x, a01.y), make_float2(a01.z, a01.w), make_float2(a23.x, a23.y),
                             make_float2(a23.z, a23.w)};
        const float2 m[4] = {make_float2(b01.x, b01.y), make_float2(b01.z, b01.w), make_float2(b23.x, b23.y),
                             make_float2(b23.z, b23.w)};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) add_lconj(acc[u][v], l[u], m[v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
        {
            c[u][v].x = sub_rn(c[u][v].x, acc[u][v].x);
            c[u][v].y = sub_rn(c[u][v].y, acc[u][v].y);
        }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
        {
            const int i = i0 + u, j = j0 + v;
            if (i < n && j <= i) st(A, lda, upper, i, j, c[u][v]);
        }
}

// Backup copy of the lower triangle (element (i, j) at W[j * n + i]) and its restore of the
// columns from the failed one on.
__global__ void cbackup_kernel(const float2 *A, int lda, int upper, int n, float2 *W)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        if (i >= j) W[e] = ld(A, lda, upper, i, j);
    }
}
__global__ void crestore_kernel(float2 *A, int lda, int upper, int n, const float2 *W, const int *info)
{
    const int f = *info;
    if (f <= 0) return;
    const int from = f - 1;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        if (j >= from && i >= j) st(A, lda, upper, i, j, W[e]);
    }
}

unsigned elementwise_grid(int64_t elements)
{
    int64_t b = (elements + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return (unsigned)(b < 1 ? 1 : b);
}
}  // namespace

size_t cpotrf_large_scratch_bytes(int n) { return (size_t)n * n * sizeof(float2); }

cudaError_t launch_cpotrf_large(float2 *A, int lda, int upper, int n, int *info, void *scratch, cudaStream_t stream)
{
    float2 *W = static_cast<float2 *>(scratch);
    const size_t herk_smem = sizeof(HerkShared);
    cudaError_t e = cudaFuncSetAttribute(cherk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)herk_smem);
    if (e == cudaSuccess) e = cudaMemsetAsync(info, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    cbackup_kernel<<<elementwise_grid((int64_t)n * n), 256, 0, stream>>>(A, lda, upper, n, W);
    for (int k0 = 0; k0 < n && e == cudaSuccess; k0 += CPB)
    {
        cdiag_kernel<<<1, 256, 0, stream>>>(A, lda, upper, k0, n, info);
        const int rows = n - k0 - CPB;
        if (rows > 0)
        {
            crows_kernel<<<(unsigned)((rows + CROWS_T - 1) / CROWS_T), CROWS_T, 0, stream>>>(A, lda, upper, k0, n,
                                                                                             info);
            const int tiles = (rows + CPB - 1) / CPB;
            cherk_kernel<<<(unsigned)(tiles * (tiles + 1) / 2), 256, herk_smem, stream>>>(A, lda, upper, k0, n, info);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        crestore_kernel<<<elementwise_grid((int64_t)n * n), 256, 0, stream>>>(A, lda, upper, n, W, info);
    return cudaGetLastError();
}

}  // namespace ops_solver
