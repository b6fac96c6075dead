// lu_solve.cu -- LU solve P A X = B for orders above the register-resident kernels
// (64 < n <= 8192), one 256-thread block per (matrix, group of up to 8 right-hand sides).
//
// Order (the oracle's orc_sgetrs, trans 0): row interchanges applied in sequence, then the
// unit-lower forward sweep x_i = fma(-l_ik, x_k, x_i) in ascending k, then the upper sweep
// x_k = x_k / u_kk, x_i = fma(-u_ik, x_k, x_i) in descending k.  Blocking keeps every
// element's sequence: columns go in blocks of 32 (the last one ragged); the 32 x 32 diagonal
// triangle is solved by one warp per right-hand side with shuffles, then every other row
// takes its block's 32 updates in order.
//
// The solution vectors stay in shared memory.  The factor is streamed from global memory
// once: thread t owns one row of each 256-row strip and keeps that row's 32 entries of the
// block column in registers, so a warp's loads are 128-byte coalesced column segments.  The
// strips form one software pipeline over the whole sweep: the registers for the next strip
// (or the next block's diagonal triangle) are loaded while the current one is applied.
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int ST = 256;  // threads per block
constexpr int KB = 32;   // column block
constexpr int MAX_RHS_PER_BLOCK = 8;

// One unit of the sweep: the diagonal triangle of block `blk` (strip < 0) or a strip of up
// to 256 rows off the diagonal block (below it going forward, above it going backward).
struct Task
{
    int blk;
    int strip;
};

template <bool FORWARD>
__device__ __forceinline__ int task_row(int n, Task task)
{
    const int t = threadIdx.x, lane = t & 31;
    const int kb = task.blk * KB;
    const int w = min(KB, n - kb);
    if (task.strip < 0) return (t < 32 && lane < w) ? kb + lane : -1;
    const int r = task.strip * ST + t;
    if (FORWARD) return kb + w + r < n ? kb + w + r : -1;
    return r < kb ? r : -1;
}

// Thread t's registers for a task: the entries of its row in the block column.
template <bool FORWARD>
__device__ __forceinline__ void load_task(const float *A, int lda, int n, Task task, float (&v)[KB])
{
    const int kb = task.blk * KB;
    const int w = min(KB, n - kb);
    const int row = task_row<FORWARD>(n, task);
#pragma unroll
    for (int k = 0; k < KB; ++k) v[k] = (row >= 0 && k < w) ? A[(int64_t)(kb + k) * lda + row] : 0.0f;
}

template <bool FORWARD>
__device__ __forceinline__ int strips(int n, int blk)
{
    const int kb = blk * KB;
    const int w = min(KB, n - kb);
    const int rows = FORWARD ? n - kb - w : kb;
    return (rows + ST - 1) / ST;
}

// Advances to the next task of the sweep; false past the end.
template <bool FORWARD>
__device__ __forceinline__ bool next_task(int n, int nblk, Task &task)
{
    if (task.strip + 1 < strips<FORWARD>(n, task.blk))
    {
        ++task.strip;
        return true;
    }
    task.blk += FORWARD ? 1 : -1;
    task.strip = -1;
    return FORWARD ? task.blk < nblk : task.blk >= 0;
}

// Thread t < 32 (warp 0) holds row kb + t of a diagonal triangle: publish it.
__device__ __forceinline__ void store_triangle(float (*tri)[KB + 1], const float (&v)[KB])
{
    if (threadIdx.x < 32)
    {
#pragma unroll
        for (int k = 0; k < KB; ++k) tri[k][threadIdx.x] = v[k];
    }
}

template <bool FORWARD>
__device__ void sweep(const float *A, int lda, int n, float *x, int nr, float (*tri)[KB][KB + 1])
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nblk = (n + KB - 1) / KB;
    Task cur{FORWARD ? 0 : nblk - 1, -1};
    float v[KB], nv[KB];
    load_task<FORWARD>(A, lda, n, cur, v);
    store_triangle(tri[cur.blk & 1], v);
    __syncthreads();
    bool more = true;
    while (more)
    {
        Task nxt = cur;
        more = next_task<FORWARD>(n, nblk, nxt);
        if (more) load_task<FORWARD>(A, lda, n, nxt, nv);
        const int kb = cur.blk * KB;
        const int w = min(KB, n - kb);
        if (cur.strip < 0)
        {
            // diagonal triangle (published in shared memory): warp r solves right-hand side
            // r, lane i on row kb + i
            if (warp < nr)
            {
                const float(*d)[KB + 1] = tri[cur.blk & 1];
                float *xr = x + (size_t)warp * n;
                float xv = lane < w ? xr[kb + lane] : 0.0f;
                if (FORWARD)
                {
#pragma unroll
                    for (int k = 0; k < KB; ++k)
                    {
                        const float xk = __shfl_sync(0xffffffffu, xv, k);
                        if (lane > k && lane < w) xv = fma_rn(-d[k][lane], xk, xv);
                    }
                }
                else
                {
#pragma unroll
                    for (int k = KB - 1; k >= 0; --k)
                    {
                        if (k < w)
                        {
                            if (lane == k) xv = div_rn(xv, d[k][lane]);
                            const float xk = __shfl_sync(0xffffffffu, xv, k);
                            if (lane < k) xv = fma_rn(-d[k][lane], xk, xv);
                        }
                    }
                }
                if (lane < w) xr[kb + lane] = xv;
            }
        }
        else
        {
            const int row = task_row<FORWARD>(n, cur);
            if (row >= 0)
            {
                for (int q = 0; q < nr; ++q)
                {
                    float *xr = x + (size_t)q * n;
                    float acc = xr[row];
                    if (FORWARD)
                    {
#pragma unroll
                        for (int k = 0; k < KB; ++k)
                            if (k < w) acc = fma_rn(-v[k], xr[kb + k], acc);
                    }
                    else
                    {
#pragma unroll
                        for (int k = KB - 1; k >= 0; --k)
                            if (k < w) acc = fma_rn(-v[k], xr[kb + k], acc);
                    }
                    xr[row] = acc;
                }
            }
        }
        // the next diagonal triangle goes to the other buffer (the current one may be in use)
        if (more && nxt.strip < 0) store_triangle(tri[nxt.blk & 1], nv);
        // a diagonal solve feeds its strips, and a block's strips feed the next diagonal
        __syncthreads();
#pragma unroll
        for (int k = 0; k < KB; ++k) v[k] = nv[k];
        cur = nxt;
    }
}

__global__ void __launch_bounds__(ST, 2) getrs_blocked_kernel(float *a_single, float *const *a_table, int a_first,
                                                            const int *ipiv, const int *perm, float *b_single,
                                                            float *const *b_table, int b_first, int n, int lda,
                                                            int ldb, int nrhs, int count, int RHS, int *info,
                                                            const int *skip)
{
    extern __shared__ float x[];  // RHS x n
    __shared__ float tri[2][KB][KB + 1];
    __shared__ int bad;
    const int groups = (nrhs + RHS - 1) / RHS;
    const int t = threadIdx.x;
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
        const int *sig = perm ? perm + q * n : nullptr;
        if (!A || !B)
        {
            if (t == 0 && info && r0 == 0) info[q] = !A ? -4 : -7;
            continue;
        }
        if (t == 0) bad = 0;
        __syncthreads();
        if (piv && !sig)
            for (int k = t; k < n; k += ST)
                if (piv[k] < k + 1 || piv[k] > n) bad = 1;
        for (int e = t; e < nr * n; e += ST)
        {
            const int r = e / n, i = e % n;
            // with a permutation, x = P b directly: row i of the permuted vector is b[perm[i]]
            x[e] = B[(int64_t)(r0 + r) * ldb + (sig ? sig[i] : i)];
        }
        __syncthreads();
        if (bad)
        {
            if (t == 0 && info && r0 == 0) info[q] = -6;
            __syncthreads();
            continue;
        }
        // interchanges, in order: one thread per right-hand side
        if (piv && !sig && t < nr)
        {
            float *xr = x + (size_t)t * n;
            for (int k = 0; k < n; ++k)
            {
                const int p = piv[k] - 1;
                if (p != k)
                {
                    const float a = xr[k];
                    xr[k] = xr[p];
                    xr[p] = a;
                }
            }
        }
        __syncthreads();
        sweep<true>(A, lda, n, x, nr, tri);
        sweep<false>(A, lda, n, x, nr, tri);
        for (int e = t; e < nr * n; e += ST)
        {
            const int r = e / n, i = e % n;
            B[(int64_t)(r0 + r) * ldb + i] = x[e];
        }
        if (t == 0 && info && r0 == 0) info[q] = 0;
        __syncthreads();
    }
}

// perm = the interchanges of ipiv applied in order to the identity: P b = b[perm].  One
// thread per matrix; out-of-range pivots are skipped (callers validate them).
__global__ void permutation_kernel(const int *ipiv, int *perm, int n, int count)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
    {
        int *p = perm + q * n;
        const int *v = ipiv + q * n;
        for (int i = 0; i < n; ++i) p[i] = i;
        for (int k = 0; k < n; ++k)
        {
            const int s = v[k] - 1;
            if (s != k && s >= 0 && s < n)
            {
                const int a = p[k];
                p[k] = p[s];
                p[s] = a;
            }
        }
    }
}
}  // namespace

cudaError_t launch_getrs_blocked(const RealBatch &a, const int *ipiv, const int *perm, const RealBatch &b, int nrhs,
                                 int *info, const int *skip, cudaStream_t stream)
{
    const size_t budget = 100 * 1024 / sizeof(float);  // two blocks per SM
    int rpb = (int)(budget / (size_t)a.n);
    if (rpb > MAX_RHS_PER_BLOCK) rpb = MAX_RHS_PER_BLOCK;
    if (rpb > nrhs) rpb = nrhs;
    if (rpb < 1) return cudaErrorInvalidValue;
    const size_t smem = (size_t)rpb * a.n * sizeof(float);
    cudaFuncSetAttribute(getrs_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int groups = (nrhs + rpb - 1) / rpb;
    int64_t jobs = (int64_t)a.count * groups;
    int64_t blocks = jobs < 148 * 8 ? jobs : 148 * 8;
    if (blocks < 1) blocks = 1;
    getrs_blocked_kernel<<<(unsigned)blocks, ST, smem, stream>>>(a.single, a.table, a.first, ipiv, perm, b.single,
                                                                 b.table, b.first, a.n, a.ld, b.ld, nrhs, a.count,
                                                                 rpb, info, skip);
    return cudaGetLastError();
}

cudaError_t launch_permutation(const int *ipiv, int *perm, int n, int count, cudaStream_t stream)
{
    int blocks = (count + 127) / 128;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (blocks < 1) blocks = 1;
    permutation_kernel<<<blocks, 128, 0, stream>>>(ipiv, perm, n, count);
    return cudaGetLastError();
}

}  // namespace ops_solver
