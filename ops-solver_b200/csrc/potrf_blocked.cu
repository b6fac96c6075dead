// potrf_blocked.cu -- real Cholesky factorisation above order 32 (sm_100a).
//
// Arithmetic (this build's orders for n > 32, where the reference hands its updates to a
// CATLASS Gram product; restated in the oracle): up to order 256 (orc_spotrf_fma) every
// a_ij, j <= i, takes its updates a_ij = fma(-l_ik, l_jk, a_ij) in ascending k; above 256
// (orc_spotrf_blocked) the same inside each 64-column panel, while an element right of the
// panel takes the panel's products as one partial sum t = fma(l_ik, l_jk, t) from zero,
// then a_ij - t (a chain of n / 64 subtractions instead of n: the rounding of a blocked
// LAPACK, which the reference's residual gate asks for at orders in the thousands).  Then
// the pivot check (d > 0 and d <= FLT_MAX), the IEEE square root of the diagonal and the IEEE
// division of the column below it.  A failed matrix keeps its completed columns; the columns
// from the failed one on keep the caller's input.  The factors equal the oracle's bit for
// bit.
//
// 33 <= n <= 256, any batch: one block per matrix, the lower triangle packed by columns in
// shared memory (n = 256: 132 KB, one block per SM; n = 128: 33 KB), factored left-looking in
// blocks of 16 columns: every earlier column is first applied to block column J0 in shared
// memory, 16 / C threads per remaining row with C adjacent columns each (broadcast loads of
// the block's L(J0 + j, k)); then thread t takes row J0 + t into registers and the sixteen
// panel steps run with one barrier each, dividing only rows that exist; every thread keeps
// the block's diagonal so the square roots need no second exchange.  Untouched columns stay untouched,
// which keeps the failure contract for free.
//
// n > 256 (one matrix over the whole GPU, 64-column panels): the matrix is first copied to
// a backup; per panel
//   diag:  one block factors the 64 x 64 diagonal block in shared memory (right-looking);
//   rows:  a thread per row below it forms L21 = A21 L11^-T row by row (ascending k, IEEE
//          division by the diagonal), 128 rows per block;
//   syrk:  the trailing lower triangle takes A22 -= L21 L21^T over 64 x 64 tiles (lower tiles
//          only), each tile's two 64 x 64 operand panels loaded by TMA (a 2-D tensor map of
//          the matrix, completion on an mbarrier with a bounded wait) when the matrix is
//          16-byte aligned with lda % 4 == 0, by plain loads otherwise; FP32 FMAs in ascending
//          k into a 4 x 4 tile of partial sums per thread, subtracted once.
// Every kernel reads the info word first and stops once a pivot has failed; after the last
// panel a restore pass copies the backup back into the columns from the failed one on.
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "device_once.h"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr float FLT_MAX_VALUE = 3.402823466e38F;

// ---------------------------------------------------------------------------------------
// 33 <= n <= 256: packed triangle per block
// ---------------------------------------------------------------------------------------
constexpr int RB = 16;  // columns per block column

__host__ __device__ constexpr int rb_tri(int n) { return n * (n + 1) / 2; }
__host__ __device__ constexpr size_t rb_smem_bytes(int n) { return ((size_t)rb_tri(n) + RB + 2 * RB + RB) * sizeof(float); }
__device__ __forceinline__ int rb_col(int j, int n) { return j * n - (j * (j - 1)) / 2; }

__device__ __forceinline__ int64_t tri_at(int lda, int upper, int i, int j)
{
    return upper ? (int64_t)i * lda + j : (int64_t)j * lda + i;
}

// The left-looking update of block column J0 (rows J0..n-1, its w columns) by every earlier
// column k < J0, in shared memory: G = RB / C threads share a row, each taking C adjacent
// columns of it, so that the whole block works however few rows remain below J0.  Every
// element still takes its updates one after another in ascending k, from one thread.
template <int C>
__device__ __forceinline__ void rb_left(float *tri, int n, int J0, int w)
{
    constexpr int G = RB / C;
    const int t = threadIdx.x;
    const int i = J0 + t / G;    // row
    const int j0 = (t % G) * C;  // first column of this thread within the block
    if (i >= n) return;
    float z[C];
#pragma unroll
    for (int u = 0; u < C; ++u)
    {
        const int j = j0 + u;
        z[u] = (j < w && J0 + j <= i) ? tri[rb_col(J0 + j, n) + i - (J0 + j)] : 0.0f;
    }
    int ok = 0;  // packed offset of column k
    for (int k = 0; k < J0; ++k)
    {
        const float a = tri[ok + i - k];
        const float *c = tri + ok + J0 - k + j0;  // c[u] = L(J0 + j0 + u, k)
#pragma unroll
        for (int u = 0; u < C; ++u) z[u] = fma_rn(-a, c[u], z[u]);
        ok += n - k;
    }
#pragma unroll
    for (int u = 0; u < C; ++u)
    {
        const int j = j0 + u;
        if (j < w && J0 + j <= i) tri[rb_col(J0 + j, n) + i - (J0 + j)] = z[u];
    }
}

template <int T>
__global__ void __launch_bounds__(T) potrf_packed_kernel(float *single, float *const *table, int first, int n,
                                                         int lda, int upper, int count, int *info)
{
    extern __shared__ __align__(16) float rb_mem[];
    float *tri = rb_mem;                   // packed lower triangle (+ RB tail)
    float *xch = tri + rb_tri(n) + RB;     // [2][RB] column exchange
    float *dsh = xch + 2 * RB;            // [RB] block diagonal
    const int t = threadIdx.x;
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        float *p = table ? slot(table, first + q) : single;
        if (!p)
        {
            if (t == 0) info[q] = -3;
            continue;
        }
        // load: thread t takes row t of every column (rows j..n-1), eight loads in flight
        for (int j0 = 0; j0 < n; j0 += 8)
        {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                v[u] = (j0 + u <= t && t < n) ? p[tri_at(lda, upper, t, j0 + u)] : 0.0f;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (j0 + u <= t && t < n) tri[rb_col(j0 + u, n) + t - (j0 + u)] = v[u];
        }
        __syncthreads();
        int failure = 0;
        for (int J0 = 0; J0 < n && !failure; J0 += RB)
        {
            const int w = min(RB, n - J0);
            if (J0 > 0)
            {
                // threads per row: the most that fit the rows left (uniform over the block)
                const int rows = n - J0;
                if (rows > T / 2)
                    rb_left<16>(tri, n, J0, w);
                else if (rows > T / 4)
                    rb_left<8>(tri, n, J0, w);
                else if (rows > T / 8)
                    rb_left<4>(tri, n, J0, w);
                else if (rows > T / 16)
                    rb_left<2>(tri, n, J0, w);
                else
                    rb_left<1>(tri, n, J0, w);
                __syncthreads();
            }
            const int i = J0 + t;
            const bool own = i < n;
            float z[RB];
#pragma unroll
            for (int j = 0; j < RB; ++j)
                z[j] = (own && j < w && J0 + j <= i) ? tri[rb_col(J0 + j, n) + i - (J0 + j)] : 0.0f;
            if (t < w)
            {
                float dv = 0.0f;
#pragma unroll
                for (int j = 0; j < RB; ++j)
                    if (j == t) dv = z[j];
                dsh[t] = dv;
            }
            __syncthreads();
            float dg[RB];
#pragma unroll
            for (int j = 0; j < RB; ++j) dg[j] = j < w ? dsh[j] : 1.0f;
#pragma unroll
            for (int kk = 0; kk < RB; ++kk)
            {
                if (kk < w && failure == 0)
                {
                    const int k = J0 + kk;
                    const float d = dg[kk];
                    if (!(d > 0.0f && d <= FLT_MAX_VALUE))
                        failure = k + 1;
                    else
                    {
                        const float sq = sqrt_rn(d);
                        const float y = div_prepare(sq);
                        const bool okd = div_range(sq);
                        float l = z[kk];
                        if (i == k)
                            l = sq;
                        else if (i > k && own)  // rows past n would take the slow division on zeros
                            l = div_by(l, sq, y, okd);
                        z[kk] = l;
                        float *sl = xch + (kk & 1) * RB;
                        if (t < w) sl[t] = l;
                        __syncthreads();
#pragma unroll
                        for (int j = kk + 1; j < RB; ++j)
                        {
                            if (j < w)
                            {
                                const float c = sl[j];
                                if (own && i >= J0 + j) z[j] = fma_rn(-l, c, z[j]);
                                dg[j] = fma_rn(-c, c, dg[j]);
                            }
                        }
                    }
                }
            }
            const int wdone = failure ? failure - 1 - J0 : w;
            if (own)
            {
#pragma unroll
                for (int j = 0; j < RB; ++j)
                    if (j < wdone && J0 + j <= i) tri[rb_col(J0 + j, n) + i - (J0 + j)] = z[j];
            }
            __syncthreads();
        }
        // store the completed columns
        const int done = failure ? failure - 1 : n;
        if (t < n)
            for (int j = 0; j < done && j <= t; ++j) p[tri_at(lda, upper, t, j)] = tri[rb_col(j, n) + t - j];
        if (t == 0) info[q] = failure;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// n > 256: right-looking 32-column panels over the whole GPU
// ---------------------------------------------------------------------------------------
constexpr int PB = 64;        // panel width
constexpr int ST = 64;        // syrk tile (rows and columns)
constexpr int ROWS_T = 128;   // panel rows per block
constexpr long long WAIT_LIMIT = 1ll << 20;  // mbarrier try_wait rounds before giving up

// info > 0: a pivot failed (the whole factorisation stops); LARGE_WAIT_ERROR: a bounded
// wait ran out.  Kernels read it first and return when it is set.
__device__ __forceinline__ int stopped(const int *info) { return *(volatile const int *)info; }

// The 64 x 64 diagonal block at k0, right-looking in shared memory.
__global__ void __launch_bounds__(256) potrf_diag_kernel(float *A, int lda, int upper, int k0, int n, int *info)
{
    __shared__ float D[PB][PB + 1];  // D[j][i] = element (k0 + i, k0 + j), i >= j
    __shared__ int fail;
    if (stopped(info) != 0) return;
    const int t = threadIdx.x;
    const int w = min(PB, n - k0);
    for (int e = t; e < PB * PB; e += 256)
    {
        const int j = e / PB, i = e % PB;
        D[j][i] = (i < w && j < w && i >= j) ? A[tri_at(lda, upper, k0 + i, k0 + j)] : 0.0f;
    }
    if (t == 0) fail = 0;
    __syncthreads();
    for (int k = 0; k < w; ++k)
    {
        const float d = D[k][k];
        if (!(d > 0.0f && d <= FLT_MAX_VALUE))
        {
            if (t == 0) fail = k0 + k + 1;
            break;  // uniform
        }
        const float sq = sqrt_rn(d);
        const float y = div_prepare(sq);
        const bool ok = div_range(sq);
        __syncthreads();  // every thread has read d
        if (t > k && t < w) D[k][t] = div_by(D[k][t], sq, y, ok);
        if (t == k) D[k][k] = sq;
        __syncthreads();
        // a thread per (row, column) of the remaining block
        for (int e = t; e < PB * PB; e += 256)
        {
            const int j = e / PB, i = e % PB;
            if (j > k && i >= j && i < w) D[j][i] = fma_rn(-D[k][i], D[k][j], D[j][i]);
        }
        __syncthreads();
    }
    __syncthreads();
    const int done = fail ? fail - 1 - k0 : w;
    for (int e = t; e < PB * PB; e += 256)
    {
        const int j = e / PB, i = e % PB;
        if (j < done && i >= j && i < w) A[tri_at(lda, upper, k0 + i, k0 + j)] = D[j][i];
    }
    if (t == 0 && fail) *info = fail;
}

// L21 of the panel: rows k0 + 32 .. n - 1, a thread per row.  After a failure inside this
// panel (info names a column of it) the completed columns are still formed.
__global__ void __launch_bounds__(ROWS_T) potrf_rows_kernel(float *A, int lda, int upper, int k0, int n, int *info)
{
    __shared__ float L11[PB][PB + 1];  // L11[j][k] = element (k0 + j, k0 + k)
    const int st = stopped(info);
    int cols = PB;
    if (st != 0)
    {
        if (st < 0 || st - 1 < k0 || st - 1 >= k0 + PB) return;  // stopped before this panel, or an error
        cols = st - 1 - k0;  // the completed columns of this panel
        if (cols == 0) return;
    }
    const int t = threadIdx.x;
    for (int e = t; e < PB * PB; e += ROWS_T)
    {
        const int j = e / PB, k = e % PB;
        L11[j][k] = (k <= j && k0 + j < n) ? A[tri_at(lda, upper, k0 + j, k0 + k)] : 1.0f;
    }
    __syncthreads();
    const int i = k0 + PB + blockIdx.x * ROWS_T + t;
    if (i >= n) return;
    float z[PB];
#pragma unroll
    for (int j = 0; j < PB; ++j) z[j] = j < cols ? A[tri_at(lda, upper, i, k0 + j)] : 0.0f;
#pragma unroll
    for (int j = 0; j < PB; ++j)
    {
        if (j < cols)
        {
#pragma unroll
            for (int k = 0; k < j; ++k) z[j] = fma_rn(-z[k], L11[j][k], z[j]);
            const float d = L11[j][j];
            z[j] = div_by(z[j], d, div_prepare(d), div_range(d));
        }
    }
#pragma unroll
    for (int j = 0; j < PB; ++j)
        if (j < cols) A[tri_at(lda, upper, i, k0 + j)] = z[j];
}

// mbarrier and TMA helpers (this GPU's own memory only; no cluster multicast)
__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity)
{
    for (long long it = 0; it < WAIT_LIMIT; ++it)
    {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// 2-D tiled TMA load: box (rows x columns) at (row, column) of the tensor map into dst.
// The row coordinate is a multiple of 4 (16 bytes of float) by construction.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int row, int col, unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(saddr(dst)), "l"(map), "r"(row), "r"(col), "r"(bar)
        : "memory");
}

struct __align__(128) SyrkShared
{
    float a[PB][ST];  // a[k][r] = element (r0 + r, k0 + k): the tile's rows of L21
    float b[PB][ST];  // b[k][c] = element (c0 + c, k0 + k): the tile's columns as rows of L21
    unsigned long long bar;
};

// The lower tiles of the trailing matrix, tile index -> (tile row ti >= tile column tj).
__device__ __forceinline__ void lower_tile(int idx, int &ti, int &tj)
{
    int r = (int)((sqrtf(8.0f * idx + 1.0f) - 1.0f) * 0.5f);
    while ((r + 1) * (r + 2) / 2 <= idx) ++r;
    while (r * (r + 1) / 2 > idx) --r;
    ti = r;
    tj = idx - r * (r + 1) / 2;
}

// A22 -= L21 L21^T on the lower tiles: per element the panel's 64 products as one partial sum
// t = fma(l_ik, l_jk, t) from zero in ascending k, then a_ij - t.  tma: the operand panels
// come by TMA through `map` (lower storage, aligned); else by plain loads.
__global__ void __launch_bounds__(256) potrf_syrk_kernel(const __grid_constant__ CUtensorMap map, bool tma, float *A,
                                                         int lda, int upper, int k0, int n, int *info)
{
    __shared__ SyrkShared sh;
    if (stopped(info) != 0) return;
    const int t = threadIdx.x;
    const int base = k0 + PB;  // first trailing row / column
    int ti, tj;
    lower_tile(blockIdx.x, ti, tj);
    const int r0 = base + ti * ST, c0 = base + tj * ST;
    if (tma)
    {
        const unsigned bar = saddr(&sh.bar);
        if (t == 0)
        {
            mbar_init(bar, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            mbar_expect(bar, 2 * PB * ST * sizeof(float));
            tma_load_2d(&sh.a[0][0], &map, r0, k0, bar);
            tma_load_2d(&sh.b[0][0], &map, c0, k0, bar);
        }
        __syncthreads();
        if (!mbar_wait(bar, 0))
        {
            if (t == 0) atomicCAS(info, 0, LARGE_WAIT_ERROR);
            return;  // the tile is not updated; the error is reported in info
        }
    }
    else
    {
        for (int e = t; e < PB * ST; e += 256)
        {
            const int k = e / ST, r = e % ST;
            sh.a[k][r] = r0 + r < n ? A[tri_at(lda, upper, r0 + r, k0 + k)] : 0.0f;
            sh.b[k][r] = c0 + r < n ? A[tri_at(lda, upper, c0 + r, k0 + k)] : 0.0f;
        }
        __syncthreads();
    }
    // thread (tr, tc): rows r0 + 4 tr .. +3, columns c0 + 4 tc .. +3
    const int tr = t & 15, tc = t >> 4;
    const int i0 = r0 + 4 * tr;
    // a thread's four rows in one 16-byte piece per column when the matrix is aligned (rows
    // start at multiples of 4) and the piece lies wholly below the diagonal and inside n
    const bool vec = tma && i0 + 3 < n && c0 + 4 * tc + 3 <= i0;
    float c[4][4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
    {
        const int j = c0 + 4 * tc + v;
        if (vec)
        {
            const float4 x = *reinterpret_cast<const float4 *>(A + (int64_t)j * lda + i0);
            c[0][v] = x.x;
            c[1][v] = x.y;
            c[2][v] = x.z;
            c[3][v] = x.w;
        }
        else
        {
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
                const int i = i0 + u;
                c[u][v] = (i < n && j <= i) ? A[tri_at(lda, upper, i, j)] : 0.0f;
            }
        }
    }
    // the panel's 64 products as one partial sum per element, then one subtraction
    float ps[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) ps[u][v] = 0.0f;
#pragma unroll 8
    for (int k = 0; k < PB; ++k)
    {
        const float4 av = *reinterpret_cast<const float4 *>(&sh.a[k][4 * tr]);
        const float4 bv = *reinterpret_cast<const float4 *>(&sh.b[k][4 * tc]);
        const float ar[4] = {av.x, av.y, av.z, av.w};
        const float bc[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) ps[u][v] = fma_rn(ar[u], bc[v], ps[u][v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) c[u][v] = sub_rn(c[u][v], ps[u][v]);
#pragma unroll
    for (int v = 0; v < 4; ++v)
    {
        const int j = c0 + 4 * tc + v;
        if (vec)
            *reinterpret_cast<float4 *>(A + (int64_t)j * lda + i0) = make_float4(c[0][v], c[1][v], c[2][v], c[3][v]);
        else
        {
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
                const int i = i0 + u;
                if (i < n && j <= i) A[tri_at(lda, upper, i, j)] = c[u][v];
            }
        }
    }
}

// Backup copy of the lower triangle (element (i, j) at W[j * n + i]) and its restore of the
// columns from the failed one on.
__global__ void potrf_backup_kernel(const float *A, int lda, int upper, int n, float *W)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        if (i >= j) W[e] = A[tri_at(lda, upper, i, j)];
    }
}
__global__ void potrf_restore_kernel(float *A, int lda, int upper, int n, const float *W, const int *info)
{
    const int f = *info;
    if (f <= 0) return;
    const int from = f - 1;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        if (j >= from && i >= j) A[tri_at(lda, upper, i, j)] = W[e];
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []
    {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
    });
    return fn;
}

// The tensor map of a lower-stored n x n matrix: dimension 0 the rows (contiguous), 1 the
// columns (stride lda floats), box 64 rows x 32 columns, zero fill past n.
bool make_map(CUtensorMap *map, const float *A, int lda, int n)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || (reinterpret_cast<uintptr_t>(A) & 15u) != 0 || (lda & 3) != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)lda * sizeof(float)};
    const cuuint32_t box[2] = {ST, PB};
    const cuuint32_t estride[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(A), dims, strides, box, estride,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

unsigned grid_of(int64_t elements)
{
    int64_t b = (elements + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return (unsigned)(b < 1 ? 1 : b);
}
}  // namespace

size_t potrf_packed_smem(int n) { return rb_smem_bytes(n); }

cudaError_t launch_potrf_packed(const RealBatch &a, int upper, int *info, cudaStream_t stream)
{
    if (a.n > POTRF_PACKED_MAX) return cudaErrorInvalidValue;
    const size_t smem = rb_smem_bytes(a.n);
    int64_t blocks = a.count;
    if (a.n <= 128)
    {
        cudaError_t e = cudaFuncSetAttribute(potrf_packed_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        if (blocks > 148 * 16) blocks = 148 * 16;
        potrf_packed_kernel<128><<<(unsigned)blocks, 128, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld,
                                                                          upper, a.count, info);
    }
    else
    {
        cudaError_t e = cudaFuncSetAttribute(potrf_packed_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        if (blocks > 148 * 8) blocks = 148 * 8;
        potrf_packed_kernel<256><<<(unsigned)blocks, 256, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld,
                                                                          upper, a.count, info);
    }
    return cudaGetLastError();
}

size_t potrf_large_scratch_bytes(int n) { return (size_t)n * n * sizeof(float); }

cudaError_t launch_potrf_large(float *A, int lda, int upper, int n, int *info, void *scratch, cudaStream_t stream)
{
    float *W = static_cast<float *>(scratch);
    CUtensorMap map;
    const bool tma = !upper && make_map(&map, A, lda, n);
    if (!tma) memset(&map, 0, sizeof(map));
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    potrf_backup_kernel<<<grid_of((int64_t)n * n), 256, 0, stream>>>(A, lda, upper, n, W);
    for (int k0 = 0; k0 < n && e == cudaSuccess; k0 += PB)
    {
        potrf_diag_kernel<<<1, 256, 0, stream>>>(A, lda, upper, k0, n, info);
        const int rows = n - k0 - PB;
        if (rows > 0)
        {
            potrf_rows_kernel<<<(unsigned)((rows + ROWS_T - 1) / ROWS_T), ROWS_T, 0, stream>>>(A, lda, upper, k0, n,
                                                                                             info);
            const int tiles = (rows + ST - 1) / ST;
            potrf_syrk_kernel<<<(unsigned)(tiles * (tiles + 1) / 2), 256, 0, stream>>>(map, tma, A, lda, upper, k0,
                                                                                        n, info);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) potrf_restore_kernel<<<grid_of((int64_t)n * n), 256, 0, stream>>>(A, lda, upper, n, W, info);
    return cudaGetLastError();
}

}  // namespace ops_solver
