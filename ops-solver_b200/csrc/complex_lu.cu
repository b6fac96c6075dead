// complex_lu.cu -- the complex64 LU family: factor (Cgetrf), solve (Cgetrs), inverse from
// an LU (Cgetri, CgetriBatched) and the direct batched inverse (CmatinvBatched).
//
// Arithmetic (complex_lu.cuh) restates the reference's SIMT helpers; the schedules are this
// build's own.  Every element of an LU receives its SubMul updates one pivot at a time in
// ascending pivot order (the reference's FactorColumn / UpdatePanel / BlockUpdateVf order,
// src/utils/complex_solver_kernel.hpp:161-250, complex_solver_update.hpp:60-82), so the
// factor is the same bits whether it runs in one block's shared memory or blocked over
// the whole GPU:
//   cgetrf_panel_kernel   one block factors a whole small matrix in shared memory: pivot search
//                         (PivotScore, earliest row on ties), row swap, Divide of the column
//                         below the diagonal, rank-1 SubMul update of the panel's columns
//   cgetrf_row_panel_kernel  a 32-column panel of a larger matrix, one row per thread over a
//                         thread-block cluster of up to 8 blocks (distributed shared memory
//                         for the pivot candidates and rows, cluster barriers)
//   claswp_kernel         a whole interchange sequence on a solve's right-hand sides
//   claswp_panel_kernel   a panel's interchanges applied to the columns outside it as one
//                         composed row move per (column, row)
//   ctrsm_block_kernel    a <= 32-row block of a triangular solve, one warp per column,
//                         the diagonal tile in shared memory (unit or Divide diagonal)
//   cchain_update_kernel  C -= A B over k <= 32 as a per-element SubMul chain in pivot
//                         order (ascending, or descending for backward solves), 64 x 64 tiles
// The inverse from an LU restates WarpResidentSolve (src/utils/complex_solver_resident.hpp:
// 45-170): column j solves L U x = P e_j with compensated updates; n <= 256 keeps each
// column's state in a warp's registers (cgetri_resident_kernel), larger orders keep it in
// two planes and sweep 64-row blocks (cinv_block_kernel + cinv_update_kernel), same order.
// The direct inverse restates InvertSmallInPlace (src/utils/complex_solver_register.hpp:
// 271-326): Gauss-Jordan with one lane per column, the matrix in registers.
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>

#include "complex_lu.cuh"
#include "device_once.h"
#include "launch_complex.h"

namespace ops_solver
{
using namespace clu;

namespace
{
constexpr int PANEL = 32;               // columns per factor panel and per update step
constexpr int PANEL_THREADS = 1024;     // one block factors a panel
constexpr int CAPACITY = 24 * 1024;     // complex elements of a panel held in shared memory
constexpr int TRSM_THREADS = 256;  // 8 columns per block, one warp each
constexpr int UPD_TILE = 64;
constexpr int INV_BLOCK = 64;           // rows per compensated block step (order > 256)
constexpr int INV_TILE_COLS = 32;

// ---------------------------------------------------------------------------------------
// Factor a panel in shared memory: rows [c0, m) x columns [c0, c_end) of A, pivot columns
// [c0, c1).  The interchanges are applied inside the panel only; ipiv entries are global
// 1-based rows.  info keeps the first zero pivot (written by thread 0, in column order).
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(PANEL_THREADS) cgetrf_panel_kernel(float2 *A, int lda, int m, int c0, int c1,
                                                                     int c_end, int *ipiv, int *info)
{
    extern __shared__ float2 sp[];
    __shared__ uint32_t red_score[PANEL_THREADS / 32];
    __shared__ int red_row[PANEL_THREADS / 32];
    const int H = m - c0, W = c_end - c0, tid = threadIdx.x, T = blockDim.x;
    int info_now = tid == 0 ? *info : 0;  // read once: this kernel alone writes it meanwhile
    for (int idx = tid; idx < H * W; idx += T)
    {
        int r = idx % H, j = idx / H;
        sp[idx] = A[(int64_t)(c0 + j) * lda + c0 + r];
    }
    __syncthreads();
    for (int lc = 0; lc < c1 - c0; ++lc)
    {
        float2 *col = sp + (int64_t)lc * H;
        int p = lc;
        if (ipiv)
        {
            uint32_t best = 0;
            int row = H;
            for (int r = lc + tid; r < H; r += T)
            {
                uint32_t s = cscore(col[r]);
                if (s > best || (s == best && r < row))
                {
                    best = s;
                    row = r;
                }
            }
            for (int off = 16; off > 0; off >>= 1)
            {
                uint32_t os = __shfl_down_sync(0xffffffffu, best, off);
                int orow = __shfl_down_sync(0xffffffffu, row, off);
                if (os > best || (os == best && orow < row))
                {
                    best = os;
                    row = orow;
                }
            }
            if ((tid & 31) == 0)
            {
                red_score[tid >> 5] = best;
                red_row[tid >> 5] = row;
            }
            __syncthreads();
            if (tid < 32)
            {
                best = tid < (T >> 5) ? red_score[tid] : 0u;
                row = tid < (T >> 5) ? red_row[tid] : H;
                for (int off = 16; off > 0; off >>= 1)
                {
                    uint32_t os = __shfl_down_sync(0xffffffffu, best, off);
                    int orow = __shfl_down_sync(0xffffffffu, row, off);
                    if (os > best || (os == best && orow < row))
                    {
                        best = os;
                        row = orow;
                    }
                }
                if (tid == 0) red_row[0] = row;
            }
            __syncthreads();
            p = red_row[0];
        }
        if (tid == 0 && ipiv) ipiv[c0 + lc] = c0 + p + 1;
        if (p != lc)
            for (int j = tid; j < W; j += T)
            {
                float2 *cj = sp + (int64_t)j * H;
                float2 t = cj[lc];
                cj[lc] = cj[p];
                cj[p] = t;
            }
        __syncthreads();
        const float2 d = col[lc];
        if (tid == 0 && info_now == 0 && czero(d))
        {
            info_now = c0 + lc + 1;
            *info = info_now;
        }
        if (!czero(d))
        {
            const Divisor dv = cprepare(d);
            for (int r = lc + 1 + tid; r < H; r += T) col[r] = cdivide(col[r], dv);
        }
        __syncthreads();
        const int rows = H - lc - 1, cols = W - lc - 1;
        if (rows > 0 && cols > 0)
        {
            const int total = rows * cols;
            for (int idx = tid; idx < total; idx += T)
            {
                int r = lc + 1 + idx % rows, j = lc + 1 + idx / rows;
                float2 *cj = sp + (int64_t)j * H;
                cj[r] = csubmul(cj[r], col[r], cj[lc]);
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < H * W; idx += T)
    {
        int r = idx % H, j = idx / H;
        A[(int64_t)(c0 + j) * lda + c0 + r] = sp[idx];
    }
}

// Row-per-thread panel: rows [c0, m) x columns [c0, c0 + w) (w <= 32), each thread of a
// cluster of `cl` blocks owning one panel row (block r: panel rows [rR, rR + R), R <= ROW_MAX,
// so the diagonal rows live in block 0), kept in the thread's own shared-memory row (pitch 33:
// a warp's rows fall in distinct banks).  Per column: each block's pivot candidate (warp
// shuffles, one barrier) published with its row, block 0 also publishing row lc; one cluster
// barrier; every block reads all candidates and the winner's row through distributed shared
// memory, the two owners take each other's row, and every thread below the diagonal divides
// its l and updates its row.  The column loop
// stays rolled (an unrolled one overflows the instruction cache).  Same per-element
// arithmetic as the single-block kernel.
constexpr int ROW_MAX = 512;
constexpr int ROW_PITCH = PANEL + 1;

__global__ void __launch_bounds__(ROW_MAX, 1) cgetrf_row_panel_kernel(float2 *A, int lda, int m, int c0, int w,
                                                                      int R, int *ipiv, int *info)
{
    namespace cg = cooperative_groups;
    extern __shared__ float2 rows_sm[];  // blockDim.x rows x ROW_PITCH
    __shared__ uint32_t red_score[ROW_MAX / 32];
    __shared__ int red_row[ROW_MAX / 32];
    // published per column, double-buffered by column parity: a block rewrites a buffer only
    // after every block has passed the next column's cluster barrier, i.e. finished reading it
    __shared__ uint32_t cand_score[2];
    __shared__ int cand_row[2];
    __shared__ float2 pub[2][PANEL], kpub[2][PANEL], prow[PANEL];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank(), cl = (int)cluster.num_blocks();
    const int H = m - c0, r0 = rank * R, tid = threadIdx.x;
    const int g = r0 + tid;  // this thread's panel row
    const bool valid = tid < R && g < H;
    float2 *a = rows_sm + (int64_t)tid * ROW_PITCH;
    for (int j = 0; j < w; ++j) a[j] = valid ? A[(int64_t)(c0 + j) * lda + c0 + g] : make_float2(0.0f, 0.0f);
    int info_now = rank == 0 && tid == 0 ? *info : 0;  // read once: this kernel alone writes it meanwhile
#pragma unroll 1
    for (int lc = 0; lc < w; ++lc)
    {
        const int buf = lc & 1;
        uint32_t best = 0;
        int row = H;
        if (ipiv && valid && g >= lc)
        {
            best = cscore(a[lc]);
            row = g;
        }
        for (int off = 16; off > 0; off >>= 1)
        {
            uint32_t os = __shfl_down_sync(0xffffffffu, best, off);
            int orow = __shfl_down_sync(0xffffffffu, row, off);
            if (os > best || (os == best && orow < row))
            {
                best = os;
                row = orow;
            }
        }
        if ((tid & 31) == 0)
        {
            red_score[tid >> 5] = best;
            red_row[tid >> 5] = row;
        }
        __syncthreads();
        if (tid < 32)
        {
            // the block's candidate, then its row (and block 0's row lc) published by this warp
            const int warps = blockDim.x >> 5;
            best = tid < warps ? red_score[tid] : 0u;
            row = tid < warps ? red_row[tid] : H;
            for (int off = 16; off > 0; off >>= 1)
            {
                uint32_t os = __shfl_down_sync(0xffffffffu, best, off);
                int orow = __shfl_down_sync(0xffffffffu, row, off);
                if (os > best || (os == best && orow < row))
                {
                    best = os;
                    row = orow;
                }
            }
            best = __shfl_sync(0xffffffffu, best, 0);
            row = __shfl_sync(0xffffffffu, row, 0);
            if (tid == 0)
            {
                cand_score[buf] = best;
                cand_row[buf] = row;
            }
            if (tid < w)
            {
                if (row < H) pub[buf][tid] = rows_sm[(int64_t)(row - r0) * ROW_PITCH + tid];
                if (rank == 0) kpub[buf][tid] = rows_sm[(int64_t)lc * ROW_PITCH + tid];
            }
        }
        cluster.sync();
        if (tid < 32)
        {
            uint32_t b = 0;
            int p = H;
            if (tid < cl)
            {
                b = cluster.map_shared_rank(cand_score, tid)[buf];
                p = cluster.map_shared_rank(cand_row, tid)[buf];
            }
            for (int off = 16; off > 0; off >>= 1)
            {
                uint32_t os = __shfl_down_sync(0xffffffffu, b, off);
                int orow = __shfl_down_sync(0xffffffffu, p, off);
                if (os > b || (os == b && orow < p))
                {
                    b = os;
                    p = orow;
                }
            }
            p = ipiv ? __shfl_sync(0xffffffffu, p, 0) : lc;
            const int owner = p / R;
            if (tid < w)
            {
                // without pivoting the pivot row is row lc, which block 0 published as kpub
                const float2 v = ipiv ? cluster.map_shared_rank(&pub[0][0], owner)[buf * PANEL + tid]
                                      : cluster.map_shared_rank(&kpub[0][0], 0)[buf * PANEL + tid];
                prow[tid] = v;
                if (rank == owner && p != lc)
                    rows_sm[(int64_t)(p - r0) * ROW_PITCH + tid] = cluster.map_shared_rank(&kpub[0][0], 0)[buf * PANEL + tid];
                if (rank == 0) rows_sm[(int64_t)lc * ROW_PITCH + tid] = v;
            }
            __syncwarp();
            if (rank == 0 && tid == 0)
            {
                if (ipiv) ipiv[c0 + lc] = c0 + p + 1;
                if (info_now == 0 && czero(prow[lc]))
                {
                    info_now = c0 + lc + 1;
                    *info = info_now;
                }
            }
        }
        __syncthreads();
        if (valid && g > lc)
        {
            const float2 d = prow[lc];
            float2 l = a[lc];
            if (!czero(d)) l = cdivide(l, cprepare(d));
            a[lc] = l;
            for (int j = lc + 1; j < w; ++j) a[j] = csubmul(a[j], l, prow[j]);
        }
    }
    if (valid)
        for (int j = 0; j < w; ++j) A[(int64_t)(c0 + j) * lda + c0 + g] = a[j];
    cluster.sync();  // no block leaves while another may still read its shared memory
}

// Interchanges ipiv[k0..k1) (global 1-based rows), in order, on columns [0, ncols) of A
// except [skip0, skip1).  reverse applies them from k1-1 down to k0.
__global__ void claswp_kernel(float2 *A, int64_t lda, int ncols, int k0, int k1, const int *ipiv, int skip0,
                              int skip1, bool reverse)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ncols || (j >= skip0 && j < skip1)) return;
    float2 *c = A + (int64_t)j * lda;
    for (int s = 0; s < k1 - k0; ++s)
    {
        int k = reverse ? k1 - 1 - s : k0 + s;
        int p = __ldg(ipiv + k) - 1;
        if (p != k)
        {
            float2 t = c[k];
            c[k] = c[p];
            c[p] = t;
        }
    }
}

// One block of a triangular solve: rows [0, w) of X's columns [0, ncols) against the w x w
// diagonal tile T, one warp per column with lane i holding row i.  FWD: x_i -= T_ip x_p for
// p < i in ascending order; BWD: for p > i in descending order; a non-unit diagonal divides
// x_p (Divide) when its turn comes.
template <bool FWD, bool UNIT>
__global__ void __launch_bounds__(TRSM_THREADS) ctrsm_block_kernel(const float2 *T, int64_t ldt, float2 *X,
                                                                   int64_t ldx, int w, int ncols)
{
    __shared__ float2 tile[PANEL][PANEL + 1];
    __shared__ Divisor dv[PANEL];
    for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x)
    {
        int i = idx % w, p = idx / w;
        tile[p][i] = T[(int64_t)p * ldt + i];
    }
    __syncthreads();
    if (!UNIT)
    {
        if (threadIdx.x < w) dv[threadIdx.x] = cprepare(tile[threadIdx.x][threadIdx.x]);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.x * (TRSM_THREADS / 32) + (threadIdx.x >> 5);
    if (j >= ncols) return;
    float2 *xc = X + (int64_t)j * ldx;
    float2 x = lane < w ? xc[lane] : make_float2(0.0f, 0.0f);
    for (int t = 0; t < w; ++t)
    {
        const int p = FWD ? t : w - 1 - t;
        if (!UNIT && lane == p) x = cdivide(x, dv[p]);
        const float2 v = make_float2(__shfl_sync(0xffffffffu, x.x, p), __shfl_sync(0xffffffffu, x.y, p));
        if (FWD ? (lane > p && lane < w) : (lane < p)) x = csubmul(x, tile[p][lane], v);
    }
    if (lane < w) xc[lane] = x;
}

// The interchanges ipiv[k0..k0+w) (global 1-based rows, w <= 32) applied in order to columns
// [0, ncols) of A except [skip0, skip1).  Their composition moves at most 2w rows; thread 0
// derives it (row_of[i] receives the original row src_of[i]), then each thread moves one
// row of one column: every value is read before any is written.
__global__ void __launch_bounds__(256) claswp_panel_kernel(float2 *A, int64_t lda, int ncols, int k0, int w,
                                                           const int *ipiv, int skip0, int skip1)
{
    __shared__ int row_of[2 * PANEL], src_of[2 * PANEL], piv_sm[PANEL], count;
    if (threadIdx.x < w) piv_sm[threadIdx.x] = __ldg(ipiv + k0 + threadIdx.x) - 1;  // one parallel load
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int cnt = w;
        for (int i = 0; i < w; ++i) row_of[i] = src_of[i] = k0 + i;
        for (int k = 0; k < w; ++k)
        {
            const int p = piv_sm[k];
            int ip = -1;
            if (p >= k0 && p < k0 + w)
                ip = p - k0;
            else
            {
                for (int e = w; e < cnt; ++e)
                    if (row_of[e] == p) ip = e;
                if (ip < 0)
                {
                    ip = cnt++;
                    row_of[ip] = src_of[ip] = p;
                }
            }
            const int t = src_of[k];
            src_of[k] = src_of[ip];
            src_of[ip] = t;
        }
        count = cnt;
    }
    __syncthreads();
    const int j = blockIdx.x * 4 + (threadIdx.x >> 6), idx = threadIdx.x & 63;
    const bool act = j < ncols && (j < skip0 || j >= skip1) && idx < count && src_of[idx] != row_of[idx];
    float2 v = make_float2(0.0f, 0.0f);
    if (act) v = A[(int64_t)j * lda + src_of[idx]];
    __syncthreads();
    if (act) A[(int64_t)j * lda + row_of[idx]] = v;
}

// C[r][j] (r < rows, j < cols) -= sum over p < k of A[r][p] B[p][j] as a SubMul chain per
// element, p ascending (or descending when DESC).  k <= 32; 64 x 64 tiles, 256 threads,
// 4 x 4 elements per thread (rows tx + 16 i, columns ty + 16 jj).
template <bool DESC>
__global__ void __launch_bounds__(256) cchain_update_kernel(float2 *C, int64_t ldc, const float2 *A, int64_t lda,
                                                            const float2 *B, int64_t ldb, int rows, int cols, int k)
{
    __shared__ float2 As[PANEL][UPD_TILE];
    __shared__ float2 Bs[PANEL][UPD_TILE];
    const int r0 = blockIdx.x * UPD_TILE, c0 = blockIdx.y * UPD_TILE;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    for (int idx = tid; idx < k * UPD_TILE; idx += 256)
    {
        int r = idx % UPD_TILE, p = idx / UPD_TILE;
        As[p][r] = r0 + r < rows ? A[(int64_t)p * lda + r0 + r] : make_float2(0.0f, 0.0f);
    }
    for (int idx = tid; idx < k * UPD_TILE; idx += 256)
    {
        int p = idx % k, c = idx / k;
        Bs[p][c] = c0 + c < cols ? B[(int64_t)(c0 + c) * ldb + p] : make_float2(0.0f, 0.0f);
    }
    float2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
        {
            int r = r0 + tx + 16 * i, c = c0 + ty + 16 * jj;
            acc[i][jj] = r < rows && c < cols ? C[(int64_t)c * ldc + r] : make_float2(0.0f, 0.0f);
        }
    __syncthreads();
    for (int s = 0; s < k; ++s)
    {
        const int p = DESC ? k - 1 - s : s;
        float2 a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[p][tx + 16 * i];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) b[jj] = Bs[p][ty + 16 * jj];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) acc[i][jj] = csubmul(acc[i][jj], a[i], b[jj]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
        {
            int r = r0 + tx + 16 * i, c = c0 + ty + 16 * jj;
            if (r < rows && c < cols) C[(int64_t)c * ldc + r] = acc[i][jj];
        }
}

// ---------------------------------------------------------------------------------------
// Inverse from an LU
// ---------------------------------------------------------------------------------------

struct InvArgs
{
    const float2 *a_single;
    const float2 *const *a_table;
    float2 *c_single;
    float2 *const *c_table;
    int n, lda, ldc;
    int64_t a_stride, c_stride;  // complex elements between single-pointer matrices
    const int *ipiv;             // n per matrix, or null
    int *info;                   // one per matrix
    int count;
};

__device__ __forceinline__ const float2 *inv_input(const InvArgs &g, int q)
{
    return g.a_table ? slot(g.a_table, q) : g.a_single + (int64_t)q * g.a_stride;
}

__device__ __forceinline__ float2 *inv_output(const InvArgs &g, int q)
{
    return g.c_table ? slot(g.c_table, q) : g.c_single + (int64_t)q * g.c_stride;
}

// ParallelCheckLu (complex_solver_kernel.hpp:262-292): -4 for a pivot outside [row+1, n],
// else the first exactly-zero diagonal, 1-based, else 0.  Block-wide; all threads return it.
__device__ int check_lu_block(const float2 *a, int n, int lda, const int *piv, int *scratch)
{
    int result = 0x7fffffff;
    for (int r = threadIdx.x; r < n; r += blockDim.x)
    {
        if (piv && (piv[r] < r + 1 || piv[r] > n)) result = -4;
        if (czero(a[(int64_t)r * lda + r]) && result > r + 1) result = r + 1;
    }
    for (int off = 16; off > 0; off >>= 1) result = min(result, __shfl_down_sync(0xffffffffu, result, off));
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = result;
    __syncthreads();
    if (threadIdx.x < 32)
    {
        int v = threadIdx.x < (blockDim.x >> 5) ? scratch[threadIdx.x] : 0x7fffffff;
        for (int off = 16; off > 0; off >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, off));
        if (threadIdx.x == 0) scratch[32] = v == 0x7fffffff ? 0 : v;
    }
    __syncthreads();
    return scratch[32];
}

// Orders <= 256: one warp per inverse column with its rows in registers (SEG x 32), 8
// columns per block; the LU streams through shared memory 32 columns at a time (forward
// panels ascending, backward panels descending).  Block (q, g) handles matrix q, columns
// [8g, 8g + 8); every block of a matrix computes the same check and block 0 writes info.
template <int SEG>
__global__ void __launch_bounds__(256) cgetri_resident_kernel(InvArgs g, int groups)
{
    extern __shared__ float2 panel[];  // PANEL columns x n rows
    __shared__ int perm[256];
    __shared__ int scratch[33];
    const int q = blockIdx.x / groups, grp = blockIdx.x % groups;
    const int n = g.n, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float2 *a = inv_input(g, q);
    const int *piv = g.ipiv ? g.ipiv + (int64_t)q * n : nullptr;
    const int status = check_lu_block(a, n, g.lda, piv, scratch);
    if (grp == 0 && threadIdx.x == 0) g.info[q] = status;
    if (status != 0) return;
    if (threadIdx.x == 0)
    {
        for (int r = 0; r < n; ++r) perm[r] = r;
        if (piv)
            for (int r = 0; r < n; ++r)
            {
                int t = piv[r] - 1, v = perm[r];
                perm[r] = perm[t];
                perm[t] = v;
            }
    }
    __syncthreads();
    const int j = grp * 8 + warp;
    float2 x[SEG], e[SEG];
#pragma unroll
    for (int s = 0; s < SEG; ++s)
    {
        int r = s * 32 + lane;
        x[s] = make_float2(r < n && perm[r] == j ? 1.0f : 0.0f, 0.0f);
        e[s] = make_float2(0.0f, 0.0f);
    }
    const int npanels = (n + PANEL - 1) / PANEL;
    for (int pb = 0; pb < 2 * npanels; ++pb)
    {
        const bool fwd = pb < npanels;
        const int panel_id = fwd ? pb : 2 * npanels - 1 - pb;
        const int p0 = panel_id * PANEL, pw = min(PANEL, n - p0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < pw * n; idx += blockDim.x)
        {
            int r = idx % n, c = idx / n;
            panel[(int64_t)c * n + r] = a[(int64_t)(p0 + c) * g.lda + r];
        }
        __syncthreads();
        if (j >= n) continue;
        for (int t = 0; t < pw; ++t)
        {
            const int pl = fwd ? t : pw - 1 - t, p = p0 + pl;
            const float2 *pc = panel + (int64_t)pl * n;
            float2 v = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int s = 0; s < SEG; ++s)
                if (p / 32 == s) v = cadd(x[s], e[s]);
            if (!fwd && lane == (p & 31)) v = cdivide(v, pc[p]);
            v.x = __shfl_sync(0xffffffffu, v.x, p & 31);
            v.y = __shfl_sync(0xffffffffu, v.y, p & 31);
#pragma unroll
            for (int s = 0; s < SEG; ++s)
            {
                const int r = s * 32 + lane;
                if (!fwd && r == p)
                {
                    x[s] = v;
                    e[s] = make_float2(0.0f, 0.0f);
                }
                if (fwd ? (r > p && r < n) : (r < p)) ccomp_submul(x[s], e[s], pc[r], v);
            }
        }
    }
    if (j >= n) return;
    float2 *c = inv_output(g, q) + (int64_t)j * g.ldc;
#pragma unroll
    for (int s = 0; s < SEG; ++s)
    {
        int r = s * 32 + lane;
        if (r < n) c[r] = x[s];
    }
}

// Orders > 256: the state (x, e) of every inverse column lives in two n x n planes (ld n).
__global__ void cinv_check_kernel(InvArgs g, int q, int *perm)
{
    __shared__ int scratch[33];
    const float2 *a = inv_input(g, q);
    const int *piv = g.ipiv ? g.ipiv + (int64_t)q * g.n : nullptr;
    int status = check_lu_block(a, g.n, g.lda, piv, scratch);
    if (threadIdx.x == 0)
    {
        g.info[q] = status;
        for (int r = 0; r < g.n; ++r) perm[r] = r;
        if (status == 0 && piv)
            for (int r = 0; r < g.n; ++r)
            {
                int t = piv[r] - 1, v = perm[r];
                perm[r] = perm[t];
                perm[t] = v;
            }
    }
}

__global__ void cinv_init_kernel(float2 *X, float2 *E, int n, const int *perm, const int *info)
{
    if (*info != 0) return;
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * n) return;
    int r = (int)(idx % n), j = (int)(idx / n);
    X[idx] = make_float2(__ldg(perm + r) == j ? 1.0f : 0.0f, 0.0f);
    E[idx] = make_float2(0.0f, 0.0f);
}

// Diagonal block [b0, b0 + w) of the compensated sweep, one warp per column (2 rows per
// lane).  Forward: p ascending, v = x_p + e_p, rows below p updated.  Backward: p
// descending, v = Divide(x_p + e_p, U_pp), x_p = v, e_p = 0, rows above p updated.
template <bool FWD>
__global__ void __launch_bounds__(256) cinv_block_kernel(const float2 *a, int lda, float2 *X, float2 *E, int n,
                                                         int b0, int w, const int *info)
{
    if (*info != 0) return;
    __shared__ float2 tile[INV_BLOCK][INV_BLOCK + 1];
    for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x)
    {
        int i = idx % w, p = idx / w;
        tile[p][i] = a[(int64_t)(b0 + p) * lda + b0 + i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, j = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (j >= n) return;
    float2 *xc = X + (int64_t)j * n + b0, *ec = E + (int64_t)j * n + b0;
    float2 x[2], e[2];
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        int i = s * 32 + lane;
        x[s] = i < w ? xc[i] : make_float2(0.0f, 0.0f);
        e[s] = i < w ? ec[i] : make_float2(0.0f, 0.0f);
    }
    for (int t = 0; t < w; ++t)
    {
        const int p = FWD ? t : w - 1 - t;
        float2 v = p < 32 ? cadd(x[0], e[0]) : cadd(x[1], e[1]);
        if (!FWD && lane == (p & 31)) v = cdivide(v, tile[p][p]);
        v.x = __shfl_sync(0xffffffffu, v.x, p & 31);
        v.y = __shfl_sync(0xffffffffu, v.y, p & 31);
#pragma unroll
        for (int s = 0; s < 2; ++s)
        {
            const int i = s * 32 + lane;
            if (!FWD && i == p)
            {
                x[s] = v;
                e[s] = make_float2(0.0f, 0.0f);
            }
            if (FWD ? (i > p && i < w) : (i < p)) ccomp_submul(x[s], e[s], tile[p][i], v);
        }
    }
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        int i = s * 32 + lane;
        if (i < w)
        {
            xc[i] = x[s];
            ec[i] = e[s];
        }
    }
}

// Rows [r0, r0 + rows) of every column: the compensated update from the solved block
// [b0, b0 + w).  Forward: p ascending with v = x_p + e_p; backward: p descending with v = x_p.
// Tiles of 32 rows x 32 columns; thread (row tx, columns ty + 8 jj).
template <bool FWD>
__global__ void __launch_bounds__(256) cinv_update_kernel(const float2 *a, int lda, float2 *X, float2 *E, int n,
                                                          int r0, int rows, int b0, int w, const int *info)
{
    if (*info != 0) return;
    __shared__ float2 Fs[INV_BLOCK][32];
    __shared__ float2 Vs[INV_BLOCK][INV_TILE_COLS];
    const int tr = blockIdx.x * 32, tc = blockIdx.y * INV_TILE_COLS;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int idx = threadIdx.x; idx < w * 32; idx += 256)
    {
        int r = idx % 32, p = idx / 32;
        Fs[p][r] = tr + r < rows ? a[(int64_t)(b0 + p) * lda + r0 + tr + r] : make_float2(0.0f, 0.0f);
    }
    for (int idx = threadIdx.x; idx < w * INV_TILE_COLS; idx += 256)
    {
        int p = idx % w, c = idx / w;
        float2 v = make_float2(0.0f, 0.0f);
        if (tc + c < n)
        {
            int64_t off = (int64_t)(tc + c) * n + b0 + p;
            v = FWD ? cadd(X[off], E[off]) : X[off];
        }
        Vs[p][c] = v;
    }
    __syncthreads();
    const int r = r0 + tr + tx;
    if (tr + tx >= rows) return;
    float2 x[4], e[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
    {
        int c = tc + ty + 8 * jj;
        x[jj] = c < n ? X[(int64_t)c * n + r] : make_float2(0.0f, 0.0f);
        e[jj] = c < n ? E[(int64_t)c * n + r] : make_float2(0.0f, 0.0f);
    }
    for (int s = 0; s < w; ++s)
    {
        const int p = FWD ? s : w - 1 - s;
        const float2 f = Fs[p][tx];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) ccomp_submul(x[jj], e[jj], f, Vs[p][ty + 8 * jj]);
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
    {
        int c = tc + ty + 8 * jj;
        if (c < n)
        {
            X[(int64_t)c * n + r] = x[jj];
            E[(int64_t)c * n + r] = e[jj];
        }
    }
}

__global__ void cinv_store_kernel(const float2 *X, int n, float2 *C, int ldc, const int *info)
{
    if (*info != 0) return;
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * n) return;
    int r = (int)(idx % n), j = (int)(idx / n);
    C[(int64_t)j * ldc + r] = X[idx];
}

// ---------------------------------------------------------------------------------------
// Direct inverse: Gauss-Jordan, W lanes per matrix (lane = column), column in registers.
// ---------------------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ float2 reg_get(const float2 (&v)[W], int i)
{
    float2 out = v[0];
#pragma unroll
    for (int r = 1; r < W; ++r)
        if (r == i) out = v[r];
    return out;
}

template <int W>
__device__ __forceinline__ void reg_set(float2 (&v)[W], int i, float2 x)
{
#pragma unroll
    for (int r = 0; r < W; ++r)
        if (r == i) v[r] = x;
}

template <int W>
__device__ __forceinline__ float2 bcast(float2 v, int src)
{
    return make_float2(__shfl_sync(0xffffffffu, v.x, src, W), __shfl_sync(0xffffffffu, v.y, src, W));
}

template <int W>
__global__ void __launch_bounds__(256) cmatinv_gj_kernel(const float2 *const *a_table, float2 *const *c_table,
                                                         int n, int lda, int ldc, int *info, int count)
{
    const int gid = (blockIdx.x * blockDim.x + threadIdx.x) / W;
    const int lane = threadIdx.x % W;
    const bool live = gid < count;  // every lane stays for the shuffles
    const int q = live ? gid : count - 1;
    const float2 *a = slot(a_table, q);
    float2 col[W];
#pragma unroll
    for (int r = 0; r < W; ++r)
        col[r] = lane < n && r < n ? a[(int64_t)lane * lda + r] : make_float2(0.0f, 0.0f);
    int status = 0, own_pivot = lane;
#pragma unroll
    for (int c = 0; c < W; ++c)
    {
        if (c < n)
        {
            int row = c;
            if (lane == c)
            {
                uint32_t best = 0;
#pragma unroll
                for (int r = 0; r < W; ++r)
                    if (r >= c && r < n)
                    {
                        uint32_t s = cscore(col[r]);
                        if (s > best)
                        {
                            best = s;
                            row = r;
                        }
                    }
            }
            const int p = __shfl_sync(0xffffffffu, row, c, W);
            if (lane == c) own_pivot = p;
            {
                float2 top = col[c];
                float2 other = reg_get<W>(col, p);
                reg_set<W>(col, p, top);
                col[c] = other;
            }
            const float2 d = bcast<W>(col[c], c);
            if (czero(d) && status == 0) status = c + 1;
            const Divisor dv = cprepare(d);
            const float2 inv = cdivide(make_float2(1.0f, 0.0f), dv);
            const float2 upper = lane == c ? inv : cdivide(col[c], dv);
            col[c] = upper;
#pragma unroll
            for (int r = 0; r < W; ++r)
                if (r != c && r < n)
                {
                    const float2 f = bcast<W>(col[r], c);
                    if (lane == c)
                        col[r] = make_float2(fma_rn(f.y, inv.y, mul_rn(-f.x, inv.x)),
                                             fma_rn(-f.x, inv.y, mul_rn(-f.y, inv.x)));
                    else
                        col[r] = csubmul(col[r], f, upper);
                }
        }
    }
    int target = lane;
    for (int r = n - 1; r >= 0; --r)
    {
        int pv = __shfl_sync(0xffffffffu, own_pivot, r, W);
        target = target == r ? pv : target == pv ? r : target;
    }
    if (!live) return;
    if (status == 0 && lane < n)
    {
        float2 *c = slot(c_table, q) + (int64_t)target * ldc;
#pragma unroll
        for (int r = 0; r < W; ++r)
            if (r < n) c[r] = col[r];
    }
    if (lane == 0) info[q] = status;
}

std::atomic<unsigned long long> g_panel_attr{0}, g_resident_attr{0};

cudaError_t panel_attr()
{
    return once_per_device(g_panel_attr,
                           []
                           {
                               cudaError_t e = cudaFuncSetAttribute(cgetrf_panel_kernel,
                                                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                    (int)(CAPACITY * sizeof(float2)));
                               if (e == cudaSuccess)
                                   e = cudaFuncSetAttribute(cgetrf_row_panel_kernel,
                                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                            (int)(ROW_MAX * ROW_PITCH * sizeof(float2)));
                               return e;
                           });
}

// Factor panel columns [k, k + w) (w <= 32) of rows [k, m): each row owned by one thread,
// over a cluster of ceil((m - k) / 512) blocks (at most 8 for m <= 4096).
cudaError_t factor_panel(float2 *A, int lda, int m, int k, int w, int *ipiv, int *info, cudaStream_t stream)
{
    const int H = m - k;
    const int cl = (H + ROW_MAX - 1) / ROW_MAX;
    if (cl > 8) return cudaErrorInvalidValue;
    const int R = (H + cl - 1) / cl;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3((R + 31) / 32 * 32);
    cfg.dynamicSmemBytes = (size_t)cfg.blockDim.x * ROW_PITCH * sizeof(float2);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, cgetrf_row_panel_kernel, A, lda, m, k, w, R, ipiv, info);
}

cudaError_t resident_attr()
{
    return once_per_device(g_resident_attr,
                           []
                           {
                               const int bytes = PANEL * 256 * (int)sizeof(float2);
                               cudaError_t e = cudaFuncSetAttribute(cgetri_resident_kernel<8>,
                                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                               if (e == cudaSuccess)
                                   e = cudaFuncSetAttribute(cgetri_resident_kernel<4>,
                                                            cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
                               return e;
                           });
}

cudaError_t chain_update(float2 *C, int64_t ldc, const float2 *A, int64_t lda, const float2 *B, int64_t ldb, int rows,
                         int cols, int k, bool desc, cudaStream_t stream)
{
    if (rows <= 0 || cols <= 0 || k <= 0) return cudaSuccess;
    dim3 grid((rows + UPD_TILE - 1) / UPD_TILE, (cols + UPD_TILE - 1) / UPD_TILE);
    if (desc)
        cchain_update_kernel<true><<<grid, 256, 0, stream>>>(C, ldc, A, lda, B, ldb, rows, cols, k);
    else
        cchain_update_kernel<false><<<grid, 256, 0, stream>>>(C, ldc, A, lda, B, ldb, rows, cols, k);
    return cudaGetLastError();
}

cudaError_t trsm_block(bool fwd, bool unit, const float2 *T, int64_t ldt, float2 *X, int64_t ldx, int w, int ncols,
                       cudaStream_t stream)
{
    if (ncols <= 0 || w <= 0) return cudaSuccess;
    const int per_block = TRSM_THREADS / 32;
    const int grid = (ncols + per_block - 1) / per_block;
    if (fwd && unit)
        ctrsm_block_kernel<true, true><<<grid, TRSM_THREADS, 0, stream>>>(T, ldt, X, ldx, w, ncols);
    else if (fwd)
        ctrsm_block_kernel<true, false><<<grid, TRSM_THREADS, 0, stream>>>(T, ldt, X, ldx, w, ncols);
    else if (unit)
        ctrsm_block_kernel<false, true><<<grid, TRSM_THREADS, 0, stream>>>(T, ldt, X, ldx, w, ncols);
    else
        ctrsm_block_kernel<false, false><<<grid, TRSM_THREADS, 0, stream>>>(T, ldt, X, ldx, w, ncols);
    return cudaGetLastError();
}

cudaError_t laswp(float2 *A, int64_t lda, int ncols, int k0, int k1, const int *ipiv, int skip0, int skip1,
                  bool reverse, cudaStream_t stream)
{
    if (ncols <= 0 || k1 <= k0 || ncols <= skip1 - skip0) return cudaSuccess;
    claswp_kernel<<<(ncols + 255) / 256, 256, 0, stream>>>(A, lda, ncols, k0, k1, ipiv, skip0, skip1, reverse);
    return cudaGetLastError();
}
}  // namespace

// ---------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------

cudaError_t launch_cgetrf(float2 *A, int lda, int m, int n, int *ipiv, int *info, cudaStream_t stream)
{
    if (m <= 0 || n <= 0) return cudaSuccess;
    cudaError_t e = panel_attr();
    if (e != cudaSuccess) return e;
    const int lim = std::min(m, n);
    if ((int64_t)m * n <= CAPACITY)
    {
        cgetrf_panel_kernel<<<1, PANEL_THREADS, (size_t)m * n * sizeof(float2), stream>>>(A, lda, m, 0, lim, n, ipiv,
                                                                                           info);
        return cudaGetLastError();
    }
    for (int k = 0; k < lim && e == cudaSuccess; k += PANEL)
    {
        const int kb = std::min(PANEL, lim - k);
        e = factor_panel(A, lda, m, k, kb, ipiv, info, stream);
        if (e == cudaSuccess && ipiv && n > kb)
        {
            claswp_panel_kernel<<<(n + 3) / 4, 256, 0, stream>>>(A, lda, n, k, kb, ipiv, k, k + kb);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && k + kb < n)
        {
            float2 *diag = A + (int64_t)k * lda + k;
            e = trsm_block(true, true, diag, lda, A + (int64_t)(k + kb) * lda + k, lda, kb, n - k - kb, stream);
            if (e == cudaSuccess)
                e = chain_update(A + (int64_t)(k + kb) * lda + k + kb, lda, A + (int64_t)k * lda + k + kb, lda,
                                 A + (int64_t)(k + kb) * lda + k, lda, m - k - kb, n - k - kb, kb, false, stream);
        }
    }
    return e;
}

cudaError_t launch_cgetrs(const float2 *M, int ldm, const int *ipiv, float2 *X, int ldx, int n, int nrhs, int trans,
                          cudaStream_t stream)
{
    if (n <= 0 || nrhs <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    const bool t0 = trans == 0;
    if (t0 && ipiv) e = laswp(X, ldx, nrhs, 0, n, ipiv, 0, 0, false, stream);
    // forward sweep: unit lower (trans 0) or non-unit lower (trans 1, 2)
    for (int b0 = 0; b0 < n && e == cudaSuccess; b0 += PANEL)
    {
        const int w = std::min(PANEL, n - b0);
        e = trsm_block(true, t0, M + (int64_t)b0 * ldm + b0, ldm, X + b0, ldx, w, nrhs, stream);
        if (e == cudaSuccess)
            e = chain_update(X + b0 + w, ldx, M + (int64_t)b0 * ldm + b0 + w, ldm, X + b0, ldx, n - b0 - w, nrhs, w,
                             false, stream);
    }
    // backward sweep: non-unit upper (trans 0) or unit upper (trans 1, 2)
    const int last = ((n - 1) / PANEL) * PANEL;
    for (int b0 = last; b0 >= 0 && e == cudaSuccess; b0 -= PANEL)
    {
        const int w = std::min(PANEL, n - b0);
        e = trsm_block(false, !t0, M + (int64_t)b0 * ldm + b0, ldm, X + b0, ldx, w, nrhs, stream);
        if (e == cudaSuccess)
            e = chain_update(X, ldx, M + (int64_t)b0 * ldm, ldm, X + b0, ldx, b0, nrhs, w, true, stream);
    }
    if (e == cudaSuccess && !t0 && ipiv) e = laswp(X, ldx, nrhs, 0, n, ipiv, 0, 0, true, stream);
    return e;
}

size_t cgetri_scratch_bytes(int n)
{
    if (n <= CGETRI_RESIDENT_MAX) return 0;
    return 2 * (size_t)n * n * sizeof(float2) + (size_t)n * sizeof(int) + 256;
}

cudaError_t launch_cgetri(const float2 *a_single, const float2 *const *a_table, int lda, int64_t a_stride,
                          const int *ipiv, float2 *c_single, float2 *const *c_table, int ldc, int64_t c_stride, int n,
                          int count, int *info, void *scratch, cudaStream_t stream)
{
    if (n <= 0 || count <= 0) return cudaSuccess;
    InvArgs g{a_single, a_table, c_single, c_table, n, lda, ldc, a_stride, c_stride, ipiv, info, count};
    if (n <= CGETRI_RESIDENT_MAX)
    {
        cudaError_t e = resident_attr();
        if (e != cudaSuccess) return e;
        const int groups = (n + 7) / 8;
        const size_t smem = (size_t)PANEL * n * sizeof(float2);
        const int64_t blocks = (int64_t)count * groups;
        if (blocks > 0x7fffffff) return cudaErrorInvalidValue;
        if (n <= 32)
            cgetri_resident_kernel<1><<<(unsigned)blocks, 256, smem, stream>>>(g, groups);
        else if (n <= 64)
            cgetri_resident_kernel<2><<<(unsigned)blocks, 256, smem, stream>>>(g, groups);
        else if (n <= 128)
            cgetri_resident_kernel<4><<<(unsigned)blocks, 256, smem, stream>>>(g, groups);
        else
            cgetri_resident_kernel<8><<<(unsigned)blocks, 256, smem, stream>>>(g, groups);
        return cudaGetLastError();
    }
    // one matrix at a time over the whole GPU, state planes in scratch
    float2 *X = static_cast<float2 *>(scratch);
    float2 *E = X + (size_t)n * n;
    int *perm = reinterpret_cast<int *>(E + (size_t)n * n);
    const int64_t nn = (int64_t)n * n;
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < count && e == cudaSuccess; ++q)
    {
        // the host may hold the pointer table only on the device: the kernels read slot q
        const float2 *a = nullptr;
        float2 *c = nullptr;
        if (a_table)
        {
            e = cudaMemcpyAsync(&a, a_table + q, sizeof(a), cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&c, c_table + q, sizeof(c), cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) break;
        }
        else
        {
            a = a_single + q * a_stride;
            c = c_single + q * c_stride;
        }
        InvArgs one = g;
        one.a_single = a;
        one.a_table = nullptr;
        one.ipiv = ipiv ? ipiv + (int64_t)q * n : nullptr;
        one.info = info + q;
        cinv_check_kernel<<<1, 256, 0, stream>>>(one, 0, perm);
        cinv_init_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, stream>>>(X, E, n, perm, info + q);
        e = cudaGetLastError();
        const int colblocks = (n + 7) / 8;
        for (int b0 = 0; b0 < n && e == cudaSuccess; b0 += INV_BLOCK)
        {
            const int w = std::min(INV_BLOCK, n - b0);
            cinv_block_kernel<true><<<colblocks, 256, 0, stream>>>(a, lda, X, E, n, b0, w, info + q);
            const int rows = n - b0 - w;
            if (rows > 0)
            {
                dim3 grid((rows + 31) / 32, (n + INV_TILE_COLS - 1) / INV_TILE_COLS);
                cinv_update_kernel<true><<<grid, 256, 0, stream>>>(a, lda, X, E, n, b0 + w, rows, b0, w, info + q);
            }
            e = cudaGetLastError();
        }
        const int last = ((n - 1) / INV_BLOCK) * INV_BLOCK;
        for (int b0 = last; b0 >= 0 && e == cudaSuccess; b0 -= INV_BLOCK)
        {
            const int w = std::min(INV_BLOCK, n - b0);
            cinv_block_kernel<false><<<colblocks, 256, 0, stream>>>(a, lda, X, E, n, b0, w, info + q);
            if (b0 > 0)
            {
                dim3 grid((b0 + 31) / 32, (n + INV_TILE_COLS - 1) / INV_TILE_COLS);
                cinv_update_kernel<false><<<grid, 256, 0, stream>>>(a, lda, X, E, n, 0, b0, b0, w, info + q);
            }
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
        {
            cinv_store_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, stream>>>(X, n, c, ldc, info + q);
            e = cudaGetLastError();
        }
    }
    return e;
}

cudaError_t launch_cmatinv(const float2 *const *a_table, float2 *const *c_table, int n, int lda, int ldc, int *info,
                           int count, cudaStream_t stream)
{
    if (n <= 0 || count <= 0) return cudaSuccess;
    if (n > 32) return cudaErrorInvalidValue;
    const int W = n <= 1 ? 1 : n <= 2 ? 2 : n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : 32;
    const int64_t threads = (int64_t)count * W;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    switch (W)
    {
    case 1: cmatinv_gj_kernel<1><<<grid, 256, 0, stream>>>(a_table, c_table, n, lda, ldc, info, count); break;
    case 2: cmatinv_gj_kernel<2><<<grid, 256, 0, stream>>>(a_table, c_table, n, lda, ldc, info, count); break;
    case 4: cmatinv_gj_kernel<4><<<grid, 256, 0, stream>>>(a_table, c_table, n, lda, ldc, info, count); break;
    case 8: cmatinv_gj_kernel<8><<<grid, 256, 0, stream>>>(a_table, c_table, n, lda, ldc, info, count); break;
    case 16: cmatinv_gj_kernel<16><<<grid, 256, 0, stream>>>(a_table, c_table, n, lda, ldc, info, count); break;
    default: cmatinv_gj_kernel<32><<<grid, 256, 0, stream>>>(a_table, c_table, n, lda, ldc, info, count); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_ccopy_ok(const float2 *src, int n, float2 *dst, int ldd, const int *info, cudaStream_t stream)
{
    if (n <= 0) return cudaSuccess;
    const int64_t nn = (int64_t)n * n;
    cinv_store_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, stream>>>(src, n, dst, ldd, info);
    return cudaGetLastError();
}

__global__ void cconj_kernel(float2 *p, int64_t count)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i].y = -p[i].y;
}

cudaError_t launch_cconj(float2 *p, int64_t count, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    cconj_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(p, count);
    return cudaGetLastError();
}

// Row-major host layout <-> column-major device layout for complex64 (8-byte elements):
// dst(c, r) = op(src(r, c)) with dst column-major (ld ldd) and src rows of length ld lds.
__global__ void ctranspose_kernel(const float2 *src, int64_t lds, float2 *dst, int64_t ldd, int rows, int cols,
                                  bool conj)
{
    __shared__ float2 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y)
    {
        int r = by + i, c = bx + threadIdx.x;
        if (r < rows && c < cols) t[i][threadIdx.x] = src[(int64_t)r * lds + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y)
    {
        int c = bx + i, r = by + threadIdx.x;
        if (r < rows && c < cols)
        {
            float2 v = t[threadIdx.x][i];
            if (conj) v.y = -v.y;
            dst[(int64_t)c * ldd + r] = v;
        }
    }
}

// src is `rows` rows of `cols` elements (row stride lds); dst(c + r*...) is its transpose.
cudaError_t launch_ctranspose(const float2 *src, int64_t lds, float2 *dst, int64_t ldd, int rows, int cols, bool conj,
                              cudaStream_t stream)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    ctranspose_kernel<<<grid, block, 0, stream>>>(src, lds, dst, ldd, rows, cols, conj);
    return cudaGetLastError();
}
}  // namespace ops_solver
