// lu_solve.cu -- LU solve P A X = B for orders above the register-resident kernels
// (64 < n <= 8192), one 256-thread block per (matrix, group of up to 8 right-hand sides).
//
// Order (the oracle's orc_sgetrs).  trans 0: row interchanges applied in sequence, then the
// unit-lower forward sweep x_i = fma(-l_ik, x_k, x_i) in ascending k, then the upper sweep
// x_k = x_k / u_kk, x_i = fma(-u_ik, x_k, x_i) in descending k.  trans 1 (A^T x = b): the
// forward sweep with U^T, x_k = x_k / u_kk, x_i = fma(-u_ki, x_k, x_i) in ascending k, the
// backward sweep with L^T, x_i = fma(-l_ki, x_k, x_i) in descending k, then the interchanges
// in reverse.  Blocking keeps every element's sequence: columns go in blocks of 32 (the last
// one ragged); the 32 x 32 diagonal triangle is solved by one warp per right-hand side with
// shuffles, then every other row takes its block's 32 updates in order.  Transposed strips
// are 32 rows of the factor (32 contiguous floats per column), staged row-major at a pitch of
// 36 floats so a thread's four-wide reads of its own row are free of bank conflicts.
//
// The solution vectors stay in shared memory.  The factor is streamed from global memory
// once, as a queue of tiles (a block's 32 x 32 diagonal triangle, then its 32-column strips
// of up to 256 rows) copied by cp.async into a three-stage shared ring: two tiles are in
// flight while the third is applied, so the sweep runs at the copy rate rather than paying
// the memory latency per tile.
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int ST = 256;  // threads per block
constexpr int KB = 32;   // column block
constexpr int MAX_RHS_PER_BLOCK = 8;
constexpr int OUTER = BLOCKED_OUTER_COLS / KB;  // column blocks per block of a factorisation's change lists
static_assert(2 * ST >= 2 * KB * MAX_RHS_PER_BLOCK, "a panel's moves for all right-hand sides, two per thread");

constexpr int SR = 256;      // rows of a strip
constexpr int SP = SR + 4;   // stage pitch (floats)
constexpr int STAGES = 3;    // tiles in flight: the one in use and two being copied
constexpr int SRT = 224;     // rows (factor columns) of a transposed strip
constexpr int TP = KB + 4;   // transposed stage pitch (floats)
static_assert(SRT * TP <= KB * SP, "a transposed strip fits a stage");

// One unit of the sweep: the diagonal triangle of block `blk` (strip < 0) or a strip of up
// to 256 rows off the diagonal block (below it going forward, above it going backward).
struct Task
{
    int blk;
    int strip;
};

template <bool TRANS>
__device__ __forceinline__ constexpr int strip_rows()
{
    return TRANS ? SRT : SR;
}

template <bool FORWARD, bool TRANS>
__device__ __forceinline__ int strips(int n, int blk)
{
    const int kb = blk * KB;
    const int w = min(KB, n - kb);
    const int rows = FORWARD ? n - kb - w : kb;
    return (rows + strip_rows<TRANS>() - 1) / strip_rows<TRANS>();
}

// Advances to the next task of the sweep; false past the end.
template <bool FORWARD, bool TRANS>
__device__ __forceinline__ bool next_task(int n, int nblk, Task &task)
{
    if (task.strip + 1 < strips<FORWARD, TRANS>(n, task.blk))
    {
        ++task.strip;
        return true;
    }
    task.blk += FORWARD ? 1 : -1;
    task.strip = -1;
    return FORWARD ? task.blk < nblk : task.blk >= 0;
}

// First row and row count of a task's tile (columns kb .. kb + w - 1; transposed: the rows
// of x it updates, which are columns of the factor).
template <bool FORWARD, bool TRANS>
__device__ __forceinline__ void task_rows(int n, Task task, int &row0, int &rows)
{
    constexpr int R = strip_rows<TRANS>();
    const int kb = task.blk * KB;
    const int w = min(KB, n - kb);
    if (task.strip < 0)
    {
        row0 = kb;
        rows = w;
    }
    else if (FORWARD)
    {
        row0 = kb + w + task.strip * R;
        rows = min(R, n - row0);
    }
    else
    {
        row0 = task.strip * R;
        rows = min(R, kb - row0);
    }
}

__device__ __forceinline__ void cp_async16(float *dst, const float *src, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(float *dst, const float *src, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Starts the copy of a task's tile into stage[k][r] (k < 32 columns, r < rows); entries past
// the tile are zero-filled.  vec: 16-byte copies (the matrix is 16-byte aligned, lda % 4 == 0).
// A transposed strip goes to stage[r][k] = A(kb + k, row0 + r) (pitch TP): factor column
// row0 + r, rows kb .. kb + 31.
template <bool FORWARD, bool TRANS>
__device__ __forceinline__ void issue_task(const float *A, int lda, int n, Task task, float *stage, bool vec,
                                          const float *dinv)
{
    int row0, rows;
    task_rows<FORWARD, TRANS>(n, task, row0, rows);
    const int kb = task.blk * KB;
    const int w = min(KB, n - kb);
    if (TRANS && task.strip >= 0)
    {
        if (vec)
        {
            for (int c = threadIdx.x; c < SRT * (KB / 4); c += ST)
            {
                const int r = c / (KB / 4), k = (c % (KB / 4)) * 4;
                const int valid = r < rows ? max(0, min(4, w - k)) : 0;
                const float *src = valid ? A + (int64_t)(row0 + r) * lda + kb + k : A;
                cp_async16(stage + r * TP + k, src, valid * 4);
            }
        }
        else
        {
            for (int c = threadIdx.x; c < SRT * KB; c += ST)
            {
                const int r = c / KB, k = c % KB;
                const bool valid = r < rows && k < w;
                const float *src = valid ? A + (int64_t)(row0 + r) * lda + kb + k : A;
                cp_async4(stage + r * TP + k, src, valid ? 4 : 0);
            }
        }
        return;
    }
    if (dinv && task.strip < 0)
    {
        // the block's inverse triangle (32 x 32, column-major): always 16-byte aligned
        const float *src = dinv + ((size_t)task.blk * 2 + (FORWARD ? 0 : 1)) * KB * KB;
        for (int c = threadIdx.x; c < KB * KB / 4; c += ST)
        {
            const int k = c / (KB / 4), r = (c % (KB / 4)) * 4;
            cp_async16(stage + k * SP + r, src + k * KB + r, 16);
        }
        return;
    }
    const int span = task.strip < 0 ? KB : SR;  // rows to fill
    if (vec)
    {
        const int per = span / 4;  // 16-byte chunks per column
        for (int c = threadIdx.x; c < KB * per; c += ST)
        {
            const int k = c / per, r = (c % per) * 4;
            const int valid = k < w ? max(0, min(4, rows - r)) : 0;
            const float *src = valid ? A + (int64_t)(kb + k) * lda + row0 + r : A;
            cp_async16(stage + k * SP + r, src, valid * 4);
        }
    }
    else
    {
        for (int c = threadIdx.x; c < KB * span; c += ST)
        {
            const int k = c / span, r = c % span;
            const bool valid = k < w && r < rows;
            const float *src = valid ? A + (int64_t)(kb + k) * lda + row0 + r : A;
            cp_async4(stage + k * SP + r, src, valid ? 4 : 0);
        }
    }
}

// Factors whose L columns keep their 128-column block's row order (launch_getrf_blocked with
// `lists`): before the forward sweep reaches such a block's first column, the vectors take the
// row changes of that block's (up to four) 32-column panels, in order, so that every L column meets the
// vectors in the row order it was stored in.  Each panel's moves are read before any is
// written.  Block-uniform control flow (the counts come from global memory).
__device__ __forceinline__ void apply_block_changes(const short *lists, int blk, int n, float *x, int nr)
{
    const int t = threadIdx.x;
    const int npanel = (n + KB - 1) / KB;
    for (int p = blk; p < min(blk + OUTER, npanel); ++p)
    {
        const short *entry = lists + (size_t)p * PANEL_LIST_SHORTS;
        const int cnt = entry[0];
        if (cnt == 0) continue;
        const int kp = p * KB;
        float v[2];
        int dst[2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int e = t + h * ST;
            dst[h] = -1;
            if (e < cnt * nr)
            {
                const int r = e / cnt, i = e % cnt;
                dst[h] = r * n + kp + entry[1 + i];
                v[h] = x[r * n + kp + entry[1 + 2 * KB + i]];
            }
        }
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (dst[h] >= 0) x[dst[h]] = v[h];
        __syncthreads();
    }
}

// The interchanges of ipiv in order (LAPACK form, validated by the caller): warp r applies them
// to right-hand side r; the pivots come 32 at a time into the lanes' registers, so the
// serial chain of swaps runs on shared memory and shuffles alone.
__device__ __forceinline__ void apply_pivots(const int *piv, int n, float *x, int nr)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp >= nr) return;
    float *xr = x + (size_t)warp * n;
    for (int c0 = 0; c0 < n; c0 += 32)
    {
        const int k = c0 + lane;
        const int pv = k < n ? piv[k] - 1 : k;
        const int cnt = min(32, n - c0);
#pragma unroll
        for (int j = 0; j < 32; ++j)
        {
            if (j >= cnt) break;  // uniform
            const int p = __shfl_sync(0xffffffffu, pv, j);
            if (lane == 0 && p != c0 + j)
            {
                const float a = xr[c0 + j];
                xr[c0 + j] = xr[p];
                xr[p] = a;
            }
        }
    }
}

// The interchanges of ipiv in reverse order (the transposed solve's last step, x = P^T z):
// warp r on right-hand side r, the pivots 32 at a time from the last chunk down.
__device__ __forceinline__ void apply_pivots_reverse(const int *piv, int n, float *x, int nr)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp >= nr) return;
    float *xr = x + (size_t)warp * n;
    for (int c0 = ((n - 1) / 32) * 32; c0 >= 0; c0 -= 32)
    {
        const int k = c0 + lane;
        const int pv = k < n ? piv[k] - 1 : k;
        const int cnt = min(32, n - c0);
#pragma unroll
        for (int j = 31; j >= 0; --j)
        {
            if (j >= cnt) continue;  // uniform
            const int p = __shfl_sync(0xffffffffu, pv, j);
            if (lane == 0 && p != c0 + j)
            {
                const float a = xr[c0 + j];
                xr[c0 + j] = xr[p];
                xr[p] = a;
            }
        }
    }
}

template <bool FORWARD, bool TRANS>
__device__ void sweep(const float *A, int lda, int n, float *x, int nr, float *stages, bool vec, const float *dinv,
                      const short *lists, const int *piv)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nblk = (n + KB - 1) / KB;
    // the task queue: q[0] is applied while the next STAGES - 1 are in flight
    Task q[STAGES];
    bool live[STAGES];
    q[0] = Task{FORWARD ? 0 : nblk - 1, -1};
    live[0] = true;
#pragma unroll
    for (int i = 1; i < STAGES; ++i)
    {
        q[i] = q[i - 1];
        live[i] = live[i - 1] && next_task<FORWARD, TRANS>(n, nblk, q[i]);
    }
#pragma unroll
    for (int i = 0; i < STAGES - 1; ++i)
    {
        if (live[i]) issue_task<FORWARD, TRANS>(A, lda, n, q[i], stages + (size_t)i * KB * SP, vec, dinv);
        cp_commit();
    }
    // the row interchanges run while the first tiles are copied (the loop's first barrier
    // publishes them)
    if (FORWARD && !TRANS && piv) apply_pivots(piv, n, x, nr);
    int slot = 0;
    while (live[0])
    {
        // One barrier per task.  This task's tile has landed (for this thread's copies: the
        // group that may still be in flight is the next task's) ...
        cp_wait<STAGES - 2>();
        // ... and for everyone's; every thread is also done with the previous task, so its
        // updates of x are visible and its stage may be refilled
        __syncthreads();
        // refill: the task STAGES - 1 ahead goes to the stage freed by the previous task
        if (live[STAGES - 1])
            issue_task<FORWARD, TRANS>(A, lda, n, q[STAGES - 1],
                                stages + (size_t)((slot + STAGES - 1) % STAGES) * KB * SP, vec, dinv);
        cp_commit();
        const float *tile = stages + (size_t)slot * KB * SP;
        const Task cur = q[0];
        const int kb = cur.blk * KB;
        const int w = min(KB, n - kb);
        if (FORWARD && lists && cur.strip < 0 && cur.blk % OUTER == 0) apply_block_changes(lists, cur.blk, n, x, nr);
        if (cur.strip < 0)
        {
            // diagonal triangle: warp r solves right-hand side r, lane i on row kb + i
            if (warp < nr && dinv)
            {
                // with the block's inverse: x_blk = inv x_blk, four partial sums per lane
                float *xr = x + (size_t)warp * n;
                const float xv = lane < w ? xr[kb + lane] : 0.0f;
                float s4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int k = 0; k < KB; ++k)
                {
                    const float xk = __shfl_sync(0xffffffffu, xv, k);
                    s4[k & 3] = fma_rn(tile[k * SP + lane], xk, s4[k & 3]);
                }
                if (lane < w) xr[kb + lane] = (s4[0] + s4[1]) + (s4[2] + s4[3]);
            }
            else if (TRANS && warp < nr)
            {
                // U^T forward (divide, then update the rows below) or L^T backward (unit); lane
                // i reads factor element (kb + k, kb + i) = tile[i][k]
                float *xr = x + (size_t)warp * n;
                float xv = lane < w ? xr[kb + lane] : 0.0f;
                if (FORWARD)
                {
                    const float dl = lane < w ? tile[lane * SP + lane] : 1.0f;
                    const float yl = div_prepare(dl);
                    const bool okl = div_range(dl);
#pragma unroll
                    for (int k = 0; k < KB; ++k)
                    {
                        if (k < w)
                        {
                            if (lane == k) xv = div_by(xv, dl, yl, okl);
                            const float xk = __shfl_sync(0xffffffffu, xv, k);
                            if (lane > k && lane < w) xv = fma_rn(-tile[lane * SP + k], xk, xv);
                        }
                    }
                }
                else
                {
#pragma unroll
                    for (int k = KB - 1; k >= 0; --k)
                    {
                        const float xk = __shfl_sync(0xffffffffu, xv, k);
                        if (lane < k && k < w) xv = fma_rn(-tile[lane * SP + k], xk, xv);
                    }
                }
                if (lane < w) xr[kb + lane] = xv;
            }
            else if (warp < nr)
            {
                float *xr = x + (size_t)warp * n;
                float xv = lane < w ? xr[kb + lane] : 0.0f;
                if (FORWARD)
                {
#pragma unroll
                    for (int k = 0; k < KB; ++k)
                    {
                        const float xk = __shfl_sync(0xffffffffu, xv, k);
                        if (lane > k && lane < w) xv = fma_rn(-tile[k * SP + lane], xk, xv);
                    }
                }
                else
                {
                    // each lane's divisor is its own diagonal entry: reciprocal ahead of the chain
                    const float dl = lane < w ? tile[lane * SP + lane] : 1.0f;
                    const float yl = div_prepare(dl);
                    const bool okl = div_range(dl);
#pragma unroll
                    for (int k = KB - 1; k >= 0; --k)
                    {
                        if (k < w)
                        {
                            if (lane == k) xv = div_by(xv, dl, yl, okl);
                            const float xk = __shfl_sync(0xffffffffu, xv, k);
                            if (lane < k) xv = fma_rn(-tile[k * SP + lane], xk, xv);
                        }
                    }
                }
                if (lane < w) xr[kb + lane] = xv;
            }
        }
        else
        {
            int row0, rows;
            task_rows<FORWARD, TRANS>(n, cur, row0, rows);
            if (TRANS && t < rows)
            {
                // this thread's factor column, rows kb .. kb + 31, four at a time
                const float *col = tile + t * TP;
                const int row = row0 + t;
                for (int r = 0; r < nr; ++r)
                {
                    float *xr = x + (size_t)r * n;
                    float acc = xr[row];
                    if (FORWARD)
                    {
#pragma unroll
                        for (int k4 = 0; k4 < KB; k4 += 4)
                        {
                            const float4 u = *reinterpret_cast<const float4 *>(col + k4);
                            if (k4 < w) acc = fma_rn(-u.x, xr[kb + k4], acc);
                            if (k4 + 1 < w) acc = fma_rn(-u.y, xr[kb + k4 + 1], acc);
                            if (k4 + 2 < w) acc = fma_rn(-u.z, xr[kb + k4 + 2], acc);
                            if (k4 + 3 < w) acc = fma_rn(-u.w, xr[kb + k4 + 3], acc);
                        }
                    }
                    else
                    {
#pragma unroll
                        for (int k4 = KB - 4; k4 >= 0; k4 -= 4)
                        {
                            const float4 u = *reinterpret_cast<const float4 *>(col + k4);
                            if (k4 + 3 < w) acc = fma_rn(-u.w, xr[kb + k4 + 3], acc);
                            if (k4 + 2 < w) acc = fma_rn(-u.z, xr[kb + k4 + 2], acc);
                            if (k4 + 1 < w) acc = fma_rn(-u.y, xr[kb + k4 + 1], acc);
                            if (k4 < w) acc = fma_rn(-u.x, xr[kb + k4], acc);
                        }
                    }
                    xr[row] = acc;
                }
            }
            else if (!TRANS && t < rows)
            {
                const int row = row0 + t;
                for (int r = 0; r < nr; ++r)
                {
                    float *xr = x + (size_t)r * n;
                    float acc = xr[row];
                    if (FORWARD)
                    {
#pragma unroll
                        for (int k = 0; k < KB; ++k)
                            if (k < w) acc = fma_rn(-tile[k * SP + t], xr[kb + k], acc);
                    }
                    else
                    {
#pragma unroll
                        for (int k = KB - 1; k >= 0; --k)
                            if (k < w) acc = fma_rn(-tile[k * SP + t], xr[kb + k], acc);
                    }
                    xr[row] = acc;
                }
            }
        }
        // a diagonal solve feeds its strips and a block's strips feed the next diagonal: the
        // next iteration's barrier orders them
#pragma unroll
        for (int i = 0; i < STAGES - 1; ++i)
        {
            q[i] = q[i + 1];
            live[i] = live[i + 1];
        }
        q[STAGES - 1] = q[STAGES - 2];
        live[STAGES - 1] = live[STAGES - 2] && next_task<FORWARD, TRANS>(n, nblk, q[STAGES - 1]);
        slot = (slot + 1) % STAGES;
    }
    cp_wait<0>();
    __syncthreads();  // the last task is done before the caller reuses the stages and reads x
}

__global__ void __launch_bounds__(ST, 2) getrs_blocked_kernel(float *a_single, float *const *a_table, int a_first,
                                                            const int *ipiv, const int *perm, float *b_single,
                                                            float *const *b_table, int b_first, int n, int lda,
                                                            int ldb, int nrhs, int count, int RHS, int *info,
                                                            const int *skip, const float *dinv_all, int nblk,
                                                            const short *lists_all, int trans)
{
    extern __shared__ __align__(16) float dyn[];
    float *stages = dyn;                          // STAGES x KB x SP
    float *x = dyn + (size_t)STAGES * KB * SP;    // RHS x n
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
            // (transposed: the permutation is applied on the way out)
            x[e] = B[(int64_t)(r0 + r) * ldb + (sig && !trans ? sig[i] : i)];
        }
        __syncthreads();
        if (bad)
        {
            if (t == 0 && info && r0 == 0) info[q] = -6;
            __syncthreads();
            continue;
        }
        const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0;
        const float *dinv = dinv_all ? dinv_all + (size_t)q * nblk * 2 * KB * KB : nullptr;
        const short *lists = lists_all ? lists_all + (size_t)q * BLOCKED_PANELS * PANEL_LIST_SHORTS : nullptr;
        if (trans)
        {
            sweep<true, true>(A, lda, n, x, nr, stages, vec, nullptr, nullptr, nullptr);
            sweep<false, true>(A, lda, n, x, nr, stages, vec, nullptr, nullptr, nullptr);
            if (piv && !sig)
            {
                apply_pivots_reverse(piv, n, x, nr);
                __syncthreads();
            }
        }
        else
        {
            sweep<true, false>(A, lda, n, x, nr, stages, vec, dinv, lists, sig ? nullptr : piv);
            sweep<false, false>(A, lda, n, x, nr, stages, vec, dinv, nullptr, nullptr);
        }
        for (int e = t; e < nr * n; e += ST)
        {
            const int r = e / n, i = e % n;
            // transposed with a permutation: x = P^T z, so z[i] lands on row perm[i]
            B[(int64_t)(r0 + r) * ldb + (sig && trans ? sig[i] : i)] = x[e];
        }
        if (t == 0 && info && r0 == 0) info[q] = 0;
        __syncthreads();
    }
}

// The inverses of the 32 x 32 diagonal blocks of the factors: warp 0 the unit-lower L
// block's, warp 1 the upper U block's; lane j computes column j by substitution against
// e_j.  Stored column-major, per (matrix, block): L inverse then U inverse.  (A ragged last
// block of order w is inverted as w x w, the rest of the 32 x 32 identity.)
__global__ void __launch_bounds__(64) diag_inverse_kernel(float *single, float *const *table, int first, int n,
                                                          int lda, int count, float *dinv)
{
    __shared__ float D[KB][KB + 1];  // D[k][i] = factor element (row kb + i, column kb + k)
    const int nblk = (n + KB - 1) / KB;
    const int64_t q = blockIdx.x;
    const int b = blockIdx.y;
    if (q >= count) return;
    const float *A = table ? slot(table, first + q) : single;
    if (!A) return;
    const int kb = b * KB, w = min(KB, n - kb);
    {
        // all sixteen loads of a thread in flight before its stores
        float v[KB * KB / 64];
#pragma unroll
        for (int u = 0; u < KB * KB / 64; ++u)
        {
            const int e = threadIdx.x + 64 * u, k = e / KB, i = e % KB;
            v[u] = (k < w && i < w) ? A[(int64_t)(kb + k) * lda + kb + i] : (k == i ? 1.0f : 0.0f);
        }
#pragma unroll
        for (int u = 0; u < KB * KB / 64; ++u)
        {
            const int e = threadIdx.x + 64 * u;
            D[e / KB][e % KB] = v[u];
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, which = threadIdx.x >> 5;
    float y[KB];
#pragma unroll
    for (int r = 0; r < KB; ++r) y[r] = r == lane ? 1.0f : 0.0f;
    if (which == 0)
    {
#pragma unroll
        for (int k = 0; k < KB; ++k)
        {
            const float yk = y[k];
#pragma unroll
            for (int r = k + 1; r < KB; ++r) y[r] = fma_rn(-D[k][r], yk, y[r]);
        }
    }
    else
    {
#pragma unroll
        for (int k = KB - 1; k >= 0; --k)
        {
            y[k] = div_rn(y[k], D[k][k]);
            const float yk = y[k];
#pragma unroll
            for (int r = 0; r < k; ++r) y[r] = fma_rn(-D[k][r], yk, y[r]);
        }
    }
    float *dst = dinv + (((size_t)q * nblk + b) * 2 + which) * KB * KB + (size_t)lane * KB;
#pragma unroll
    for (int r = 0; r < KB; r += 4) *reinterpret_cast<float4 *>(dst + r) = make_float4(y[r], y[r + 1], y[r + 2], y[r + 3]);
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
                                 int *info, const int *skip, cudaStream_t stream, const float *dinv,
                                 const short *lists, int trans)
{
    if (lists && (a.n > BLOCKED_MAX_N || ipiv || perm)) return cudaErrorInvalidValue;
    if (trans && (dinv || lists)) return cudaErrorInvalidValue;
    const size_t stage_floats = (size_t)STAGES * KB * SP;
    // two blocks per SM when the vectors fit beside the ring, else one
    int rpb = (int)((110 * 1024 / sizeof(float) - stage_floats) / (size_t)a.n);
    if (rpb < 1) rpb = (int)((220 * 1024 / sizeof(float) - stage_floats) / (size_t)a.n);
    if (rpb > MAX_RHS_PER_BLOCK) rpb = MAX_RHS_PER_BLOCK;
    if (rpb > nrhs) rpb = nrhs;
    if (rpb < 1) return cudaErrorInvalidValue;
    const size_t smem = (stage_floats + (size_t)rpb * a.n) * sizeof(float);
    cudaFuncSetAttribute(getrs_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int groups = (nrhs + rpb - 1) / rpb;
    int64_t jobs = (int64_t)a.count * groups;
    int64_t blocks = jobs < 148 * 8 ? jobs : 148 * 8;
    if (blocks < 1) blocks = 1;
    getrs_blocked_kernel<<<(unsigned)blocks, ST, smem, stream>>>(a.single, a.table, a.first, ipiv, perm, b.single,
                                                                 b.table, b.first, a.n, a.ld, b.ld, nrhs, a.count,
                                                                 rpb, info, skip, dinv, (a.n + KB - 1) / KB,
                                                                 lists, trans);
    return cudaGetLastError();
}

cudaError_t launch_diag_inverses(const RealBatch &a, float *dinv, cudaStream_t stream)
{
    const int nblk = (a.n + KB - 1) / KB;
    diag_inverse_kernel<<<dim3((unsigned)a.count, (unsigned)nblk), 64, 0, stream>>>(a.single, a.table, a.first, a.n,
                                                                                   a.ld, a.count, dinv);
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
