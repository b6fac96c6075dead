// lu_small.cu -- batched real LU factor, solve and inverse for n <= 64 on sm_100a.
//
// getrf: one warp (or a width-N sub-warp for N < 32) owns a matrix; lane l holds rows
// l and l+32 (N = 64) in registers (order 64: getrf_rot_kernel, the columns rotated through
// the registers four at a time so that the step loop stays small).  Row interchanges are never moved in memory: each row
// carries its current position and the pivot search reduces (|a| key, position) with
// redux.sync, so the earliest-row tie rule of the reference sees the swapped order.  The
// pivot row is broadcast through a per-warp shared-memory row buffer; every other row
// takes the IEEE quotient l = a_ik / u_kk and the FMA update a_ij = fma(-l, u_kj, a_ij)
// in ascending k -- the order of real_lu.hpp:409-448 (FactorLocalCore), bit for bit.
//
// getrs: same row layout; forward (unit L) and backward (U) substitution run
// right-looking in time with one broadcast per step (oracle orc_sgetrs order).
//
// getri: one thread per inverse column, the LU factors staged once in shared memory and
// read as warp-wide broadcasts; thread t solves the permuted unit vector e_t (column
// perm[t] of the inverse), so a warp whose rows all lie below k skips the leading forward
// steps whose source is exactly zero.  Per-element order is that of
// real_lu_blocked_inverse_kernel.cpp:766-830 (forward fma(-s, L, rhs), backward
// s = rhs * (1/U_kk), fma(-s, U, rhs)).
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int LU_THREADS = 128;

template <int W>
__device__ __forceinline__ unsigned warp_max_u32(unsigned v)
{
    if constexpr (W == 32)
        return __reduce_max_sync(0xffffffffu, v);
    else
    {
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o, W));
        return v;
    }
}
template <int W>
__device__ __forceinline__ unsigned warp_min_u32(unsigned v)
{
    if constexpr (W == 32)
        return __reduce_min_sync(0xffffffffu, v);
    else
    {
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o, W));
        return v;
    }
}

// ---------------------------------------------------------------------------------------
// getrf
// ---------------------------------------------------------------------------------------
// m x n matrices with m, n <= N; steps = min(m, n) (FactorLocalCore handles rectangles).
template <int N>
__global__ void __launch_bounds__(LU_THREADS) getrf_small_kernel(float *single, float *const *table, int first, int m,
                                                                  int n, int lda, int count, int *ipiv, int *info)
{
    constexpr int SUBW = N < 32 ? N : 32;  // lanes per matrix
    constexpr int RPL = N / SUBW;           // rows per lane
    constexpr int MPW = 32 / SUBW;          // matrices per warp
    __shared__ __align__(16) float prow_all[LU_THREADS / 32][MPW][N];
    const int lane = threadIdx.x & 31;
    const int lrow = lane % SUBW;
    const int sub = lane / SUBW;
    const int warp_global = (blockIdx.x * LU_THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * LU_THREADS) >> 5;
    float *prow = prow_all[threadIdx.x >> 5][sub];
    const bool pivoting = ipiv != nullptr;
    const int steps = m < n ? m : n;

    for (int64_t group = warp_global; group * MPW < count; group += warps_total)
    {
        const int64_t q = group * MPW + sub;
        const bool in_batch = q < count;
        float *p = nullptr;
        if (in_batch) p = table ? slot(table, first + q) : single;
        const bool live = p != nullptr;

        float a[RPL][N];
        int pos[RPL];
        int pv[RPL];
#pragma unroll
        for (int s = 0; s < RPL; ++s)
        {
            const int phys = lrow + s * SUBW;
            pos[s] = phys;
            pv[s] = phys + 1;
#pragma unroll
            for (int j = 0; j < N; ++j)
                a[s][j] = (live && phys < m && j < n) ? p[phys + (int64_t)j * lda] : 0.0f;
        }
        int state = 0;

#pragma unroll
        for (int k = 0; k < N; ++k)
        {
            if (k < steps)
            {
                int pr = k, ph = k;
                if (pivoting)
                {
                    unsigned key[RPL];
#pragma unroll
                    for (int s = 0; s < RPL; ++s)
                    {
                        const int phys = lrow + s * SUBW;
                        const float v = a[s][k];
                        key[s] = (pos[s] >= k && phys < m) ? pivot_key(v) : 0u;
                        if (pos[s] == k && v != v) key[s] = 0xffffffffu;
                    }
                    unsigned best = key[0];
#pragma unroll
                    for (int s = 1; s < RPL; ++s) best = max(best, key[s]);
                    const unsigned mx = warp_max_u32<SUBW>(best);
                    unsigned cand = 0xffffffffu;
#pragma unroll
                    for (int s = 0; s < RPL; ++s)
                        if (key[s] == mx) cand = min(cand, (unsigned)((pos[s] << 8) | (lrow + s * SUBW)));
                    const unsigned mn = warp_min_u32<SUBW>(cand);
                    pr = (int)(mn >> 8);
                    ph = (int)(mn & 255u);
                    if (lrow == k % SUBW) pv[k / SUBW] = pr + 1;
#pragma unroll
                    for (int s = 0; s < RPL; ++s) pos[s] = pos[s] == k ? pr : (pos[s] == pr ? k : pos[s]);
                }
                // Broadcast the pivot row's columns >= k (aligned down to 4).
                __syncwarp();
                {
                    const int owner_slot = ph / SUBW;  // uniform within the sub-warp
                    const bool owner = lrow == (ph % SUBW);
#pragma unroll
                    for (int s = 0; s < RPL; ++s)
                    {
                        if (owner && owner_slot == s)
                        {
#pragma unroll
                            for (int j = (k & ~3); j < N; j += 4)
                                *reinterpret_cast<float4 *>(prow + j) =
                                    make_float4(a[s][j], a[s][j + 1], a[s][j + 2], a[s][j + 3]);
                        }
                    }
                }
                __syncwarp();
                const float d = prow[k];
                if (d == 0.0f && state == 0) state = k + 1;
                const bool update = d != 0.0f && k + 1 < m;
#pragma unroll
                for (int s = 0; s < RPL; ++s)
                {
                    const int phys = lrow + s * SUBW;
                    if (update && pos[s] > k && phys < m)
                    {
                        const float l = div_rn(a[s][k], d);
                        a[s][k] = l;
#pragma unroll
                        for (int j4 = ((k + 1) & ~3); j4 < N; j4 += 4)
                        {
                            const float4 u = *reinterpret_cast<const float4 *>(prow + j4);
                            if (j4 + 0 > k) a[s][j4 + 0] = fma_rn(-l, u.x, a[s][j4 + 0]);
                            if (j4 + 1 > k) a[s][j4 + 1] = fma_rn(-l, u.y, a[s][j4 + 1]);
                            if (j4 + 2 > k) a[s][j4 + 2] = fma_rn(-l, u.z, a[s][j4 + 2]);
                            if (j4 + 3 > k) a[s][j4 + 3] = fma_rn(-l, u.w, a[s][j4 + 3]);
                        }
                    }
                }
            }
        }

        if (live)
        {
#pragma unroll
            for (int s = 0; s < RPL; ++s)
            {
                const int phys = lrow + s * SUBW;
                if (phys < m)
                {
#pragma unroll
                    for (int j = 0; j < N; ++j)
                        if (j < n) p[pos[s] + (int64_t)j * lda] = a[s][j];
                    if (pivoting && phys < steps) ipiv[q * steps + phys] = pv[s];
                }
            }
        }
        if (in_batch && lrow == 0) info[q] = live ? state : -2;
    }
}

// Order 64 (m, n <= 64), the same arithmetic as getrf_small_kernel<64> with the columns
// rotated through the registers in blocks of KB: the step loop is KB steps long and runs
// 64 / KB times, so the kernel body fits the instruction cache (the fully unrolled 64-step
// body did not: its warps stalled on instruction fetch).  Register column c holds matrix
// column K0 + c.  After each block of KB steps its KB columns are final; they are parked
// in a per-warp shared-memory copy indexed by physical row (pitch 65 floats: the lanes'
// rows fall in different banks) and the remaining register columns shift down by KB.  The
// final store reads the parked copy, each row to its final position.
constexpr int ROT_N = 64;
constexpr int ROT_PITCH = ROT_N + 1;
constexpr size_t rot_smem_bytes()
{
    return (size_t)(LU_THREADS / 32) * (ROT_N + ROT_N * ROT_PITCH) * sizeof(float);
}

template <int KB>
__global__ void __launch_bounds__(LU_THREADS, 3) getrf_rot_kernel(float *single, float *const *table, int first, int m,
                                                               int n, int lda, int count, int *ipiv, int *info)
{
    constexpr int N = ROT_N, SUBW = 32, RPL = 2;
    static_assert(KB % 4 == 0 && N % KB == 0, "blocks of whole 16-byte column groups");
    extern __shared__ __align__(16) float rot_mem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *prow = rot_mem + warp * N;
    float *fin = rot_mem + (LU_THREADS / 32) * N + warp * N * ROT_PITCH;
    const int warp_global = (blockIdx.x * LU_THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * LU_THREADS) >> 5;
    const bool pivoting = ipiv != nullptr;
    const int steps = m < n ? m : n;

    for (int64_t q = warp_global; q < count; q += warps_total)
    {
        float *p = table ? slot(table, first + q) : single;
        const bool live = p != nullptr;

        float a[RPL][N];
        int pos[RPL];
        int pv[RPL];
#pragma unroll
        for (int s = 0; s < RPL; ++s)
        {
            const int phys = lane + s * SUBW;
            pos[s] = phys;
            pv[s] = phys + 1;
#pragma unroll
            for (int j = 0; j < N; ++j)
                a[s][j] = (live && phys < m && j < n) ? p[phys + (int64_t)j * lda] : 0.0f;
        }
        int state = 0;

#pragma unroll 1
        for (int K0 = 0; K0 < N; K0 += KB)
        {
            const int width = N - K0;  // register columns that hold matrix columns
#pragma unroll
            for (int kk = 0; kk < KB; ++kk)
            {
                const int k = K0 + kk;
                if (k < steps)
                {
                    int pr = k, ph = k;
                    if (pivoting)
                    {
                        unsigned key[RPL];
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                        {
                            const int phys = lane + s * SUBW;
                            const float v = a[s][kk];
                            key[s] = (pos[s] >= k && phys < m) ? pivot_key(v) : 0u;
                            if (pos[s] == k && v != v) key[s] = 0xffffffffu;
                        }
                        const unsigned mx = warp_max_u32<SUBW>(max(key[0], key[1]));
                        unsigned cand = 0xffffffffu;
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                            if (key[s] == mx) cand = min(cand, (unsigned)((pos[s] << 8) | (lane + s * SUBW)));
                        const unsigned mn = warp_min_u32<SUBW>(cand);
                        pr = (int)(mn >> 8);
                        ph = (int)(mn & 255u);
                        if (lane == k % SUBW)
                        {
                            if (k < SUBW)
                                pv[0] = pr + 1;
                            else
                                pv[1] = pr + 1;
                        }
#pragma unroll
                        for (int s = 0; s < RPL; ++s) pos[s] = pos[s] == k ? pr : (pos[s] == pr ? k : pos[s]);
                    }
                    // the pivot row's register columns >= kk (aligned down to 4) to the row buffer
                    __syncwarp();
                    {
                        const int owner_slot = ph / SUBW;
                        const bool owner = lane == (ph % SUBW);
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                        {
                            if (owner && owner_slot == s)
                            {
#pragma unroll
                                for (int j = (kk & ~3); j < N; j += 4)
                                    if (j < width)
                                        *reinterpret_cast<float4 *>(prow + j) =
                                            make_float4(a[s][j], a[s][j + 1], a[s][j + 2], a[s][j + 3]);
                            }
                        }
                    }
                    __syncwarp();
                    const float d = prow[kk];
                    if (d == 0.0f && state == 0) state = k + 1;
                    const bool update = d != 0.0f && k + 1 < m;
#pragma unroll
                    for (int s = 0; s < RPL; ++s)
                    {
                        const int phys = lane + s * SUBW;
                        if (update && pos[s] > k && phys < m)
                        {
                            const float l = div_rn(a[s][kk], d);
                            a[s][kk] = l;
#pragma unroll
                            for (int j4 = ((kk + 1) & ~3); j4 < N; j4 += 4)
                            {
                                if (j4 < width)
                                {
                                    const float4 u = *reinterpret_cast<const float4 *>(prow + j4);
                                    if (j4 + 0 > kk) a[s][j4 + 0] = fma_rn(-l, u.x, a[s][j4 + 0]);
                                    if (j4 + 1 > kk) a[s][j4 + 1] = fma_rn(-l, u.y, a[s][j4 + 1]);
                                    if (j4 + 2 > kk) a[s][j4 + 2] = fma_rn(-l, u.z, a[s][j4 + 2]);
                                    if (j4 + 3 > kk) a[s][j4 + 3] = fma_rn(-l, u.w, a[s][j4 + 3]);
                                }
                            }
                        }
                    }
                }
            }
            // columns K0 .. K0 + KB - 1 are final: park them, shift the rest down
#pragma unroll
            for (int s = 0; s < RPL; ++s)
            {
                float *row = fin + (lane + s * SUBW) * ROT_PITCH + K0;
#pragma unroll
                for (int c = 0; c < KB; ++c) row[c] = a[s][c];
#pragma unroll
                for (int j = 0; j + KB < N; ++j) a[s][j] = a[s][j + KB];
            }
        }
        __syncwarp();
        if (live)
        {
#pragma unroll
            for (int s = 0; s < RPL; ++s)
            {
                const int phys = lane + s * SUBW;
                if (phys < m)
                {
                    const float *row = fin + phys * ROT_PITCH;
                    for (int j = 0; j < n; ++j) p[pos[s] + (int64_t)j * lda] = row[j];
                    if (pivoting && phys < steps) ipiv[q * steps + phys] = pv[s];
                }
            }
        }
        if (lane == 0) info[q] = live ? state : -2;
        __syncwarp();  // the parked copy and the row buffer are rewritten by the next matrix
    }
}

// ---------------------------------------------------------------------------------------
// getrs
// ---------------------------------------------------------------------------------------
// trans 0: rows in lanes (A(i, :) in a[][]); trans 1: the transpose is staged so that
// lane i holds column i of A, and the same two sweeps run on A^T's triangles.
constexpr int RS_THREADS = 64;

template <int N, int TRANS>
__global__ void __launch_bounds__(RS_THREADS) getrs_small_kernel(float *a_single, float *const *a_table,
                                                                  int a_first, const int *ipiv, float *b_single,
                                                                  float *const *b_table, int b_first, int n, int lda,
                                                                  int ldb, int nrhs, int count, int *info)
{
    constexpr int SUBW = N < 32 ? N : 32;
    constexpr int RPL = N / SUBW;
    constexpr int MPW = 32 / SUBW;
    constexpr int P = N + 1;
    constexpr int TILE = TRANS ? N * P : 1;
    __shared__ float tstage[(RS_THREADS / 32) * MPW * TILE];
    __shared__ int pstage[(RS_THREADS / 32) * MPW * N];
    const int lane = threadIdx.x & 31;
    const int lrow = lane % SUBW;
    const int sub = lane / SUBW;
    const int warp_global = (blockIdx.x * RS_THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * RS_THREADS) >> 5;
    float *tile = tstage + ((threadIdx.x >> 5) * MPW + sub) * TILE;
    int *pv = pstage + ((threadIdx.x >> 5) * MPW + sub) * N;
    const int trans = TRANS;

    for (int64_t group = warp_global; group * MPW < count; group += warps_total)
    {
        const int64_t q = group * MPW + sub;
        const bool in_batch = q < count;
        float *pa = nullptr, *pb = nullptr;
        if (in_batch)
        {
            pa = a_table ? slot(a_table, a_first + q) : a_single;
            pb = b_table ? slot(b_table, b_first + q) : b_single;
        }
        bool live = pa != nullptr && pb != nullptr;
        float a[RPL][N];
        if (trans == 0)
        {
            // issued before the pivot check so that both wait on memory together; a matrix
            // whose pivots fail the check is loaded but never written back
#pragma unroll
            for (int s = 0; s < RPL; ++s)
            {
                const int r = lrow + s * SUBW;
#pragma unroll
                for (int j = 0; j < N; ++j) a[s][j] = (live && r < n && j < n) ? pa[r + (int64_t)j * lda] : 0.0f;
            }
        }
        // Pivots of this matrix, validated: each must lie in [k+1, n].
        __syncwarp();
        bool bad = false;
#pragma unroll
        for (int s = 0; s < RPL; ++s)
        {
            const int k = lrow + s * SUBW;
            int v = k + 1;
            if (live && ipiv && k < n) v = ipiv[q * n + k];
            if (k < n && (v < k + 1 || v > n)) bad = true;
            pv[k] = v;
        }
        const unsigned bad_any = warp_max_u32<SUBW>(bad ? 1u : 0u);
        if (bad_any) live = false;

        if constexpr (TRANS != 0)
        {
            // tile[j*P + i] = A(i, j); lane r then reads row r of A^T = column r of A.
            for (int idx = lrow; idx < N * N; idx += SUBW)
            {
                const int i = idx % N, j = idx / N;
                tile[j * P + i] = (live && i < n && j < n) ? pa[i + (int64_t)j * lda] : 0.0f;
            }
            __syncwarp();
#pragma unroll
            for (int s = 0; s < RPL; ++s)
            {
                const int r = lrow + s * SUBW;
#pragma unroll
                for (int j = 0; j < N; ++j) a[s][j] = tile[r * P + j];
            }
        }
        __syncwarp();
        // Final position of each right-hand-side row after the swap sequence: the value
        // that ends at position t started at the position reached by undoing the swaps.
        int src[RPL];
#pragma unroll
        for (int s = 0; s < RPL; ++s)
        {
            int t = lrow + s * SUBW;
            for (int k = n - 1; k >= 0; --k)
            {
                const int pk = pv[k] - 1;
                t = t == k ? pk : (t == pk ? k : t);
            }
            src[s] = t;
        }

        for (int rhs = 0; rhs < nrhs; ++rhs)
        {
            float *xb = live ? pb + (int64_t)rhs * ldb : nullptr;
            float x[RPL];
            if (trans == 0)
            {
#pragma unroll
                for (int s = 0; s < RPL; ++s)
                    x[s] = (live && lrow + s * SUBW < n) ? xb[src[s]] : 0.0f;
                // forward, unit lower
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                    if (k < n)
                    {
                        const float xk = __shfl_sync(0xffffffffu, x[k / SUBW], k % SUBW, SUBW);
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                            if (lrow + s * SUBW > k) x[s] = fma_rn(-a[s][k], xk, x[s]);
                    }
                }
                // backward, upper
#pragma unroll
                for (int k = N - 1; k >= 0; --k)
                {
                    if (k < n)
                    {
                        {
                            // the reciprocal does not depend on x: it is taken off the chain
                            const float d = a[k / SUBW][k];
                            const float y = div_prepare(d);
                            if (lrow == k % SUBW) x[k / SUBW] = div_by(x[k / SUBW], d, y, div_range(d));
                        }
                        const float xk = __shfl_sync(0xffffffffu, x[k / SUBW], k % SUBW, SUBW);
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                            if (lrow + s * SUBW < k) x[s] = fma_rn(-a[s][k], xk, x[s]);
                    }
                }
#pragma unroll
                for (int s = 0; s < RPL; ++s)
                    if (live && lrow + s * SUBW < n) xb[lrow + s * SUBW] = x[s];
            }
            else
            {
#pragma unroll
                for (int s = 0; s < RPL; ++s) x[s] = (live && lrow + s * SUBW < n) ? xb[lrow + s * SUBW] : 0.0f;
                // U^T w = b: lane i holds A(:, i) = column i; U(k,i) = a[.][k] on lane i.
#pragma unroll
                for (int k = 0; k < N; ++k)
                {
                    if (k < n)
                    {
                        {
                            // the reciprocal does not depend on x: it is taken off the chain
                            const float d = a[k / SUBW][k];
                            const float y = div_prepare(d);
                            if (lrow == k % SUBW) x[k / SUBW] = div_by(x[k / SUBW], d, y, div_range(d));
                        }
                        const float xk = __shfl_sync(0xffffffffu, x[k / SUBW], k % SUBW, SUBW);
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                            if (lrow + s * SUBW > k) x[s] = fma_rn(-a[s][k], xk, x[s]);
                    }
                }
                // L^T z = w: L(k, i) = a[.][k] on lane i.
#pragma unroll
                for (int k = N - 1; k >= 0; --k)
                {
                    if (k < n)
                    {
                        const float xk = __shfl_sync(0xffffffffu, x[k / SUBW], k % SUBW, SUBW);
#pragma unroll
                        for (int s = 0; s < RPL; ++s)
                            if (lrow + s * SUBW < k) x[s] = fma_rn(-a[s][k], xk, x[s]);
                    }
                }
                // x = P^T z: the row at position t goes back to src[t].
#pragma unroll
                for (int s = 0; s < RPL; ++s)
                    if (live && lrow + s * SUBW < n) xb[src[s]] = x[s];
            }
            __syncwarp();
        }
        if (in_batch && lrow == 0 && info)
            info[q] = (in_batch && !pa) ? -4 : (in_batch && !pb) ? -7 : bad_any ? -6 : 0;
    }
}

// ---------------------------------------------------------------------------------------
// getri
// ---------------------------------------------------------------------------------------
constexpr int RI_THREADS = 64;

template <int N>
__global__ void __launch_bounds__(RI_THREADS, 6) getri_small_kernel(float *a_single, float *const *a_table,
                                                                  int a_first, const int *ipiv, float *c_single,
                                                                  float *const *c_table, int c_first, int n, int lda,
                                                                  int ldc, int count, int *info)
{
    constexpr int MPC = RI_THREADS / N;  // matrices per block
    constexpr int LP = N;                // LU pitch (16-byte aligned columns)
    constexpr int SP = N + 1;            // output stage pitch
    constexpr int BUF = (N * SP + 3) & ~3;
    __shared__ __align__(16) float buf[MPC][BUF];
    __shared__ float rec[MPC][N];
    __shared__ int pv[MPC][N];
    __shared__ int zero_at[MPC];
    __shared__ int bad_pivot[MPC];
    const int t = threadIdx.x % N;
    const int m = threadIdx.x / N;
    float *lu = buf[m];

    for (int64_t base = (int64_t)blockIdx.x * MPC; base < count; base += (int64_t)gridDim.x * MPC)
    {
        const int64_t q = base + m;
        const bool in_batch = q < count;
        float *pa = nullptr, *pc = nullptr;
        if (in_batch)
        {
            pa = a_table ? slot(a_table, a_first + q) : a_single;
            pc = c_table ? slot(c_table, c_first + q) : c_single;
        }
        const bool live = pa != nullptr && pc != nullptr;
        __syncthreads();
        if (t == 0)
        {
            zero_at[m] = 0x7fffffff;
            bad_pivot[m] = 0;
        }
        {
            // row t of every column, in batches of up to 32 loads issued before their stores, so
            // a block waits for memory once or twice per matrix rather than once per column
            constexpr int LB = N < 32 ? N : 32;
            const float *src = live && t < n ? pa + t : nullptr;
#pragma unroll
            for (int j0 = 0; j0 < N; j0 += LB)
            {
                float v[LB];
#pragma unroll
                for (int j = 0; j < LB; ++j)
                    v[j] = (src && j0 + j < n) ? src[(int64_t)(j0 + j) * lda] : (t == j0 + j ? 1.0f : 0.0f);
#pragma unroll
                for (int j = 0; j < LB; ++j) lu[(j0 + j) * LP + t] = v[j];
            }
        }
        pv[m][t] = (live && ipiv && t < n) ? ipiv[q * n + t] : t + 1;
        __syncthreads();
        if (t < n)
        {
            const float u = lu[t * LP + t];
            rec[m][t] = div_rn(1.0f, u);
            if (u == 0.0f) atomicMin(&zero_at[m], t + 1);
            if (pv[m][t] < t + 1 || pv[m][t] > n) atomicOr(&bad_pivot[m], 1);
        }
        __syncthreads();
        // src: column of the inverse whose permuted unit vector has its 1 at row t.
        int col = t;
        if (!bad_pivot[m])
            for (int k = n - 1; k >= 0; --k)
            {
                const int pk = pv[m][k] - 1;
                col = col == k ? pk : (col == pk ? k : col);
            }
        const int failed = bad_pivot[m] ? -4 : (zero_at[m] == 0x7fffffff ? 0 : zero_at[m]);

        // the right-hand side in pairs of rows, r2[c] = (rhs[2c], rhs[2c + 1]); every update is
        // rhs_i = fma(-s, a_ik, rhs_i), two rows per paired FMA (lane by lane the same rounding)
        f32x2 r2[N / 2];
#pragma unroll
        for (int c = 0; c < N / 2; ++c) r2[c] = f2_pack(2 * c == t ? 1.0f : 0.0f, 2 * c + 1 == t ? 1.0f : 0.0f);
        const int kstart = (t / 32) * 32;  // warp-uniform: rows below the warp's first row are zero
        // forward, unit lower; the pivot row's partner row (k + 1 for even k) separately
#pragma unroll
        for (int k = 0; k < N; ++k)
        {
            if (k >= kstart && k < n)
            {
                const float s = (k & 1) ? f2_hi(r2[k / 2]) : f2_lo(r2[k / 2]);
                const f32x2 ns = f2_pack(-s, -s);
                if (!(k & 1) && k + 1 < N)
                    r2[k / 2] = f2_pack(s, fma_rn(-s, lu[k * LP + k + 1], f2_hi(r2[k / 2])));
#pragma unroll
                for (int c = k / 2 + 1; c < N / 2; ++c) fma2(r2[c], ns, *reinterpret_cast<const f32x2 *>(lu + k * LP + 2 * c));
            }
        }
        // backward, upper with reciprocal diagonal; the row above k in k's pair separately
#pragma unroll
        for (int k = N - 1; k >= 0; --k)
        {
            if (k < n)
            {
                const float s = mul_rn((k & 1) ? f2_hi(r2[k / 2]) : f2_lo(r2[k / 2]), rec[m][k]);
                const f32x2 ns = f2_pack(-s, -s);
                if (k & 1)
                    r2[k / 2] = f2_pack(fma_rn(-s, lu[k * LP + k - 1], f2_lo(r2[k / 2])), s);
                else
                    r2[k / 2] = f2_pack(s, f2_hi(r2[k / 2]));
#pragma unroll
                for (int c = 0; c < k / 2; ++c) fma2(r2[c], ns, *reinterpret_cast<const f32x2 *>(lu + k * LP + 2 * c));
            }
        }
        __syncthreads();
        float *stage = buf[m];
        if (t < n)
        {
#pragma unroll
            for (int c = 0; c < N / 2; ++c)
            {
                stage[col * SP + 2 * c] = f2_lo(r2[c]);
                stage[col * SP + 2 * c + 1] = f2_hi(r2[c]);
            }
        }
        __syncthreads();
        if (live && !failed)
        {
            for (int idx = t; idx < n * n; idx += N)
            {
                const int i = idx % n, j = idx / n;
                pc[i + (int64_t)j * ldc] = stage[j * SP + i];
            }
        }
        if (in_batch && t == 0) info[q] = live ? failed : -2;
    }
}

template <int N>
cudaError_t getrf_n(const RealBatch &a, int m, int *ipiv, int *info, cudaStream_t stream)
{
    constexpr int MPW = N < 32 ? 32 / N : 1;
    int64_t warps = (a.count + MPW - 1) / MPW;
    int64_t blocks = (warps * 32 + LU_THREADS - 1) / LU_THREADS;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    getrf_small_kernel<N><<<(unsigned)blocks, LU_THREADS, 0, stream>>>(a.single, a.table, a.first, m, a.n, a.ld,
                                                                       a.count, ipiv, info);
    return cudaGetLastError();
}

constexpr int GETRF_ROT_KB = 4;  // columns per rotation block of the order-64 factorisation

template <int KB>
cudaError_t getrf_rot(const RealBatch &a, int m, int *ipiv, int *info, cudaStream_t stream)
{
    const size_t smem = rot_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(getrf_rot_kernel<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int64_t blocks = (a.count * 32 + LU_THREADS - 1) / LU_THREADS;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    getrf_rot_kernel<KB><<<(unsigned)blocks, LU_THREADS, smem, stream>>>(a.single, a.table, a.first, m, a.n, a.ld,
                                                                        a.count, ipiv, info);
    return cudaGetLastError();
}

template <int N>
cudaError_t getrs_n(const RealBatch &a, const int *ipiv, const RealBatch &b, int nrhs, int trans, int *info,
                    cudaStream_t stream)
{
    constexpr int MPW = N < 32 ? 32 / N : 1;
    int64_t warps = (a.count + MPW - 1) / MPW;
    int64_t blocks = (warps * 32 + RS_THREADS - 1) / RS_THREADS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    if (trans == 0)
        getrs_small_kernel<N, 0><<<(unsigned)blocks, RS_THREADS, 0, stream>>>(
            a.single, a.table, a.first, ipiv, b.single, b.table, b.first, a.n, a.ld, b.ld, nrhs, a.count, info);
    else
        getrs_small_kernel<N, 1><<<(unsigned)blocks, RS_THREADS, 0, stream>>>(
            a.single, a.table, a.first, ipiv, b.single, b.table, b.first, a.n, a.ld, b.ld, nrhs, a.count, info);
    return cudaGetLastError();
}

template <int N>
cudaError_t getri_n(const RealBatch &a, const int *ipiv, const RealBatch &c, int *info, cudaStream_t stream)
{
    constexpr int MPC = RI_THREADS / N;
    int64_t blocks = (a.count + MPC - 1) / MPC;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    getri_small_kernel<N><<<(unsigned)blocks, RI_THREADS, 0, stream>>>(
        a.single, a.table, a.first, ipiv, c.single, c.table, c.first, a.n, a.ld, c.ld, a.count, info);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_getrf_small(const RealBatch &a, int m, int *ipiv, int *info, cudaStream_t stream)
{
    const int big = m > a.n ? m : a.n;
    if (big <= 8) return getrf_n<8>(a, m, ipiv, info, stream);
    if (big <= 16) return getrf_n<16>(a, m, ipiv, info, stream);
    if (big <= 32) return getrf_n<32>(a, m, ipiv, info, stream);
    return getrf_rot<GETRF_ROT_KB>(a, m, ipiv, info, stream);
}

cudaError_t launch_getrs_small(const RealBatch &a, const int *ipiv, const RealBatch &b, int nrhs, int trans,
                               int *info, cudaStream_t stream)
{
    if (a.n <= 8) return getrs_n<8>(a, ipiv, b, nrhs, trans, info, stream);
    if (a.n <= 16) return getrs_n<16>(a, ipiv, b, nrhs, trans, info, stream);
    if (a.n <= 32) return getrs_n<32>(a, ipiv, b, nrhs, trans, info, stream);
    return getrs_n<64>(a, ipiv, b, nrhs, trans, info, stream);
}

cudaError_t launch_getri_small(const RealBatch &a, const int *ipiv, const RealBatch &c, int *info,
                               cudaStream_t stream)
{
    if (a.n <= 8) return getri_n<8>(a, ipiv, c, info, stream);
    if (a.n <= 16) return getri_n<16>(a, ipiv, c, info, stream);
    if (a.n <= 32) return getri_n<32>(a, ipiv, c, info, stream);
    return getri_n<64>(a, ipiv, c, info, stream);
}

}  // namespace ops_solver
