// complex_block.cuh -- complex64 Cholesky factor and solve of one matrix of order n <= T per
// block of T threads, the lower triangle packed in shared memory (sm_100a).
//
// Arithmetic: the per-element order of orc_cpotrf / orc_cpotrs (oracle/oracle.c) and of the
// other complex kernels -- every a_ij takes its updates a_ij -= l_ik conj(l_jk) as four FMAs
// in ascending k, then (below the diagonal) the IEEE division of each component by
// s = sqrt(Re a_jj); the solves take their right-looking updates in ascending (forward) or
// descending (backward) k before their division.  Only the schedule differs from a plain
// right-looking loop, and no element sees its operations in another order:
//   factor, left-looking in blocks of CB = 16 columns: every earlier column k < J0 is first
//   applied to block column J0 in shared memory, 16 / C threads per remaining row with C
//   adjacent columns each (the row's L(i, k) is a thread's own load, the block's L(J0 + j, k)
//   broadcast loads); then thread t takes row J0 + t into registers and the sixteen panel
//   steps run with one barrier each (the column's L values for the block rows go through a
//   double-buffered shared slot; every thread keeps the block's diagonal real parts, so the
//   square roots need no second exchange);
//   solve, a warp per right-hand side (or per group of them) with no block barrier: the
//   owner lane of row k divides, one shuffle per component broadcasts the quotient, and
//   every lane updates its rows from the packed triangle.
// Shared memory: the lower triangle packed by columns (column j holds rows j..n-1), plus a
// 16-element tail so the broadcast loads of a ragged last block stay inside the buffer, plus
// small exchange slots.  cb_smem_bytes(n) gives the size; n = 128 takes 66 KB, so three
// blocks share an SM.
#pragma once
#include "common.cuh"

namespace ops_solver
{
constexpr int CB = 16;               // columns per factor block
constexpr int CB_RHS = 4;            // right-hand sides a block keeps in flight in the solve
constexpr float CB_FLT_MAX = 3.402823466e38F;

__host__ __device__ constexpr int cb_tri(int n) { return n * (n + 1) / 2; }
// floats of shared memory: packed triangle + tail, two column slots, block diagonal
__host__ __device__ constexpr size_t cb_smem_bytes(int n)
{
    return ((size_t)(cb_tri(n) + CB) * 2 + 2 * CB * 2 + CB) * sizeof(float);
}
// packed offset of column j (rows j..n-1)
__device__ __forceinline__ int cb_col(int j, int n) { return j * n - (j * (j - 1)) / 2; }

struct CbShared
{
    float2 *tri;    // packed lower triangle
    float2 *slot;   // [2][CB] column exchange
    float *diag;    // [CB] block diagonal real parts
};

__device__ __forceinline__ CbShared cb_carve(float *base, int n)
{
    CbShared s;
    s.tri = reinterpret_cast<float2 *>(base);
    s.slot = s.tri + cb_tri(n) + CB;
    s.diag = reinterpret_cast<float *>(s.slot + 2 * CB);
    return s;
}

// z -= l * conj(c), the factor's update
__device__ __forceinline__ void cb_sub_lconj(float &re, float &im, float ar, float ai, float cr, float ci)
{
    re = fma_rn(-ar, cr, re);
    re = fma_rn(-ai, ci, re);
    im = fma_rn(-ai, cr, im);
    im = fma_rn(ar, ci, im);
}
// z -= l * y, the solves' update
__device__ __forceinline__ void cb_sub_prod(float &re, float &im, float ar, float ai, float yr, float yi)
{
    re = fma_rn(-ar, yr, re);
    re = fma_rn(ai, yi, re);
    im = fma_rn(-ar, yi, im);
    im = fma_rn(-ai, yr, im);
}

// Global lower (or conjugated upper) triangle -> packed shared triangle.  Thread t takes
// row t of every column (n <= T), eight columns' loads in flight before their stores; lower
// storage reads each column row-contiguous (coalesced).
template <int T>
__device__ __forceinline__ void cb_load(const CbShared &s, const float2 *pa, int lda, int upper, int n)
{
    const int i = threadIdx.x;
    for (int j0 = 0; j0 < n; j0 += 8)
    {
        float2 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
        {
            const int j = j0 + u;
            v[u] = make_float2(0.0f, 0.0f);
            if (j <= i && i < n)
            {
                if (upper)
                {
                    const float2 w = pa[(int64_t)i * lda + j];
                    v[u] = make_float2(w.x, -w.y);
                }
                else
                    v[u] = pa[(int64_t)j * lda + i];
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
        {
            const int j = j0 + u;
            if (j <= i && i < n) s.tri[cb_col(j, n) + i - j] = v[u];
        }
    }
}

// Packed shared triangle -> global, columns 0..done-1 only (a failed matrix keeps the rest).
template <int T>
__device__ __forceinline__ void cb_store(const CbShared &s, float2 *pa, int lda, int upper, int n, int done)
{
    const int i = threadIdx.x;
    if (i >= n) return;
    for (int j = 0; j < done && j <= i; ++j)
    {
        const float2 v = s.tri[cb_col(j, n) + i - j];
        if (upper)
            pa[(int64_t)i * lda + j] = make_float2(v.x, -v.y);
        else
            pa[(int64_t)j * lda + i] = v;
    }
}

// The left-looking update of block column J0 (rows J0..n-1, its w columns) by every earlier
// column k < J0, in shared memory: G = CB / C threads share a row, each taking C adjacent
// columns of it, so that the whole block works however few rows remain below J0 (the rows
// shrink from n to 16 over the factorisation; one thread per row left most of the block
// waiting at the next barrier).  Every element still takes its updates one after another in
// ascending k, from one thread.
template <int C>
__device__ __forceinline__ void cb_left(const CbShared &s, int n, int J0, int w)
{
    constexpr int G = CB / C;
    const int t = threadIdx.x;
    const int i = J0 + t / G;    // row
    const int j0 = (t % G) * C;  // first column of this thread within the block
    if (i >= n) return;
    float zr[C], zi[C];
#pragma unroll
    for (int u = 0; u < C; ++u)
    {
        const int j = j0 + u;
        zr[u] = 0.0f;
        zi[u] = 0.0f;
        if (j < w && J0 + j <= i)
        {
            const float2 v = s.tri[cb_col(J0 + j, n) + i - (J0 + j)];
            zr[u] = v.x;
            zi[u] = v.y;
        }
    }
    int ok = 0;  // packed offset of column k
    for (int k = 0; k < J0; ++k)
    {
        const float2 a = s.tri[ok + i - k];
        const float2 *c = s.tri + ok + J0 - k + j0;  // c[u] = L(J0 + j0 + u, k)
#pragma unroll
        for (int u = 0; u < C; ++u)
        {
            const float2 cj = c[u];
            cb_sub_lconj(zr[u], zi[u], a.x, a.y, cj.x, cj.y);
        }
        ok += n - k;
    }
#pragma unroll
    for (int u = 0; u < C; ++u)
    {
        const int j = j0 + u;
        if (j < w && J0 + j <= i) s.tri[cb_col(J0 + j, n) + i - (J0 + j)] = make_float2(zr[u], zi[u]);
    }
}

// Factor the packed triangle in place.  Returns info (0, or the first failed column + 1),
// the same on every thread.  Columns before a failure are final in shared memory.
template <int T>
__device__ __forceinline__ int cb_factor(const CbShared &s, int n)
{
    const int t = threadIdx.x;
    for (int J0 = 0; J0 < n; J0 += CB)
    {
        const int w = min(CB, n - J0);
        if (J0 > 0)
        {
            // threads per row: the most that fit the rows left (uniform over the block)
            const int rows = n - J0;
            if (rows > T / 2)
                cb_left<16>(s, n, J0, w);
            else if (rows > T / 4)
                cb_left<8>(s, n, J0, w);
            else if (rows > T / 8)
                cb_left<4>(s, n, J0, w);
            else if (rows > T / 16)
                cb_left<2>(s, n, J0, w);
            else
                cb_left<1>(s, n, J0, w);
            __syncthreads();
        }
        const int i = J0 + t;  // this thread's row
        const bool own = i < n;
        float zr[CB], zi[CB];
        // the block column's current values (the upper part of the diagonal block and the
        // columns past a ragged end take junk that is never stored)
#pragma unroll
        for (int j = 0; j < CB; ++j)
        {
            zr[j] = 0.0f;
            zi[j] = 0.0f;
            if (own && j < w && J0 + j <= i)
            {
                const float2 v = s.tri[cb_col(J0 + j, n) + i - (J0 + j)];
                zr[j] = v.x;
                zi[j] = v.y;
            }
        }
        // the block's diagonal real parts to every thread
        if (t < w)
        {
            float dv = 0.0f;
#pragma unroll
            for (int j = 0; j < CB; ++j)
                if (j == t) dv = zr[j];
            s.diag[t] = dv;
        }
        __syncthreads();
        float dre[CB];
#pragma unroll
        for (int j = 0; j < CB; ++j) dre[j] = j < w ? s.diag[j] : 1.0f;
        int failure = 0;
#pragma unroll
        for (int kk = 0; kk < CB; ++kk)
        {
            if (kk < w && failure == 0)
            {
                const int k = J0 + kk;
                const float d = dre[kk];
                if (!(d > 0.0f && d <= CB_FLT_MAX))
                    failure = k + 1;
                else
                {
                    const float sq = sqrt_rn(d);
                    const float y = div_prepare(sq);
                    const bool ok = div_range(sq);
                    float lr = zr[kk], li = zi[kk];
                    if (i == k)
                    {
                        lr = sq;
                        li = 0.0f;
                    }
                    else if (i > k && own)  // rows past n would take the slow division on junk
                    {
                        lr = div_by(lr, sq, y, ok);
                        li = div_by(li, sq, y, ok);
                    }
                    zr[kk] = lr;
                    zi[kk] = li;
                    float2 *slot = s.slot + (kk & 1) * CB;
                    if (t < w) slot[t] = make_float2(lr, li);
                    __syncthreads();
#pragma unroll
                    for (int j = kk + 1; j < CB; ++j)
                    {
                        if (j < w)
                        {
                            const float2 c = slot[j];
                            if (own && i >= J0 + j) cb_sub_lconj(zr[j], zi[j], lr, li, c.x, c.y);
                            dre[j] = fma_rn(-c.y, c.y, fma_rn(-c.x, c.x, dre[j]));
                        }
                    }
                }
            }
        }
        // the block column's finished values (before a failure: its completed columns)
        const int wdone = failure ? failure - 1 - J0 : w;
        if (own)
        {
#pragma unroll
            for (int j = 0; j < CB; ++j)
                if (j < wdone && J0 + j <= i) s.tri[cb_col(J0 + j, n) + i - (J0 + j)] = make_float2(zr[j], zi[j]);
        }
        __syncthreads();
        if (failure) return failure;
    }
    return 0;
}

// Solve L L^H X = B for nrhs columns of B (global, ldb) with the factor in shared memory.
// Each warp solves its own right-hand sides (T / 32 warps; up to four right-hand sides in
// flight per warp when the block has fewer than four warps) with no block barrier: lane l
// keeps rows l, l + 32, ... in registers; step k divides row k on its owner lane (the
// lane's own diagonal entries and their reciprocals are taken once, ahead of both sweeps,
// and every other lane divides 1 by its own diagonal so that no lane leaves the fast
// division), broadcasts the quotient with one shuffle per component, and every row below
// (forward) or above (backward) takes its update from the packed triangle.  Each element
// receives its updates in ascending (forward) or descending (backward) k, as before.
template <int T>
__device__ __forceinline__ void cb_solve(const CbShared &s, int n, float2 *pb, int ldb, int nrhs)
{
    constexpr int NW = T / 32;                    // warps
    constexpr int M = T / 32;                     // rows per lane (n <= T)
    constexpr int RW = NW >= CB_RHS ? 1 : CB_RHS / NW;  // right-hand sides per warp in flight
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float dd[M], rd[M];
    bool dk[M];
#pragma unroll
    for (int m = 0; m < M; ++m)
    {
        const int row = lane + 32 * m;
        dd[m] = row < n ? s.tri[cb_col(row, n)].x : 1.0f;
        rd[m] = div_prepare(dd[m]);
        dk[m] = div_range(dd[m]);
    }
    for (int r0 = warp * RW; r0 < nrhs; r0 += NW * RW)
    {
        // rows past n hold 1 (never stored), so their junk divisions stay on the fast path
        float zr[RW][M], zi[RW][M];
#pragma unroll
        for (int u = 0; u < RW; ++u)
#pragma unroll
            for (int m = 0; m < M; ++m)
            {
                const int row = lane + 32 * m;
                zr[u][m] = 1.0f;
                zi[u][m] = 1.0f;
                if (r0 + u < nrhs && row < n)
                {
                    const float2 v = pb[(int64_t)(r0 + u) * ldb + row];
                    zr[u][m] = v.x;
                    zi[u][m] = v.y;
                }
            }
        // forward: y_k = z_k / l_kk, z_i -= l_ik y_k for i > k, k ascending
#pragma unroll
        for (int m = 0; m < M; ++m)
        {
#pragma unroll 2
            for (int k0 = 0; k0 < 32; ++k0)
            {
                const int k = 32 * m + k0;
                if (k >= n) break;
                const float2 *col = s.tri + cb_col(k, n) - k;  // col[i] = L(i, k)
                float qr[RW], qi[RW];
#pragma unroll
                for (int u = 0; u < RW; ++u)
                {
                    const float nr = lane == k0 ? zr[u][m] : 1.0f, ni = lane == k0 ? zi[u][m] : 1.0f;
                    qr[u] = __shfl_sync(0xffffffffu, div_by(nr, dd[m], rd[m], dk[m]), k0);
                    qi[u] = __shfl_sync(0xffffffffu, div_by(ni, dd[m], rd[m], dk[m]), k0);
                    if (lane == k0)
                    {
                        zr[u][m] = qr[u];
                        zi[u][m] = qi[u];
                    }
                }
#pragma unroll
                for (int mm = m; mm < M; ++mm)
                {
                    const int row = lane + 32 * mm;
                    if (row > k && row < n)
                    {
                        const float2 l = col[row];
#pragma unroll
                        for (int u = 0; u < RW; ++u) cb_sub_prod(zr[u][mm], zi[u][mm], l.x, l.y, qr[u], qi[u]);
                    }
                }
            }
        }
        // backward: x_k = z_k / l_kk, z_i -= conj(l_ki) x_k for i < k, k descending
#pragma unroll
        for (int m = M - 1; m >= 0; --m)
        {
#pragma unroll 2
            for (int k0 = 31; k0 >= 0; --k0)
            {
                const int k = 32 * m + k0;
                if (k >= n) continue;
                float qr[RW], qi[RW];
#pragma unroll
                for (int u = 0; u < RW; ++u)
                {
                    const float nr = lane == k0 ? zr[u][m] : 1.0f, ni = lane == k0 ? zi[u][m] : 1.0f;
                    qr[u] = __shfl_sync(0xffffffffu, div_by(nr, dd[m], rd[m], dk[m]), k0);
                    qi[u] = __shfl_sync(0xffffffffu, div_by(ni, dd[m], rd[m], dk[m]), k0);
                    if (lane == k0)
                    {
                        zr[u][m] = qr[u];
                        zi[u][m] = qi[u];
                    }
                }
#pragma unroll
                for (int mm = 0; mm <= m; ++mm)
                {
                    const int row = lane + 32 * mm;
                    if (row < k)
                    {
                        const float2 l = s.tri[cb_col(row, n) + k - row];  // L(k, row)
#pragma unroll
                        for (int u = 0; u < RW; ++u) cb_sub_prod(zr[u][mm], zi[u][mm], l.x, -l.y, qr[u], qi[u]);
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < RW; ++u)
#pragma unroll
            for (int m = 0; m < M; ++m)
            {
                const int row = lane + 32 * m;
                if (r0 + u < nrhs && row < n) pb[(int64_t)(r0 + u) * ldb + row] = make_float2(zr[u][m], zi[u][m]);
            }
    }
}

}  // namespace ops_solver
