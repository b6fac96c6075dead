// complex_block.cuh -- complex64 Cholesky factor and solve of one matrix of order n <= T per
// block of T threads, the lower triangle packed in shared memory (sm_100a).
//
// Arithmetic: the per-element order of orc_cpotrf / orc_cpotrs (oracle/oracle.c) and of the
// other complex kernels -- every a_ij takes its updates a_ij -= l_ik conj(l_jk) as four FMAs
// in ascending k, then (below the diagonal) the IEEE division of each component by
// s = sqrt(Re a_jj); the solves take their right-looking updates in ascending (forward) or
// descending (backward) k before their division.  Only the schedule differs from a plain
// right-looking loop, and no element sees its operations in another order:
//   factor, left-looking in blocks of CB = 16 columns: thread t owns row J0 + t of block
//   column J0 (in registers) and first applies every earlier column k < J0 to it (the
//   block's sixteen L(J0 + j, k) are broadcast loads; a thread's row value L(i, k) is its own
//   load), then the sixteen panel steps run with one barrier each (the column's L values
//   for the block rows go through a double-buffered shared slot; every thread keeps the
//   block's diagonal real parts, so the square roots need no second exchange);
//   solve, blocked by 16 rows: the warp owning a block's rows solves its triangle by
//   shuffles, the block's solution values are published once, and every other row applies
//   the block's sixteen updates in order.
// Shared memory: the lower triangle packed by columns (column j holds rows j..n-1), plus a
// 16-element tail so the broadcast loads of a ragged last block stay inside the buffer, plus
// small exchange slots.  cb_smem_bytes(n) gives the size; n = 128 takes 66 KB, so three
// blocks share an SM.
#pragma once
#include "common.cuh"

namespace ops_solver
{
constexpr int CB = 16;               // columns per block, rows per solve block
constexpr int CB_RHS = 4;            // right-hand sides solved together
constexpr float CB_FLT_MAX = 3.402823466e38F;

__host__ __device__ constexpr int cb_tri(int n) { return n * (n + 1) / 2; }
// floats of shared memory: packed triangle + tail, two column slots, block diagonal, solve
// exchange (two buffers of CB rows x CB_RHS complex)
__host__ __device__ constexpr size_t cb_smem_bytes(int n)
{
    return ((size_t)(cb_tri(n) + CB) * 2 + 2 * CB * 2 + CB + 2 * CB * CB_RHS * 2) * sizeof(float);
}
// packed offset of column j (rows j..n-1)
__device__ __forceinline__ int cb_col(int j, int n) { return j * n - (j * (j - 1)) / 2; }

struct CbShared
{
    float2 *tri;    // packed lower triangle
    float2 *slot;   // [2][CB] column exchange
    float *diag;    // [CB] block diagonal real parts
    float2 *ybuf;   // [2][CB][CB_RHS] solve exchange
};

__device__ __forceinline__ CbShared cb_carve(float *base, int n)
{
    CbShared s;
    s.tri = reinterpret_cast<float2 *>(base);
    s.slot = s.tri + cb_tri(n) + CB;
    s.diag = reinterpret_cast<float *>(s.slot + 2 * CB);
    s.ybuf = reinterpret_cast<float2 *>(s.diag + CB + (CB & 1));
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

// Factor the packed triangle in place.  Returns info (0, or the first failed column + 1),
// the same on every thread.  Columns before a failure are final in shared memory.
template <int T>
__device__ int cb_factor(const CbShared &s, int n)
{
    const int t = threadIdx.x;
    for (int J0 = 0; J0 < n; J0 += CB)
    {
        const int w = min(CB, n - J0);
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
        // every earlier column, ascending k
        if (own)
        {
            int ok = 0;  // packed offset of column k
            for (int k = 0; k < J0; ++k)
            {
                const float2 a = s.tri[ok + i - k];
                const float2 *c = s.tri + ok + J0 - k;
#pragma unroll
                for (int j = 0; j < CB; ++j)
                {
                    const float2 cj = c[j];
                    cb_sub_lconj(zr[j], zi[j], a.x, a.y, cj.x, cj.y);
                }
                ok += n - k;
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
                    else if (i > k)
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
// Rows are owned by threads (row t), CB_RHS right-hand sides at a time.
template <int T>
__device__ void cb_solve(const CbShared &s, int n, float2 *pb, int ldb, int nrhs)
{
    const int t = threadIdx.x, warp = t >> 5;
    const int i = t;
    const bool own = i < n;
    const int nblk = (n + CB - 1) / CB;
    for (int r0 = 0; r0 < nrhs; r0 += CB_RHS)
    {
        const int nr = min(CB_RHS, nrhs - r0);
        float zr[CB_RHS], zi[CB_RHS];
#pragma unroll
        for (int r = 0; r < CB_RHS; ++r)
        {
            zr[r] = 0.0f;
            zi[r] = 0.0f;
            if (own && r < nr)
            {
                const float2 v = pb[(int64_t)(r0 + r) * ldb + i];
                zr[r] = v.x;
                zi[r] = v.y;
            }
        }
        // forward: y_k = z_k / l_kk, z_i -= l_ik y_k for i > k
        for (int b = 0; b < nblk; ++b)
        {
            const int J0 = b * CB, w = min(CB, n - J0);
            float2 *yb = s.ybuf + (b & 1) * CB * CB_RHS;
            if (warp == J0 / 32)
            {
#pragma unroll
                for (int kk = 0; kk < CB; ++kk)
                {
                    if (kk < w)
                    {
                        const int k = J0 + kk;
                        const float d = s.tri[cb_col(k, n)].x;
                        const float yv = div_prepare(d);
                        const bool okd = div_range(d);
                        const int src = k & 31;
                        float lr = 0.0f, li = 0.0f;
                        if (i > k && i < J0 + w)
                        {
                            const float2 l = s.tri[cb_col(k, n) + i - k];
                            lr = l.x;
                            li = l.y;
                        }
#pragma unroll
                        for (int r = 0; r < CB_RHS; ++r)
                        {
                            const float qr = __shfl_sync(0xffffffffu, div_by(zr[r], d, yv, okd), src);
                            const float qi = __shfl_sync(0xffffffffu, div_by(zi[r], d, yv, okd), src);
                            if (i == k)
                            {
                                zr[r] = qr;
                                zi[r] = qi;
                            }
                            else if (i > k && i < J0 + w)
                                cb_sub_prod(zr[r], zi[r], lr, li, qr, qi);
                        }
                    }
                }
                if (i >= J0 && i < J0 + w)
                {
#pragma unroll
                    for (int r = 0; r < CB_RHS; ++r) yb[(i - J0) * CB_RHS + r] = make_float2(zr[r], zi[r]);
                }
            }
            __syncthreads();
            if (own && i >= J0 + w)
            {
                for (int kk = 0; kk < w; ++kk)
                {
                    const int k = J0 + kk;
                    const float2 l = s.tri[cb_col(k, n) + i - k];
#pragma unroll
                    for (int r = 0; r < CB_RHS; ++r)
                    {
                        const float2 y = yb[kk * CB_RHS + r];
                        cb_sub_prod(zr[r], zi[r], l.x, l.y, y.x, y.y);
                    }
                }
            }
        }
        // backward: x_k = z_k / l_kk, z_i -= conj(l_ki) x_k for i < k, k descending.  The
        // exchange slots alternate by block, so one barrier per block suffices once the
        // forward sweep's last readers are done.
        __syncthreads();
        for (int b = nblk - 1; b >= 0; --b)
        {
            const int J0 = b * CB, w = min(CB, n - J0);
            float2 *yb = s.ybuf + (b & 1) * CB * CB_RHS;
            if (warp == J0 / 32)
            {
#pragma unroll
                for (int kk = CB - 1; kk >= 0; --kk)
                {
                    if (kk < w)
                    {
                        const int k = J0 + kk;
                        const float d = s.tri[cb_col(k, n)].x;
                        const float yv = div_prepare(d);
                        const bool okd = div_range(d);
                        const int src = k & 31;
                        float lr = 0.0f, li = 0.0f;
                        if (i < k && i >= J0)
                        {
                            const float2 l = s.tri[cb_col(i, n) + k - i];  // L(k, i)
                            lr = l.x;
                            li = -l.y;  // conj
                        }
#pragma unroll
                        for (int r = 0; r < CB_RHS; ++r)
                        {
                            const float qr = __shfl_sync(0xffffffffu, div_by(zr[r], d, yv, okd), src);
                            const float qi = __shfl_sync(0xffffffffu, div_by(zi[r], d, yv, okd), src);
                            if (i == k)
                            {
                                zr[r] = qr;
                                zi[r] = qi;
                            }
                            else if (i < k && i >= J0)
                                cb_sub_prod(zr[r], zi[r], lr, li, qr, qi);
                        }
                    }
                }
                if (i >= J0 && i < J0 + w)
                {
#pragma unroll
                    for (int r = 0; r < CB_RHS; ++r) yb[(i - J0) * CB_RHS + r] = make_float2(zr[r], zi[r]);
                }
            }
            __syncthreads();
            if (i < J0)
            {
                const float2 *col = s.tri + cb_col(i, n) - i;  // col[k] = L(k, i)
                for (int kk = w - 1; kk >= 0; --kk)
                {
                    const int k = J0 + kk;
                    const float2 l = col[k];
#pragma unroll
                    for (int r = 0; r < CB_RHS; ++r)
                    {
                        const float2 x = yb[kk * CB_RHS + r];
                        cb_sub_prod(zr[r], zi[r], l.x, -l.y, x.x, x.y);
                    }
                }
            }
        }
        if (own)
        {
#pragma unroll
            for (int r = 0; r < CB_RHS; ++r)
                if (r < nr) pb[(int64_t)(r0 + r) * ldb + i] = make_float2(zr[r], zi[r]);
        }
        __syncthreads();  // the exchange slots are free for the next group
    }
}

}  // namespace ops_solver
