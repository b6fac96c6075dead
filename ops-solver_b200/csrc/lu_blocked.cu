// lu_blocked.cu -- blocked right-looking LU for 64 < n <= 512, one block (256 threads) per
// matrix, plain FP32 or with the trailing update on the BF16 tensor cores.
//
// Per panel of NB = 32 columns (k0 = 0, 32, ...):
//  1. panel: rows k0..n-1 of columns k0..k0+w-1 are held in registers (thread t owns panel
//     rows t and t+256), factored with the reference's rules -- first-maximum |a| pivot with
//     the earliest position on ties and the NaN rule, IEEE division, FMA rank-1 updates --
//     with row interchanges kept as position labels (no data movement);
//  2. the panel is written back in its final row order and the permutation of rows k0..n-1
//     is applied to the other columns (left: the finished L; right: the trailing matrix);
//  3. U12 = L11^-1 A12 by column-oriented forward substitution, one thread per column;
//  4. A22 -= L21 U12, a 128 x 128 tile per block iteration.
// Plain mode: every trailing element takes a = fma(-l_ik, u_kj, a) in ascending k, the
// order of the unblocked reference (real_lu.hpp:345-368, FactorLocalCore :409-448), so the
// factors and pivots are bit-identical to the oracle's orc_sgetrf at every n.  (The
// reference itself switches to a reciprocal-multiply panel and a Cube GEMM at these sizes,
// real_lu_blocked_kernel.cpp:391-483, 1119-1158: parity with it is by residual.)
// Mixed modes: the trailing product is formed by mma.sync m16n8k16 BF16 with FP32
// accumulation from a 1-term (BF16) or 3-term (hi/lo split: hi*hi + hi*lo + lo*hi) split
// of L21 and U12; accuracy is then recovered by iterative refinement (refine.cu).
#include <cuda_bf16.h>

#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int BT = 256;  // threads per block
constexpr int NB = 32;   // panel width
constexpr int MAXN = 512;
constexpr int TILE = 128;

__device__ __forceinline__ unsigned block_max(unsigned v, unsigned *red)
{
    v = __reduce_max_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    unsigned r = red[0];
#pragma unroll
    for (int w = 1; w < BT / 32; ++w) r = max(r, red[w]);
    __syncthreads();
    return r;
}
__device__ __forceinline__ unsigned block_min(unsigned v, unsigned *red)
{
    v = __reduce_min_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    unsigned r = red[0];
#pragma unroll
    for (int w = 1; w < BT / 32; ++w) r = min(r, red[w]);
    __syncthreads();
    return r;
}

struct Shared
{
    float prow[NB];           // pivot row broadcast
    unsigned red[BT / 32];
    int perm[MAXN];           // perm[pos - k0] = physical panel row at that position
    int pos_of[MAXN];         // the inverse
    int changed[2 * NB];      // positions whose row changed
    int nchanged;
    unsigned zmask;           // bit j: panel column j had a zero pivot (not used for updates)
    int state;
};

// Panel factorisation; returns (through sh) the final position of each panel row.
__device__ void panel_factor(float *A, int lda, int n, int k0, int w, int *ipiv, Shared &sh, float (&r)[2][NB],
                             int (&pos)[2], int pivoting)
{
    const int t = threadIdx.x;
    const int m = n - k0;
    if (t == 0) sh.zmask = 0u;
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        const int i = t + s * BT;
        pos[s] = i;
#pragma unroll
        for (int c = 0; c < NB; ++c) r[s][c] = (i < m && c < w) ? A[(int64_t)(k0 + c) * lda + k0 + i] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < NB; ++j)
    {
        if (j < w && j < m)
        {
            int pr = j;
            if (pivoting)
            {
                unsigned key[2];
#pragma unroll
                for (int s = 0; s < 2; ++s)
                {
                    const float v = r[s][j];
                    key[s] = (pos[s] >= j && t + s * BT < m) ? pivot_key(v) : 0u;
                    if (pos[s] == j && v != v) key[s] = 0xffffffffu;
                }
                const unsigned mx = block_max(max(key[0], key[1]), sh.red);
                unsigned cand = 0xffffffffu;
#pragma unroll
                for (int s = 0; s < 2; ++s)
                    if (key[s] == mx) cand = min(cand, (unsigned)pos[s]);
                pr = (int)block_min(cand, sh.red);
#pragma unroll
                for (int s = 0; s < 2; ++s) pos[s] = pos[s] == j ? pr : (pos[s] == pr ? j : pos[s]);
                if (t == 0) ipiv[k0 + j] = k0 + pr + 1;
            }
            // broadcast the pivot row (now at position j)
#pragma unroll
            for (int s = 0; s < 2; ++s)
                if (pos[s] == j && t + s * BT < m)
                {
#pragma unroll
                    for (int c = 0; c < NB; ++c) sh.prow[c] = r[s][c];
                }
            __syncthreads();
            const float d = sh.prow[j];
            if (d == 0.0f && t == 0)
            {
                if (sh.state == 0) sh.state = k0 + j + 1;
                sh.zmask |= 1u << j;
            }
            if (d != 0.0f && k0 + j + 1 < n)
            {
#pragma unroll
                for (int s = 0; s < 2; ++s)
                {
                    if (pos[s] > j && t + s * BT < m)
                    {
                        const float l = div_rn(r[s][j], d);
                        r[s][j] = l;
#pragma unroll
                        for (int c = j + 1; c < NB; ++c) r[s][c] = fma_rn(-l, sh.prow[c], r[s][c]);
                    }
                }
            }
            __syncthreads();
        }
    }
    // final positions -> permutation tables
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        const int i = t + s * BT;
        if (i < m)
        {
            sh.perm[pos[s]] = i;
            sh.pos_of[i] = pos[s];
        }
    }
    __syncthreads();
    // write the panel back in final row order
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        const int i = t + s * BT;
        if (i < m)
        {
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (c < w) A[(int64_t)(k0 + c) * lda + k0 + pos[s]] = r[s][c];
        }
    }
    if (t == 0) sh.nchanged = 0;
    __syncthreads();
    // rows whose position changed (at most 2 * w)
    for (int p = t; p < m; p += BT)
        if (sh.perm[p] != p)
        {
            const int slot_i = atomicAdd(&sh.nchanged, 1);
            if (slot_i < 2 * NB) sh.changed[slot_i] = p;
        }
    __syncthreads();
}

// Apply the panel permutation to column j (rows k0..n-1) and, for trailing columns, the
// forward substitution with L11 (column-oriented, ascending k, FMA).
__device__ void update_column(float *A, int lda, int k0, int w, int j, bool trsm, const Shared &sh,
                              const float *panel_l)
{
    float *col = A + (int64_t)j * lda + k0;
    float top[NB];
    float moved[2 * NB];
    const int nc = sh.nchanged;
    // gather: old values of the rows landing at changed positions, and the top rows
#pragma unroll
    for (int c = 0; c < 2 * NB; ++c)
        if (c < nc) moved[c] = col[sh.perm[sh.changed[c]]];
#pragma unroll
    for (int i = 0; i < NB; ++i)
        if (i < w) top[i] = col[sh.perm[i]];
    // scatter the changed lower rows
#pragma unroll
    for (int c = 0; c < 2 * NB; ++c)
        if (c < nc && sh.changed[c] >= w) col[sh.changed[c]] = moved[c];
    if (trsm)
    {
        const unsigned zmask = sh.zmask;
#pragma unroll
        for (int k = 0; k < NB; ++k)
        {
            if (k < w && !((zmask >> k) & 1u))
            {
                const float u = top[k];
#pragma unroll
                for (int i = k + 1; i < NB; ++i)
                    if (i < w) top[i] = fma_rn(-panel_l[k * (MAXN + 1) + i], u, top[i]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i)
        if (i < w) col[i] = top[i];
}

// ----------------------------------------------------------------------------------------
// trailing update tiles
// ----------------------------------------------------------------------------------------
// L21 rows come from the staged panel (column-major, pitch MAXN + 1, rows relative to k0);
// U12 rows from the trailing columns (global, already solved).
__device__ void tile_plain(float *A, int lda, int n, int k0, int w, unsigned zmask, int r0, int c0,
                           const float *panel_l, float *us)
{
    const int t = threadIdx.x;
    const int tr = t % 16, tc = t / 16;
    const int lrow = r0 - k0 + tr * 8;
    // stage U12 (w x 128) for this tile's columns
    for (int e = t; e < NB * TILE; e += BT)
    {
        const int k = e / TILE, c = e % TILE;
        us[k * (TILE + 4) + c] = (k < w && c0 + c < n) ? A[(int64_t)(c0 + c) * lda + k0 + k] : 0.0f;
    }
    __syncthreads();
    float acc[8][8];
#pragma unroll
    for (int jj = 0; jj < 8; ++jj)
    {
        const int col = c0 + tc * 8 + jj;
#pragma unroll
        for (int ii = 0; ii < 8; ++ii)
        {
            const int row = r0 + tr * 8 + ii;
            acc[ii][jj] = (row < n && col < n) ? A[(int64_t)col * lda + row] : 0.0f;
        }
    }
#pragma unroll 4
    for (int k = 0; k < NB; ++k)
    {
        if (k < w && !((zmask >> k) & 1u))
        {
            float a[8], b[8];
#pragma unroll
            for (int ii = 0; ii < 8; ++ii) a[ii] = panel_l[k * (MAXN + 1) + min(lrow + ii, MAXN)];  // rows past n: unused
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) b[jj] = us[k * (TILE + 4) + tc * 8 + jj];
#pragma unroll
            for (int ii = 0; ii < 8; ++ii)
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) acc[ii][jj] = fma_rn(-a[ii], b[jj], acc[ii][jj]);
        }
    }
#pragma unroll
    for (int jj = 0; jj < 8; ++jj)
    {
        const int col = c0 + tc * 8 + jj;
#pragma unroll
        for (int ii = 0; ii < 8; ++ii)
        {
            const int row = r0 + tr * 8 + ii;
            if (row < n && col < n) A[(int64_t)col * lda + row] = acc[ii][jj];
        }
    }
    __syncthreads();
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Mixed tile: 8 warps, each a 32 x 64 sub-tile (2 x 8 mma tiles of 16 x 8), k = 32 in two
// k16 steps.  TERMS = 1: C -= bf16(L) bf16(U); TERMS = 3: hi/lo split, three products.
template <int TERMS>
__device__ void tile_mixed(float *A, int lda, int n, int k0, int w, unsigned zmask, int r0, int c0,
                           const float *panel_l, float *us)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int e = t; e < NB * TILE; e += BT)
    {
        const int k = e / TILE, c = e % TILE;
        us[k * (TILE + 4) + c] = (k < w && c0 + c < n) ? A[(int64_t)(c0 + c) * lda + k0 + k] : 0.0f;
    }
    __syncthreads();
    const int wr = r0 + (warp & 3) * 32;  // warp rows
    const int wc = c0 + (warp >> 2) * 64;  // warp cols
    const int g = lane >> 2, q = lane & 3;
    float acc[2][8][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 8; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e)
            {
                const int row = wr + mi * 16 + g + (e >= 2 ? 8 : 0);
                const int col = wc + ni * 8 + q * 2 + (e & 1);
                acc[mi][ni][e] = (row < n && col < n) ? A[(int64_t)col * lda + row] : 0.0f;
            }
#pragma unroll
    for (int ks = 0; ks < 2; ++ks)
    {
        const int kb = ks * 16;
        // A fragments (row-major 16 x 16): rows g, g+8; cols q*2, q*2+1, +8
        unsigned ah[2][4], al[2][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
        {
            float v[8];
            const int rr = wr - k0 + mi * 16 + g;
            const int kk = kb + q * 2;
            // negated L so that the accumulation subtracts; columns past w or with a zero
            // pivot contribute nothing
            const int ks[8] = {kk, kk + 1, kk, kk + 1, kk + 8, kk + 9, kk + 8, kk + 9};
#pragma unroll
            for (int e = 0; e < 8; ++e)
            {
                const bool use = ks[e] < w && !((zmask >> ks[e]) & 1u);
                v[e] = use ? -panel_l[ks[e] * (MAXN + 1) + min(rr + ((e & 2) ? 8 : 0), MAXN)] : 0.0f;  // rows past n: unused
            }
#pragma unroll
            for (int p = 0; p < 4; ++p)
            {
                ah[mi][p] = pack_bf16(v[2 * p], v[2 * p + 1]);
                if (TERMS > 1)
                {
                    const float h0 = __bfloat162float(__float2bfloat16_rn(v[2 * p]));
                    const float h1 = __bfloat162float(__float2bfloat16_rn(v[2 * p + 1]));
                    al[mi][p] = pack_bf16(v[2 * p] - h0, v[2 * p + 1] - h1);
                }
            }
        }
#pragma unroll
        for (int ni = 0; ni < 8; ++ni)
        {
            // B fragment (16 x 8, col-major): k = q*2, q*2+1 (+8), n = g
            const int cc = (wc - c0) + ni * 8 + g;
            const int kk = kb + q * 2;
            float u[4] = {us[(kk + 0) * (TILE + 4) + cc], us[(kk + 1) * (TILE + 4) + cc],
                          us[(kk + 8) * (TILE + 4) + cc], us[(kk + 9) * (TILE + 4) + cc]};
            unsigned bh[2] = {pack_bf16(u[0], u[1]), pack_bf16(u[2], u[3])};
            unsigned bl[2];
            if (TERMS > 1)
            {
                float h[4];
#pragma unroll
                for (int p = 0; p < 4; ++p) h[p] = __bfloat162float(__float2bfloat16_rn(u[p]));
                bl[0] = pack_bf16(u[0] - h[0], u[1] - h[1]);
                bl[1] = pack_bf16(u[2] - h[2], u[3] - h[3]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
            {
                if (TERMS > 1)
                {
                    mma_bf16(acc[mi][ni], al[mi], bh);
                    mma_bf16(acc[mi][ni], ah[mi], bl);
                }
                mma_bf16(acc[mi][ni], ah[mi], bh);
            }
        }
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 8; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e)
            {
                const int row = wr + mi * 16 + g + (e >= 2 ? 8 : 0);
                const int col = wc + ni * 8 + q * 2 + (e & 1);
                if (row < n && col < n) A[(int64_t)col * lda + row] = acc[mi][ni][e];
            }
    __syncthreads();
}

template <int MODE>  // 0 plain FP32, 1 BF16, 3 split BF16 (three products)
__global__ void __launch_bounds__(BT) getrf_blocked_kernel(float *single, float *const *table, int first, int n,
                                                            int lda, int *ipiv, int *info, int count)
{
    extern __shared__ float dyn[];
    float *panel_l = dyn;                          // NB x (MAXN + 1), column-major (rows rel. to k0)
    float *us = panel_l + NB * (MAXN + 1);         // NB x (TILE + 4)
    __shared__ Shared sh;
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        float *A = table ? slot(table, first + q) : single;
        if (!A)
        {
            if (threadIdx.x == 0) info[q] = -2;
            continue;
        }
        int *piv = ipiv ? ipiv + q * n : nullptr;
        if (threadIdx.x == 0) sh.state = 0;
        __syncthreads();
        for (int k0 = 0; k0 < n; k0 += NB)
        {
            const int w = min(NB, n - k0);
            float r[2][NB];
            int pos[2];
            panel_factor(A, lda, n, k0, w, piv, sh, r, pos, piv != nullptr);
            // stage L (rows k0..n-1 of the panel, final order) for TRSM and the update
#pragma unroll
            for (int s = 0; s < 2; ++s)
            {
                const int i = threadIdx.x + s * BT;
                if (i < n - k0)
                {
#pragma unroll
                    for (int c = 0; c < NB; ++c) panel_l[c * (MAXN + 1) + pos[s]] = r[s][c];
                }
            }
            __syncthreads();
            // permutation to the other columns, TRSM on the trailing ones
            for (int j = threadIdx.x; j < n; j += BT)
                if (j < k0 || j >= k0 + w) update_column(A, lda, k0, w, j, j >= k0 + w, sh, panel_l);
            __syncthreads();
            // trailing update
            const int start = k0 + w;
            for (int r0 = start; r0 < n; r0 += TILE)
                for (int c0 = start; c0 < n; c0 += TILE)
                {
                    if (MODE == 0)
                        tile_plain(A, lda, n, k0, w, sh.zmask, r0, c0, panel_l, us);
                    else
                        tile_mixed<MODE>(A, lda, n, k0, w, sh.zmask, r0, c0, panel_l, us);
                }
            __syncthreads();
        }
        if (threadIdx.x == 0) info[q] = sh.state;
        __syncthreads();
    }
}

}  // namespace

size_t getrf_blocked_smem() { return ((size_t)NB * (MAXN + 1) + (size_t)NB * (TILE + 4)) * sizeof(float); }

cudaError_t launch_getrf_blocked(const RealBatch &a, int *ipiv, int *info, int mode, cudaStream_t stream)
{
    const size_t smem = getrf_blocked_smem();
    int64_t blocks = a.count < 148 * 3 ? a.count : 148 * 3;
    if (blocks < 1) blocks = 1;
    switch (mode)
    {
        case 0:
            cudaFuncSetAttribute(getrf_blocked_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            getrf_blocked_kernel<0><<<(unsigned)blocks, BT, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld, ipiv, info,
                                                                             a.count);
            break;
        case 1:
            cudaFuncSetAttribute(getrf_blocked_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            getrf_blocked_kernel<1><<<(unsigned)blocks, BT, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld, ipiv, info,
                                                                             a.count);
            break;
        default:
            cudaFuncSetAttribute(getrf_blocked_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            getrf_blocked_kernel<3><<<(unsigned)blocks, BT, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld, ipiv, info,
                                                                             a.count);
            break;
    }
    return cudaGetLastError();
}

}  // namespace ops_solver
