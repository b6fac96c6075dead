// lu_blocked.cu -- blocked right-looking LU for 64 < n <= 512, one 256-thread block per
// matrix (two resident per SM), plain FP32 or with the trailing update on the BF16 tensor
// cores.
//
// Per panel of NB = 32 columns (k0 = 0, 32, ...):
//  1. panel: rows k0..n-1 of the panel columns sit in registers (thread t owns panel rows t
//     and t + 256) and are factored with the reference's rules -- first-maximum |a| pivot,
//     earliest position on ties, the NaN rule, IEEE division, FMA rank-1 updates.  Rows are
//     never moved while the panel is factored: each carries its current position, and the
//     pivot search is one barrier per column (warp redux of an order-preserving |a| key and
//     of the position, then the eight warp winners through double-buffered shared slots that
//     also carry the winning row, so the pivot row needs no second broadcast);
//  2. the panel goes back to global memory in its final row order and its L is staged in
//     shared memory (FP32, or negated BF16 hi/lo for the tensor cores);
//  3. the trailing columns go in tiles of 64: a warp per column gathers the 32 U12 rows
//     through the panel permutation and moves the rows whose position changed (coalesced
//     column segments), U12 = L11^-1 A12 is solved in shared memory by four threads per
//     column, and A22 -= L21 U12 runs over 128-row tiles;
//  4. after the last panel, the row interchanges of every later panel are applied to each
//     panel's L columns in one gather per column (LAPACK's final row order).
// Plain mode: every element takes a = fma(-l_ik, u_kj, a) in ascending k, the order of the
// unblocked reference (real_lu.hpp:345-368, FactorLocalCore :409-448), so factors, pivots and
// info are bit-identical to the oracle's orc_sgetrf at every n.  (The reference itself
// switches to a reciprocal-multiply panel and a Cube GEMM at these sizes,
// real_lu_blocked_kernel.cpp:391-483, 1119-1158: parity with it is by residual.)
// Mixed modes: the trailing product is formed by mma.sync m16n8k16 BF16 with FP32
// accumulation from a one-term (BF16) or three-term split (hi*hi + hi*lo + lo*hi) of L21 and
// U12; accuracy is recovered by iterative refinement.
#include <cuda_bf16.h>

#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int BT = 256;  // threads per block
constexpr int NW = BT / 32;
constexpr int NB = 32;   // panel width
constexpr int MAXN = BLOCKED_MAX_N;
constexpr int CT = 64;   // trailing column tile
constexpr int RT = 128;  // trailing row tile
constexpr int UP = CT + 4;  // pitch of the FP32 U12 tile
constexpr int HP = NB + 8;  // pitch (halfs) of the BF16 tiles: 80 bytes, ldmatrix conflict-free
constexpr unsigned FULL = 0xffffffffu;

struct __align__(16) Shared
{
    float slot[2][NW][NB];     // each warp's best pivot row, double buffered by column parity
    unsigned key[2][NW][2];    // each warp's (best key, its position)
    short perm[MAXN];          // perm[p]: panel-relative row now at panel position p
    short tmap[MAXN];          // left-column permutation (epilogue)
    short umap[MAXN];
    int changed[2 * NB];       // panel positions whose row changed
    int nchanged;
    unsigned zmask;            // bit j: panel column j had a zero pivot (not used for updates)
    int state;                 // info of the matrix
};

// Staged rows per panel: the trailing tiles start at position NB and cover RT rows each, so
// the last tile reads up to NB + round_up(m - NB, RT) - 1 < round_up(n, RT) + NB.
__host__ __device__ constexpr int round_rows(int n) { return (n + RT - 1) / RT * RT + NB; }

// Dynamic shared memory (bytes) for order n.
//   plain: L (NB x LP floats, L[k][p]), U12 tile (NB x UP floats)
//   mixed: L11 (NB x (NB + 4) floats), U12 tile, L21 hi/lo (rows x HP bf16), U12 hi/lo (CT x HP)
__host__ __device__ constexpr size_t lp_pitch(int n) { return (size_t)round_rows(n) + 4; }
__host__ __device__ size_t dyn_bytes(int n, int mode)
{
    if (mode == 0) return ((size_t)NB * lp_pitch(n) + (size_t)NB * UP) * sizeof(float);
    const int terms = mode == 1 ? 1 : 2;
    return ((size_t)NB * (NB + 4) + (size_t)NB * UP) * sizeof(float) +
           (size_t)terms * ((size_t)round_rows(n) * HP + (size_t)CT * HP) * sizeof(__nv_bfloat16);
}

// ---------------------------------------------------------------------------------------
// panel
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void panel_factor(float *A, int lda, int n, int k0, int w, int *ipiv, bool pivoting,
                                             Shared &sh, float (&r)[2][NB], int (&pos)[2])
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int m = n - k0;
    bool valid[2];
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        const int i = t + s * BT;
        valid[s] = i < m;
        pos[s] = i;
#pragma unroll
        for (int c = 0; c < NB; ++c) r[s][c] = (valid[s] && c < w) ? A[(int64_t)(k0 + c) * lda + k0 + i] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < NB; ++j)
    {
        if (j >= w) break;  // uniform
        const int buf = j & 1;
        unsigned key[2];
#pragma unroll
        for (int s = 0; s < 2; ++s)
        {
            const float v = r[s][j];
            if (!valid[s])
                key[s] = 0u;
            else if (pivoting)
                key[s] = pos[s] == j && v != v ? 0xffffffffu : (pos[s] >= j ? pivot_key(v) : 0u);
            else
                key[s] = pos[s] == j ? 1u : 0u;
        }
        const unsigned wmax = __reduce_max_sync(FULL, max(key[0], key[1]));
        unsigned cand = 0xffffffffu;
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (valid[s] && key[s] == wmax) cand = min(cand, (unsigned)pos[s]);
        const unsigned wpos = __reduce_min_sync(FULL, cand);
#pragma unroll
        for (int s = 0; s < 2; ++s)
            if (valid[s] && key[s] == wmax && (unsigned)pos[s] == wpos)
            {
                float4 *dst = reinterpret_cast<float4 *>(sh.slot[buf][warp]);
#pragma unroll
                for (int c = 0; c < NB; c += 4) dst[c / 4] = make_float4(r[s][c], r[s][c + 1], r[s][c + 2], r[s][c + 3]);
            }
        if (lane == 0)
        {
            sh.key[buf][warp][0] = wmax;
            sh.key[buf][warp][1] = wpos;
        }
        __syncthreads();
        // the block's winner: largest key, then the smallest position (a warp without
        // candidates reports key 0 and always loses: the position-j row has key >= 1)
        unsigned gmax = 0u, gpos = 0xffffffffu;
        int gw = 0;
#pragma unroll
        for (int q = 0; q < NW; ++q)
        {
            const unsigned kq = sh.key[buf][q][0], pq = sh.key[buf][q][1];
            if (kq > gmax || (kq == gmax && pq < gpos))
            {
                gmax = kq;
                gpos = pq;
                gw = q;
            }
        }
        const int pr = (int)gpos;
        const float *prow = sh.slot[buf][gw];
        if (pivoting && t == 0) ipiv[k0 + j] = k0 + pr + 1;
#pragma unroll
        for (int s = 0; s < 2; ++s) pos[s] = pos[s] == j ? pr : (pos[s] == pr ? j : pos[s]);
        const float d = prow[j];
        if (d == 0.0f)
        {
            if (t == 0)
            {
                if (sh.state == 0) sh.state = k0 + j + 1;
                sh.zmask |= 1u << j;
            }
        }
        else if (k0 + j + 1 < n)
        {
#pragma unroll
            for (int s = 0; s < 2; ++s)
            {
                if (valid[s] && pos[s] > j)
                {
                    const float l = div_rn(r[s][j], d);
                    r[s][j] = l;
#pragma unroll
                    for (int c = j + 1; c < NB; ++c) r[s][c] = fma_rn(-l, prow[c], r[s][c]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// trailing update tiles: C (positions r0.., columns j0..) -= L21 U12
// ---------------------------------------------------------------------------------------
// Plain: thread (tr, tc) owns rows {tr*4 + i, 64 + tr*4 + i} x columns tc*4 + j; ascending k.
__device__ __forceinline__ void tile_plain(float *A, int lda, int m, int k0, int j0, int nc, int r0, unsigned zmask,
                                           const float *L, int lp, const float *us, bool vec)
{
    const int t = threadIdx.x;
    const int tr = t & 15, tc = t >> 4;
    float acc[8][4];
    int rows[8];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int i = 0; i < 4; ++i) rows[h * 4 + i] = r0 + h * 64 + tr * 4 + i;
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const int cj = tc * 4 + j;
        const float *col = A + (int64_t)(j0 + cj) * lda + k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int rb = rows[h * 4];
            if (vec && cj < nc && rb + 3 < m)
            {
                const float4 v = *reinterpret_cast<const float4 *>(col + rb);
                acc[h * 4 + 0][j] = v.x;
                acc[h * 4 + 1][j] = v.y;
                acc[h * 4 + 2][j] = v.z;
                acc[h * 4 + 3][j] = v.w;
            }
            else
            {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    acc[h * 4 + i][j] = (cj < nc && rows[h * 4 + i] < m) ? col[rows[h * 4 + i]] : 0.0f;
            }
        }
    }
#pragma unroll 8
    for (int k = 0; k < NB; ++k)
    {
        if ((zmask >> k) & 1u) continue;  // uniform
        const float4 a0 = *reinterpret_cast<const float4 *>(L + k * lp + r0 + tr * 4);
        const float4 a1 = *reinterpret_cast<const float4 *>(L + k * lp + r0 + 64 + tr * 4);
        const float4 b = *reinterpret_cast<const float4 *>(us + k * UP + tc * 4);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(-a[i], bb[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const int cj = tc * 4 + j;
        float *col = A + (int64_t)(j0 + cj) * lda + k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int rb = rows[h * 4];
            if (vec && cj < nc && rb + 3 < m)
                *reinterpret_cast<float4 *>(col + rb) =
                    make_float4(acc[h * 4 + 0][j], acc[h * 4 + 1][j], acc[h * 4 + 2][j], acc[h * 4 + 3][j]);
            else
            {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (cj < nc && rows[h * 4 + i] < m) col[rows[h * 4 + i]] = acc[h * 4 + i][j];
            }
        }
    }
}

__device__ __forceinline__ void ldsm_x4(unsigned (&d)[4], const void *p)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3])
                 : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Mixed: warp (wm = warp & 3, wn = warp >> 2) owns rows r0 + wm*32 .. +31, columns
// wn*32 .. +31 of the tile: 2 x 4 mma tiles of 16 x 8, K = 32 in two k16 steps.  The staged
// L21 halves are negated, so C + (-L) U accumulates the update.
template <int TERMS>
__device__ __forceinline__ void tile_mixed(float *A, int lda, int m, int k0, int j0, int nc, int r0,
                                           const __nv_bfloat16 *lh, const __nv_bfloat16 *ll,
                                           const __nv_bfloat16 *uh, const __nv_bfloat16 *ul)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = r0 + (warp & 3) * 32;
    const int wc = (warp >> 2) * 32;
    const int g = lane >> 2, q = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e)
            {
                const int row = wr + mi * 16 + g + (e >= 2 ? 8 : 0);
                const int cj = wc + ni * 8 + q * 2 + (e & 1);
                acc[mi][ni][e] = (row < m && cj < nc) ? A[(int64_t)(j0 + cj) * lda + k0 + row] : 0.0f;
            }
#pragma unroll
    for (int ks = 0; ks < 2; ++ks)
    {
        unsigned ah[2][4], al[2][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
        {
            const int row = wr + mi * 16 + (lane & 15);
            const int kk = ks * 16 + (lane >> 4) * 8;
            ldsm_x4(ah[mi], lh + (size_t)row * HP + kk);
            if (TERMS > 1) ldsm_x4(al[mi], ll + (size_t)row * HP + kk);
        }
#pragma unroll
        for (int np = 0; np < 2; ++np)
        {
            const int mt = lane >> 3, rr = lane & 7;
            const int col = wc + np * 16 + (mt >> 1) * 8 + rr;
            const int kk = ks * 16 + (mt & 1) * 8;
            unsigned bh[4], bl[4];
            ldsm_x4(bh, uh + (size_t)col * HP + kk);
            if (TERMS > 1) ldsm_x4(bl, ul + (size_t)col * HP + kk);
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ni = np * 2 + h;
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
                {
                    if (TERMS > 1)
                    {
                        mma_bf16(acc[mi][ni], al[mi], bh[2 * h], bh[2 * h + 1]);
                        mma_bf16(acc[mi][ni], ah[mi], bl[2 * h], bl[2 * h + 1]);
                    }
                    mma_bf16(acc[mi][ni], ah[mi], bh[2 * h], bh[2 * h + 1]);
                }
            }
        }
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e)
            {
                const int row = wr + mi * 16 + g + (e >= 2 ? 8 : 0);
                const int cj = wc + ni * 8 + q * 2 + (e & 1);
                if (row < m && cj < nc) A[(int64_t)(j0 + cj) * lda + k0 + row] = acc[mi][ni][e];
            }
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// ---------------------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------------------
template <int MODE>  // 0 plain FP32, 1 BF16, 3 split BF16 (three products)
__global__ void __launch_bounds__(BT, 2) getrf_blocked_kernel(float *single, float *const *table, int first, int n,
                                                               int lda, int *ipiv, int *info, int count)
{
    constexpr int TERMS = MODE == 1 ? 1 : 3;
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ Shared sh;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int rows = round_rows(n);
    const int lp = (int)lp_pitch(n);
    // carve the dynamic area
    float *L = reinterpret_cast<float *>(dyn);  // plain: NB x lp; mixed: L11 NB x (NB + 4)
    float *us = L + (MODE == 0 ? (size_t)NB * lp : (size_t)NB * (NB + 4));
    __nv_bfloat16 *lh = reinterpret_cast<__nv_bfloat16 *>(us + (size_t)NB * UP);
    __nv_bfloat16 *ll = lh + (size_t)rows * HP;
    __nv_bfloat16 *uh = ll + (TERMS > 1 ? (size_t)rows * HP : 0);
    __nv_bfloat16 *ul = uh + (size_t)CT * HP;
    const int l11p = MODE == 0 ? lp : NB + 4;

    for (int64_t q = blockIdx.x; q < count; q += gridDim.x)
    {
        float *A = table ? slot(table, first + q) : single;
        if (!A)
        {
            if (t == 0) info[q] = -2;
            continue;
        }
        int *piv = ipiv ? ipiv + q * n : nullptr;
        const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0;
        if (t == 0) sh.state = 0;
        for (int k0 = 0; k0 < n; k0 += NB)
        {
            const int w = min(NB, n - k0);
            const int m = n - k0;
            if (t == 0)
            {
                sh.zmask = 0u;
                sh.nchanged = 0;
            }
            float r[2][NB];
            int pos[2];
            panel_factor(A, lda, n, k0, w, piv, piv != nullptr, sh, r, pos);
            // write back in final order, stage L, record the permutation
#pragma unroll
            for (int s = 0; s < 2; ++s)
            {
                const int i = t + s * BT;
                if (i < m)
                {
                    const int p = pos[s];
#pragma unroll
                    for (int c = 0; c < NB; ++c)
                        if (c < w) A[(int64_t)(k0 + c) * lda + k0 + p] = r[s][c];
                    sh.perm[p] = (short)i;
                    if (MODE == 0)
                    {
#pragma unroll
                        for (int c = 0; c < NB; ++c) L[c * lp + p] = r[s][c];
                    }
                    else if (p < NB)
                    {
#pragma unroll
                        for (int c = 0; c < NB; ++c) L[c * l11p + p] = r[s][c];
                    }
                }
            }
            __syncthreads();  // perm, zmask and the staged L are complete
            if (MODE != 0 && k0 + w < n)
            {
                const unsigned zm = sh.zmask;
#pragma unroll
                for (int s = 0; s < 2; ++s)
                {
                    const int i = t + s * BT;
                    if (i < m && pos[s] >= NB)
                    {
                        __nv_bfloat16 h[NB], l[NB];
#pragma unroll
                        for (int c = 0; c < NB; ++c)
                        {
                            const float v = ((zm >> c) & 1u) ? 0.0f : -r[s][c];
                            split_bf16(v, h[c], l[c]);
                        }
                        uint4 *dh = reinterpret_cast<uint4 *>(lh + (size_t)pos[s] * HP);
                        uint4 *dl = reinterpret_cast<uint4 *>(ll + (size_t)pos[s] * HP);
#pragma unroll
                        for (int c = 0; c < NB; c += 8)
                        {
                            dh[c / 8] = *reinterpret_cast<const uint4 *>(&h[c]);
                            if (TERMS > 1) dl[c / 8] = *reinterpret_cast<const uint4 *>(&l[c]);
                        }
                    }
                }
            }
            for (int p = t; p < m; p += BT)
                if (sh.perm[p] != p)
                {
                    const int at = atomicAdd(&sh.nchanged, 1);
                    if (at < 2 * NB) sh.changed[at] = p;
                }
            __syncthreads();
            if (k0 + w >= n) break;  // last panel: no trailing columns (w == NB below)
            const unsigned zmask = sh.zmask;
            const int nch = min(sh.nchanged, 2 * NB);
            for (int j0 = k0 + NB; j0 < n; j0 += CT)
            {
                const int nc = min(CT, n - j0);
                // (a) a warp per column: U12 rows through the permutation, moved rows in place
                for (int jj = warp; jj < nc; jj += NW)
                {
                    float *col = A + (int64_t)(j0 + jj) * lda + k0;
                    const float top = col[sh.perm[lane]];
                    int p0 = -1, p1 = -1;
                    float v0 = 0.0f, v1 = 0.0f;
                    if (lane < nch)
                    {
                        p0 = sh.changed[lane];
                        v0 = col[sh.perm[p0]];
                    }
                    if (lane + 32 < nch)
                    {
                        p1 = sh.changed[lane + 32];
                        v1 = col[sh.perm[p1]];
                    }
                    __syncwarp();
                    if (p0 >= NB) col[p0] = v0;
                    if (p1 >= NB) col[p1] = v1;
                    us[lane * UP + jj] = top;
                }
                __syncthreads();
                // (b) U12 = L11^-1 A12: four threads per column, thread part owns rows part + 4s
                {
                    const int jj = t >> 2, part = t & 3;
                    float v[8];
#pragma unroll
                    for (int s = 0; s < 8; ++s) v[s] = jj < nc ? us[(part + 4 * s) * UP + jj] : 0.0f;
#pragma unroll
                    for (int k = 0; k < NB; ++k)
                    {
                        if ((zmask >> k) & 1u) continue;  // uniform
                        const float u = __shfl_sync(FULL, v[k >> 2], (lane & ~3) | (k & 3));
#pragma unroll
                        for (int s = 0; s < 8; ++s)
                        {
                            const int i = part + 4 * s;
                            if (i > k) v[s] = fma_rn(-L[k * l11p + i], u, v[s]);
                        }
                    }
                    if (jj < nc)
                    {
#pragma unroll
                        for (int s = 0; s < 8; ++s) us[(part + 4 * s) * UP + jj] = v[s];
                    }
                }
                __syncthreads();
                // (c) U12 to global; mixed: its BF16 split, stored [column][k]
                for (int jj = warp; jj < nc; jj += NW) A[(int64_t)(j0 + jj) * lda + k0 + lane] = us[lane * UP + jj];
                if (MODE != 0)
                {
                    for (int e = t; e < CT * (NB / 2); e += BT)
                    {
                        const int jj = e / (NB / 2), k = (e % (NB / 2)) * 2;
                        const float u0 = jj < nc ? us[k * UP + jj] : 0.0f;
                        const float u1 = jj < nc ? us[(k + 1) * UP + jj] : 0.0f;
                        __nv_bfloat16 h0, l0, h1, l1;
                        split_bf16(u0, h0, l0);
                        split_bf16(u1, h1, l1);
                        *reinterpret_cast<__nv_bfloat162 *>(uh + (size_t)jj * HP + k) = __halves2bfloat162(h0, h1);
                        if (TERMS > 1)
                            *reinterpret_cast<__nv_bfloat162 *>(ul + (size_t)jj * HP + k) = __halves2bfloat162(l0, l1);
                    }
                    __syncthreads();
                }
                // (d) A22 -= L21 U12 over 128-row tiles (positions NB..m-1)
                for (int r0 = NB; r0 < m; r0 += RT)
                {
                    if (MODE == 0)
                        tile_plain(A, lda, m, k0, j0, nc, r0, zmask, L, lp, us, vec);
                    else
                        tile_mixed<TERMS>(A, lda, m, k0, j0, nc, r0, lh, ll, uh, ul);
                }
                __syncthreads();
            }
        }
        // Epilogue: the L columns of panel p take the row interchanges of panels p+1.. as
        // one gather, final[pos] = stored[T[pos]], T composed from the last panel backwards.
        const int npanel = (n + NB - 1) / NB;
        if (piv && npanel > 1)
        {
            for (int i = t; i < n; i += BT) sh.tmap[i] = (short)i;
            float *stage = L + (size_t)warp * MAXN;  // the L staging area is free now
            for (int p = npanel - 2; p >= 0; --p)
            {
                const int kq = (p + 1) * NB, wq = min(NB, n - kq);
                for (int i = t; i < n; i += BT) sh.umap[i] = (short)i;
                __syncthreads();
                if (t == 0)
                    for (int k = kq; k < kq + wq; ++k)
                    {
                        const int s = piv[k] - 1;
                        const short a = sh.umap[k];
                        sh.umap[k] = sh.umap[s];
                        sh.umap[s] = a;
                    }
                __syncthreads();
                for (int i = kq + t; i < n; i += BT) sh.tmap[i] = sh.umap[sh.tmap[i]];
                __syncthreads();
                for (int c = warp; c < NB; c += NW)
                {
                    float *col = A + (int64_t)(p * NB + c) * lda;
                    for (int i = kq + lane; i < n; i += 32) stage[i - kq] = col[i];
                    __syncwarp();
                    for (int i = kq + lane; i < n; i += 32) col[i] = stage[sh.tmap[i] - kq];
                    __syncwarp();
                }
            }
        }
        __syncthreads();
        if (t == 0) info[q] = sh.state;
        __syncthreads();
    }
}

template <int MODE>
cudaError_t launch_mode(const RealBatch &a, int *ipiv, int *info, cudaStream_t stream)
{
    const size_t smem = dyn_bytes(a.n, MODE);
    cudaError_t e = cudaFuncSetAttribute(getrf_blocked_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int64_t blocks = a.count < 148 * 2 ? a.count : 148 * 2;
    if (blocks < 1) blocks = 1;
    getrf_blocked_kernel<MODE><<<(unsigned)blocks, BT, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld, ipiv,
                                                                       info, a.count);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_getrf_blocked(const RealBatch &a, int *ipiv, int *info, int mode, cudaStream_t stream)
{
    if (a.n > MAXN || a.n < 1) return cudaErrorInvalidValue;
    switch (mode)
    {
        case 0:
            return launch_mode<0>(a, ipiv, info, stream);
        case 1:
            return launch_mode<1>(a, ipiv, info, stream);
        default:
            return launch_mode<3>(a, ipiv, info, stream);
    }
}

}  // namespace ops_solver
