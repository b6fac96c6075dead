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
//     also carry the winning row, so the pivot row needs no second broadcast); final values
//     go to the row's own place in A as they are produced;
//  2. the columns of the panel's outer block (W2 = 128 columns) take the panel's row
//     interchanges (a warp per column, 32 columns in flight, only the rows whose position
//     changed) and the panel's L is staged in shared memory (FP32, or negated BF16 hi/lo for
//     the tensor cores);
//  3. inside the outer block: U12 = L11^-1 A12 (a thread per column, in registers), then
//     A22 -= L21 U12 over 128 x 64 tiles whose U12
//     block is prefetched into the other half of a double-buffered shared tile and whose C
//     is prefetched into registers one row tile ahead;
//  4. after the block's four panels, the columns right of it take the block's composed
//     interchanges, U12 = L11^-1 A12 with the block's 128 x 128 L11 (in 32-row chunks), and
//     one rank-128 update A22 -= L21 U12 (128 x 64 tiles, L21 row tile staged once), so the
//     trailing matrix makes one trip through memory per 128 columns instead of per 32;
//  5. a second kernel, one block per (matrix, panel), applies the row interchanges of the
//     later outer blocks to that panel's L columns in one gather per column (LAPACK's final
//     row order): bandwidth-bound work that no longer waits behind the factorisation.
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
constexpr int NPANEL = MAXN / NB;
constexpr int CT = 64;   // trailing column tile
constexpr int RT = 128;  // trailing row tile
constexpr int UP = CT + 4;  // pitch of the FP32 U12 tile
constexpr int HP = NB + 8;  // pitch (halfs) of the BF16 tiles: 80 bytes, ldmatrix conflict-free
constexpr int L11P = NB + 4;
constexpr int SWAP_COLS = 32;  // columns in flight per warp during the row interchanges
constexpr int W2 = 128;        // outer block: inner panels update only its columns; the rest of the
                              // matrix takes one rank-128 update per outer block
constexpr int LTP = RT + 4;   // plain outer update: L21 tile Lt[k][row] pitch (floats)
constexpr int UTP = CT + 4;   // plain outer update: U12 tile Ut[k][col] pitch (floats)
constexpr int BHP = W2 + 8;   // mixed outer update: [row][k] and [col][k] BF16 pitch (272 bytes)
constexpr int LOP = W2 + 4;   // outer L11 Lo[k][i] pitch (floats)
constexpr int BSWAP = 4;      // columns in flight per warp in the outer row interchanges
constexpr unsigned FULL = 0xffffffffu;
static_assert(MAXN == 512, "the mixed panel's packed pivot key holds a 9-bit position");
static_assert(NPANEL == BLOCKED_PANELS && PANEL_LIST_SHORTS >= 1 + 4 * NB && W2 == BLOCKED_OUTER_COLS,
              "panel change lists");

struct __align__(16) Shared
{
    float slot[2][NW][NB];     // each warp's best pivot row, double buffered by column parity
    uint2 key[2][NW];          // each warp's (best key, its position)
    int krow[2][NW];           // each warp's best row (panel-relative index)
    short perm[MAXN];          // perm[p]: panel-relative row now at panel position p
    int changed[2 * NB];       // panel positions whose row changed
    short chg[NPANEL][2 * NB];  // per panel: changed positions and the rows they received,
    short src[NPANEL][2 * NB];  // kept for the epilogue
    int nchg[NPANEL];
    int nchanged;
    unsigned bz[W2 / NB];      // zero-pivot bits of the outer block's panels
    unsigned zmask;            // bit j: panel column j had a zero pivot (not used for updates)
    int state;                 // info of the matrix
};

__host__ __device__ constexpr int lp_pitch(int n) { return (n + 3) / 4 * 4 + 4; }

// Dynamic shared memory (bytes) for order n.
//   plain: L (NB x lp floats, L[k][p]), U12 tiles (2 x NB x UP floats)
//   mixed: L11 (NB x L11P floats), L21 hi/lo (n x HP bf16 each), U12 hi/lo tiles (2 x CT x HP each)
__host__ __device__ size_t dyn_bytes(int n, int mode)
{
    const int terms = mode == 1 ? 1 : 2;
    const size_t inner = mode == 0 ? ((size_t)NB * lp_pitch(n) + 2 * (size_t)NB * UP) * sizeof(float)
                                   : (size_t)NB * L11P * sizeof(float) +
                                         (size_t)terms * ((size_t)n * HP + 2 * (size_t)CT * HP) * sizeof(__nv_bfloat16);
    if (n <= W2) return inner;
    const size_t trsm = ((size_t)W2 * LOP + (size_t)CT * LOP) * sizeof(float);
    const size_t tiles = mode == 0 ? ((size_t)W2 * LTP + (size_t)W2 * UTP) * sizeof(float)
                                   : (size_t)terms * ((size_t)RT * BHP + (size_t)CT * BHP) * sizeof(__nv_bfloat16);
    // mixed U12 through X = L11^-1: X (FP32, 128 x LOP) and the A12 tile (128 x UTP), both FP32
    const size_t xsplit = mode == 0 ? 0 : ((size_t)W2 * LOP + (size_t)W2 * UTP) * sizeof(float);
    size_t need = inner > trsm ? inner : trsm;
    need = need > xsplit ? need : xsplit;
    return need > tiles ? need : tiles;
}

// ---------------------------------------------------------------------------------------
// panel
// ---------------------------------------------------------------------------------------
// The panel's rows stay in registers, but rotated: in a group of four steps the current
// column is r[s][u] (u = 0..3), and after the group every row shifts left by four, so all
// register indices are compile-time constants inside a short loop body.  Columns are held
// in pairs (r[s][p] = columns 2p, 2p + 1) and updated with paired FMAs; a pair whose first
// column is the step's own takes a dead update there.  Only the window's live columns
// (< w - j0) are updated and published.  Each value that becomes final is stored at its
// row's place in A as it is produced (an L entry at its step, the pivot row's U entries at
// the pivot step, from the slot); rows are brought into their final order afterwards, with
// the interchanges of the trailing columns.
// EXACT (plain mode): largest |a| with the earliest position on ties, IEEE division.  The
// mixed modes, whose factors are refined, take one warp reduction over a packed key (the
// |a| key's top 22 bits above the position's complement: ties within 2^-13 relative go to
// the earliest position) and multiply by the pivot's reciprocal.
template <bool EXACT, int NR>
__device__ __forceinline__ void panel_rows(float *A, int lda, int n, int k0, int w, int *ipiv, bool pivoting,
                                           Shared &sh, int (&pos)[2])
{
    constexpr int NP = NB / 2;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int m = n - k0;
    const bool active = warp * 32 < m;  // warp-uniform: some row of this warp is in the panel
    float *pan = A + (int64_t)k0 * lda + k0;  // panel element (row i, column c) at pan[c * lda + i]
    f32x2 r[NR][NP];
    bool valid[NR];
    pos[1] = t + BT;  // one row per thread: the second is past the panel
#pragma unroll
    for (int s = 0; s < NR; ++s)
    {
        const int i = t + s * BT;
        valid[s] = i < m;
        pos[s] = i;
#pragma unroll
        for (int p = 0; p < NP; ++p)
        {
            const float lo = (valid[s] && 2 * p < w) ? pan[(int64_t)(2 * p) * lda + i] : 0.0f;
            const float hi = (valid[s] && 2 * p + 1 < w) ? pan[(int64_t)(2 * p + 1) * lda + i] : 0.0f;
            r[s][p] = f2_pack(lo, hi);
        }
    }
    for (int j0 = 0; j0 < w; j0 += 4)
    {
        const int wl = w - j0;  // live columns of the window
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
            const int j = j0 + u;
            if (j >= w) break;  // uniform
            const int buf = j & 1;
            float cur[NR];
#pragma unroll
            for (int s = 0; s < NR; ++s) cur[s] = (u & 1) ? f2_hi(r[s][u / 2]) : f2_lo(r[s][u / 2]);
            if (active)
            {
                unsigned key[NR];
#pragma unroll
                for (int s = 0; s < NR; ++s)
                {
                    const float v = cur[s];
                    if (!valid[s])
                        key[s] = 0u;
                    else if (pivoting)
                        key[s] = pos[s] == j && v != v ? 0xffffffffu : (pos[s] >= j ? pivot_key(v) : 0u);
                    else
                        key[s] = pos[s] == j ? 1u : 0u;
                }
                unsigned wmax, wpos;
                if (EXACT)
                {
                    wmax = __reduce_max_sync(FULL, NR > 1 ? max(key[0], key[NR - 1]) : key[0]);
                    unsigned cand = 0xffffffffu;
#pragma unroll
                    for (int s = 0; s < NR; ++s)
                        if (valid[s] && key[s] == wmax) cand = min(cand, (unsigned)pos[s]);
                    wpos = __reduce_min_sync(FULL, cand);
                }
                else
                {
#pragma unroll
                    for (int s = 0; s < NR; ++s)
                        key[s] = key[s] == 0u ? 0u : (((key[s] >> 10) + 1u) << 9) | (unsigned)(MAXN - 1 - pos[s]);
                    wmax = __reduce_max_sync(FULL, NR > 1 ? max(key[0], key[NR - 1]) : key[0]);
                    wpos = wmax == 0u ? 0xffffffffu : (unsigned)(MAXN - 1) - (wmax & (MAXN - 1));
                }
#pragma unroll
                for (int s = 0; s < NR; ++s)
                    if (valid[s] && key[s] == wmax && (unsigned)pos[s] == wpos)
                    {
                        ulonglong2 *dst = reinterpret_cast<ulonglong2 *>(sh.slot[buf][warp]);
#pragma unroll
                        for (int q = 0; q < NP / 2; ++q)
                            if (4 * q < wl) dst[q] = make_ulonglong2(r[s][2 * q], r[s][2 * q + 1]);
                        sh.krow[buf][warp] = t + s * BT;
                    }
                if (lane == 0) sh.key[buf][warp] = make_uint2(wmax, wpos);
            }
            else if (lane == 0)
                sh.key[buf][warp] = make_uint2(0u, 0xffffffffu);
            __syncthreads();
            if (!active) continue;  // no rows here: nothing to eliminate
            // the block's winner: largest key, then the smallest position (a warp without
            // candidates reports key 0 and always loses: the position-j row has key >= 1).
            // Lane i reads warp i & 7's report; the lowest matching lane names the warp.
            const uint2 kw = sh.key[buf][lane & (NW - 1)];
            const unsigned gmax = __reduce_max_sync(FULL, kw.x);
            // the refined modes' keys carry the position, so the largest one names it (a live
            // row always has a nonzero key); the exact mode settles ties by a second reduction
            const unsigned gpos = EXACT ? __reduce_min_sync(FULL, kw.x == gmax ? kw.y : 0xffffffffu)
                                        : (unsigned)(MAXN - 1) - (gmax & (MAXN - 1));
            const int gw = __ffs(__ballot_sync(FULL, kw.x == gmax && kw.y == gpos)) - 1;
            const int pr = (int)gpos;
            const float *prow = sh.slot[buf][gw];  // prow[c]: the pivot row at column j0 + c
            if (pivoting && t == 0) ipiv[k0 + j] = k0 + pr + 1;
            // the pivot row's U entries (columns j .. w - 1) are final now
            if (t < w - j) pan[(int64_t)(j + t) * lda + sh.krow[buf][gw]] = prow[u + t];
#pragma unroll
            for (int s = 0; s < NR; ++s) pos[s] = pos[s] == j ? pr : (pos[s] == pr ? j : pos[s]);
            const float d = prow[u];
            bool go[NR];
#pragma unroll
            for (int s = 0; s < NR; ++s) go[s] = valid[s] && pos[s] > j;
            if (d == 0.0f)
            {
                if (t == 0)
                {
                    if (sh.state == 0) sh.state = k0 + j + 1;
                    sh.zmask |= 1u << j;
                }
                // a zero pivot scales nothing: the column keeps its values as L entries
#pragma unroll
                for (int s = 0; s < NR; ++s)
                    if (go[s]) pan[(int64_t)j * lda + t + s * BT] = cur[s];
            }
            else
            {
                float l[NR];
                // the reciprocal serves both: the refined modes multiply by it, the plain mode
                // divides through it (div_by: IEEE-exact)
                const float rinv = __frcp_rn(d);
                const bool dok = div_range(d);
#pragma unroll
                for (int s = 0; s < NR; ++s)
                {
                    l[s] = go[s] ? (EXACT ? div_by(cur[s], d, rinv, dok) : cur[s] * rinv) : 0.0f;
                    if (go[s]) pan[(int64_t)j * lda + t + s * BT] = l[s];
                }
                f32x2 nl[NR];
#pragma unroll
                for (int s = 0; s < NR; ++s) nl[s] = f2_pack(-l[s], -l[s]);
                // the pivot row four columns (two pairs) at a time, shared by both rows
                const ulonglong2 *p2 = reinterpret_cast<const ulonglong2 *>(prow);
#pragma unroll
                for (int q = 0; q < NP / 2; ++q)
                {
                    if (4 * q + 3 <= u) continue;  // compile-time: columns already final
                    if (4 * q >= wl) break;        // uniform: past the panel
                    const ulonglong2 v = p2[q];
                    if (4 * q + 1 > u)
                    {
#pragma unroll
                        for (int s = 0; s < NR; ++s)
                            if (go[s]) fma2(r[s][2 * q], nl[s], v.x);
                    }
#pragma unroll
                    for (int s = 0; s < NR; ++s)
                        if (go[s]) fma2(r[s][2 * q + 1], nl[s], v.y);
                }
            }
        }
        // rotate: the next four columns (two pairs) move to the front
#pragma unroll
        for (int s = 0; s < NR; ++s)
        {
#pragma unroll
            for (int p = 0; p < NP - 2; ++p) r[s][p] = r[s][p + 2];
            r[s][NP - 2] = 0ull;
            r[s][NP - 1] = 0ull;
        }
    }
}


// Two rows per thread while the panel is taller than the block, one row after.
template <bool EXACT>
__device__ __forceinline__ void panel_factor(float *A, int lda, int n, int k0, int w, int *ipiv, bool pivoting,
                                             Shared &sh, int (&pos)[2])
{
    if (n - k0 > BT)
        panel_rows<EXACT, 2>(A, lda, n, k0, w, ipiv, pivoting, sh, pos);
    else
        panel_rows<EXACT, 1>(A, lda, n, k0, w, ipiv, pivoting, sh, pos);
}

// ---------------------------------------------------------------------------------------
// trailing update tiles: C (positions r0.., columns j0..) -= L21 U12
// ---------------------------------------------------------------------------------------
// Plain: thread (tr, tc) owns rows {tr*4 + i, 64 + tr*4 + i} x columns tc*4 + j.
__device__ __forceinline__ void plain_c_load(const float *A, int lda, int m, int k0, int j0, int nc, int r0, bool vec,
                                             float (&c)[8][4])
{
    const int t = threadIdx.x;
    const int tr = t & 15, tc = t >> 4;
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const int cj = tc * 4 + j;
        const float *col = A + (int64_t)(j0 + min(cj, nc - 1)) * lda + k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int rb = r0 + h * 64 + tr * 4;
            if (vec && rb + 3 < m)
            {
                const float4 v = *reinterpret_cast<const float4 *>(col + rb);
                c[h * 4 + 0][j] = v.x;
                c[h * 4 + 1][j] = v.y;
                c[h * 4 + 2][j] = v.z;
                c[h * 4 + 3][j] = v.w;
            }
            else
            {
#pragma unroll
                for (int i = 0; i < 4; ++i) c[h * 4 + i][j] = rb + i < m ? col[rb + i] : 0.0f;
            }
        }
    }
}

__device__ __forceinline__ void plain_c_store(float *A, int lda, int m, int k0, int j0, int nc, int r0, bool vec,
                                              const float (&c)[8][4])
{
    const int t = threadIdx.x;
    const int tr = t & 15, tc = t >> 4;
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const int cj = tc * 4 + j;
        if (cj >= nc) continue;
        float *col = A + (int64_t)(j0 + cj) * lda + k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int rb = r0 + h * 64 + tr * 4;
            if (vec && rb + 3 < m)
                *reinterpret_cast<float4 *>(col + rb) =
                    make_float4(c[h * 4 + 0][j], c[h * 4 + 1][j], c[h * 4 + 2][j], c[h * 4 + 3][j]);
            else
            {
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (rb + i < m) col[rb + i] = c[h * 4 + i][j];
            }
        }
    }
}

// acc -= L21 U12 in ascending k (zero-pivot columns skipped).  Rows past the staged ones
// read clamped (in-range, unused) entries.
__device__ __forceinline__ void plain_c_update(float (&acc)[8][4], const float *L, int lp, int r0, unsigned zmask,
                                               const float *us)
{
    const int t = threadIdx.x;
    const int tr = t & 15, tc = t >> 4;
    const int ra = min(r0 + tr * 4, lp - 4), rb = min(r0 + 64 + tr * 4, lp - 4);
    if (zmask == 0u)
    {
        // no zero pivot in the panel (the usual case): a branch-free loop the compiler can
        // software-pipeline
#pragma unroll 8
        for (int k = 0; k < NB; ++k)
        {
            const float4 a0 = *reinterpret_cast<const float4 *>(L + k * lp + ra);
            const float4 a1 = *reinterpret_cast<const float4 *>(L + k * lp + rb);
            const float4 b = *reinterpret_cast<const float4 *>(us + k * UP + tc * 4);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(-a[i], bb[j], acc[i][j]);
        }
        return;
    }
#pragma unroll 8
    for (int k = 0; k < NB; ++k)
    {
        if ((zmask >> k) & 1u) continue;  // uniform
        const float4 a0 = *reinterpret_cast<const float4 *>(L + k * lp + ra);
        const float4 a1 = *reinterpret_cast<const float4 *>(L + k * lp + rb);
        const float4 b = *reinterpret_cast<const float4 *>(us + k * UP + tc * 4);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(-a[i], bb[j], acc[i][j]);
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

// Mixed: warp (wm = warp & 3, wn = warp >> 2) owns rows r0 + wm*32 .. +31 and columns
// wn*32 .. +31 of the tile: 2 x 4 mma tiles of 16 x 8, K = 32 in two k16 steps.  Element
// e of mma tile (mi, ni) is row g + 8*(e >= 2) + 16 mi, column 2q + (e & 1) + 8 ni.
__device__ __forceinline__ void mixed_c_load(const float *A, int lda, int m, int k0, int j0, int nc, int r0,
                                             float (&c)[2][4][4])
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = r0 + (warp & 3) * 32, wc = (warp >> 2) * 32;
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e)
            {
                const int row = wr + mi * 16 + g + (e >= 2 ? 8 : 0);
                const int cj = wc + ni * 8 + q * 2 + (e & 1);
                c[mi][ni][e] = (row < m && cj < nc) ? A[(int64_t)(j0 + cj) * lda + k0 + row] : 0.0f;
            }
}

__device__ __forceinline__ void mixed_c_store(float *A, int lda, int m, int k0, int j0, int nc, int r0,
                                              const float (&c)[2][4][4])
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = r0 + (warp & 3) * 32, wc = (warp >> 2) * 32;
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e)
            {
                const int row = wr + mi * 16 + g + (e >= 2 ? 8 : 0);
                const int cj = wc + ni * 8 + q * 2 + (e & 1);
                if (row < m && cj < nc) A[(int64_t)(j0 + cj) * lda + k0 + row] = c[mi][ni][e];
            }
}

// The staged L21 halves are negated, so C + (-L) U accumulates the update.
template <int TERMS>
__device__ __forceinline__ void mixed_c_update(float (&acc)[2][4][4], int n, int r0, const __nv_bfloat16 *lh,
                                               const __nv_bfloat16 *ll, const __nv_bfloat16 *uh,
                                               const __nv_bfloat16 *ul)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = r0 + (warp & 3) * 32, wc = (warp >> 2) * 32;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks)
    {
        unsigned ah[2][4], al[2][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
        {
            const int row = min(wr + mi * 16 + (lane & 15), n - 1);  // rows past n: unused
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
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// U12 tile prefetch: thread t holds rows kq .. kq + 7 (kq = 8 (t & 3)) of column t >> 2.
__device__ __forceinline__ void u_load(const float *A, int lda, int k0, int j0, int nc, bool vec, float (&u)[8])
{
    const int t = threadIdx.x;
    const int cc = t >> 2, kq = (t & 3) * 8;
    const float *src = A + (int64_t)(j0 + min(cc, nc - 1)) * lda + k0 + kq;
    if (vec)
    {
        const float4 a = *reinterpret_cast<const float4 *>(src);
        const float4 b = *reinterpret_cast<const float4 *>(src + 4);
        u[0] = a.x, u[1] = a.y, u[2] = a.z, u[3] = a.w, u[4] = b.x, u[5] = b.y, u[6] = b.z, u[7] = b.w;
    }
    else
    {
#pragma unroll
        for (int i = 0; i < 8; ++i) u[i] = src[i];
    }
    if (cc >= nc)
    {
#pragma unroll
        for (int i = 0; i < 8; ++i) u[i] = 0.0f;
    }
}

template <int MODE, int TERMS>
__device__ __forceinline__ void u_store(const float (&u)[8], float *us, __nv_bfloat16 *uh, __nv_bfloat16 *ul)
{
    const int t = threadIdx.x;
    const int cc = t >> 2, kq = (t & 3) * 8;
    if (MODE == 0)
    {
#pragma unroll
        for (int i = 0; i < 8; ++i) us[(kq + i) * UP + cc] = u[i];
    }
    else
    {
        __nv_bfloat16 h[8], l[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) split_bf16(u[i], h[i], l[i]);
        *reinterpret_cast<uint4 *>(uh + (size_t)cc * HP + kq) = *reinterpret_cast<const uint4 *>(h);
        if (TERMS > 1) *reinterpret_cast<uint4 *>(ul + (size_t)cc * HP + kq) = *reinterpret_cast<const uint4 *>(l);
    }
}

// Global -> shared staging with BATCH loads in flight per thread: the loads of a batch are
// issued before any of its shared stores, so the copy is paced by bandwidth rather than by
// one memory round trip per element (the compiler cannot reorder a global load past a store
// through a generic pointer on its own).
template <int BATCH, typename Load, typename Store>
__device__ __forceinline__ void staged_copy(int total, Load load, Store store)
{
    for (int e0 = threadIdx.x; e0 < total; e0 += BT * BATCH)
    {
        float v[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; ++u)
        {
            const int e = e0 + u * BT;
            v[u] = e < total ? load(e) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < BATCH; ++u)
        {
            const int e = e0 + u * BT;
            if (e < total) store(e, v[u]);
        }
    }
}

// ---------------------------------------------------------------------------------------
// outer-block update: the trailing columns take the outer block's interchanges, its U12
// (rank-W2 triangular solve) and one rank-W2 update
// ---------------------------------------------------------------------------------------
// Plain: acc -= Lt[k][rows] Ut[k][cols] over k < W2 in ascending order, zero pivots skipped.
__device__ __forceinline__ void plain_outer_update(float (&acc)[8][4], const float *Lt, const float *Ut,
                                                   const unsigned *bz)
{
    const int t = threadIdx.x;
    const int tr = t & 15, tc = t >> 4;
    unsigned any_zero = 0u;
#pragma unroll
    for (int i = 0; i < W2 / 32; ++i) any_zero |= bz[i];
    if (any_zero == 0u)
    {
#pragma unroll 8
        for (int kk = 0; kk < W2; ++kk)
        {
            const float4 a0 = *reinterpret_cast<const float4 *>(Lt + kk * LTP + tr * 4);
            const float4 a1 = *reinterpret_cast<const float4 *>(Lt + kk * LTP + 64 + tr * 4);
            const float4 b = *reinterpret_cast<const float4 *>(Ut + kk * UTP + tc * 4);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(-a[i], bb[j], acc[i][j]);
        }
        return;
    }
#pragma unroll 1
    for (int kb = 0; kb < W2; kb += 32)
    {
        const unsigned z = bz[kb / 32];
#pragma unroll 8
        for (int k = 0; k < 32; ++k)
        {
            if ((z >> k) & 1u) continue;  // uniform
            const int kk = kb + k;
            const float4 a0 = *reinterpret_cast<const float4 *>(Lt + kk * LTP + tr * 4);
            const float4 a1 = *reinterpret_cast<const float4 *>(Lt + kk * LTP + 64 + tr * 4);
            const float4 b = *reinterpret_cast<const float4 *>(Ut + kk * UTP + tc * 4);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(-a[i], bb[j], acc[i][j]);
        }
    }
}

// Mixed: the tile's negated L21 halves Lh/Ll[row][k] and U12 halves Uh/Ul[col][k], K = W2.
template <int TERMS>
__device__ __forceinline__ void mixed_outer_update(float (&acc)[2][4][4], const __nv_bfloat16 *lh,
                                                   const __nv_bfloat16 *ll, const __nv_bfloat16 *uh,
                                                   const __nv_bfloat16 *ul)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wr = (warp & 3) * 32, wc = (warp >> 2) * 32;
#pragma unroll 2
    for (int ks = 0; ks < W2 / 16; ++ks)
    {
        unsigned ah[2][4], al[2][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
        {
            const int row = wr + mi * 16 + (lane & 15);
            const int kk = ks * 16 + (lane >> 4) * 8;
            ldsm_x4(ah[mi], lh + (size_t)row * BHP + kk);
            if (TERMS > 1) ldsm_x4(al[mi], ll + (size_t)row * BHP + kk);
        }
#pragma unroll
        for (int np = 0; np < 2; ++np)
        {
            const int mt = lane >> 3, rr = lane & 7;
            const int col = wc + np * 16 + (mt >> 1) * 8 + rr;
            const int kk = ks * 16 + (mt & 1) * 8;
            unsigned bh[4], bl[4];
            ldsm_x4(bh, uh + (size_t)col * BHP + kk);
            if (TERMS > 1) ldsm_x4(bl, ul + (size_t)col * BHP + kk);
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
}

// Mixed modes, U12 of the outer block: X = L11^-1 (unit lower, 128 x 128) is built once in
// FP32 -- the four 32 x 32 diagonal inverses by substitution (a warp each, a lane per
// column), then the off-diagonal blocks by distance, X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj
// -- and every 64-column tile of A12 becomes U12 = X A12 by FP32 FMAs: no serial chain over
// the 128 rows, and FP32-level accuracy (a BF16 split of X and A12 cost the refinement a
// correction on the worst-conditioned systems).  Zero-pivot columns of L are zeroed first, so they take
// no part, as in the plain solve.  Layout while X is built: L(i, k) (i > k) at Lo[k][i] and
// X(r, c) (c <= r) at Lo[r][c], the staged block's upper triangle being free.
__device__ void mixed_outer_u12(float *A, int lda, int n, int K0, Shared &sh, unsigned char *dyn)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int kend = K0 + W2;
    float *Lo = reinterpret_cast<float *>(dyn);
    float *T = Lo + (size_t)W2 * LOP;  // S blocks of one distance: T[b][r][c], pitch 33
    staged_copy<16>(
        W2 * W2,
        [&](int e) {
            const int k = e / W2, i = e % W2;
            const bool zero = i > k && ((sh.bz[k / 32] >> (k & 31)) & 1u);
            return zero ? 0.0f : A[(int64_t)(K0 + k) * lda + K0 + i];
        },
        [&](int e, float v) { Lo[(e / W2) * LOP + e % W2] = v; });
    __syncthreads();
    // (1) diagonal blocks: warp b inverts L_bb, lane j computing column j of the inverse
    if (warp < W2 / 32)
    {
        const int b0 = warp * 32;
        float y[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) y[r] = r == lane ? 1.0f : 0.0f;
#pragma unroll
        for (int k = 0; k < 32; ++k)
        {
            const float yk = y[k];
#pragma unroll
            for (int r = k + 1; r < 32; ++r) y[r] = fma_rn(-Lo[(b0 + k) * LOP + b0 + r], yk, y[r]);
        }
        // reads were of the lower triangle, writes go to the upper one (and the diagonal)
#pragma unroll
        for (int r = 0; r < 32; ++r)
            if (r >= lane) Lo[(b0 + r) * LOP + b0 + lane] = y[r];
    }
    __syncthreads();
    // (2) off-diagonal blocks, distance d = i - j: thread (warp, lane) owns rows 4 warp .. +3
    //     and column lane of every block
    const int rq = warp * 4, c = lane;
#pragma unroll 1
    for (int d = 1; d < W2 / 32; ++d)
    {
        const int nblk = W2 / 32 - d;
#pragma unroll 1
        for (int b = 0; b < nblk; ++b)
        {
            const int j = b, i = b + d;
            float sv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 1
            for (int kb = j; kb < i; ++kb)
            {
#pragma unroll 8
                for (int kk = 0; kk < 32; ++kk)
                {
                    const int K = kb * 32 + kk;
                    // X(K, 32 j + c): zero above the diagonal of X_jj
                    const float x = (kb > j || kk >= c) ? Lo[K * LOP + j * 32 + c] : 0.0f;
                    const float4 l = *reinterpret_cast<const float4 *>(Lo + (size_t)K * LOP + i * 32 + rq);
                    sv[0] = fma_rn(l.x, x, sv[0]);
                    sv[1] = fma_rn(l.y, x, sv[1]);
                    sv[2] = fma_rn(l.z, x, sv[2]);
                    sv[3] = fma_rn(l.w, x, sv[3]);
                }
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) T[(b * 32 + rq + e) * 33 + c] = sv[e];
        }
        __syncthreads();
#pragma unroll 1
        for (int b = 0; b < nblk; ++b)
        {
            const int j = b, i = b + d;
            float xv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 8
            for (int kk = 0; kk < 32; ++kk)
            {
                const float s = T[(b * 32 + kk) * 33 + c];
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (kk <= rq + e) xv[e] = fma_rn(Lo[(i * 32 + rq + e) * LOP + i * 32 + kk], s, xv[e]);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) Lo[(i * 32 + rq + e) * LOP + j * 32 + c] = -xv[e];
        }
        __syncthreads();
    }
    // (3) X complete: the strictly upper part of Lo (the staged L values) is cleared, so
    //     Lo[r][k] = X(r, k) for every k
    for (int e = t; e < W2 * W2; e += BT)
    {
        const int r = e / W2, k = e % W2;
        if (k > r) Lo[r * LOP + k] = 0.0f;
    }
    // (4) U12 = X A12 in FP32, a 64-column tile at a time: the tile staged k-major, thread
    //     (tr, tc) computing rows tr + 16 i (i < 8, conflict-free X reads) by columns 4tc..+3
    float *At = Lo + (size_t)W2 * LOP;  // At[k][col], pitch UTP
    const int tr = t & 15, tc = t >> 4;
    for (int c0 = kend; c0 < n; c0 += CT)
    {
        const int nc = min(CT, n - c0);
        __syncthreads();  // the previous tile's products are done with At (and (3) with Lo)
        staged_copy<16>(
            W2 * CT, [&](int e) { return e / W2 < nc ? A[(int64_t)(c0 + e / W2) * lda + K0 + e % W2] : 0.0f; },
            [&](int e, float v) { At[(e % W2) * UTP + e / W2] = v; });
        __syncthreads();
        float acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
#pragma unroll 2
        for (int k4 = 0; k4 < W2; k4 += 4)
        {
            float4 xr[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                xr[i] = *reinterpret_cast<const float4 *>(Lo + (size_t)(16 * i + tr) * LOP + k4);
            float4 ak[4];
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) ak[kk] = *reinterpret_cast<const float4 *>(At + (k4 + kk) * UTP + 4 * tc);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
            {
                const float a4[4] = {ak[kk].x, ak[kk].y, ak[kk].z, ak[kk].w};
#pragma unroll
                for (int i = 0; i < 8; ++i)
                {
                    const float xv = kk == 0 ? xr[i].x : kk == 1 ? xr[i].y : kk == 2 ? xr[i].z : xr[i].w;
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma_rn(xv, a4[j], acc[i][j]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int cj = 4 * tc + j;
            if (cj >= nc) continue;
            float *col = A + (int64_t)(c0 + cj) * lda + K0;
#pragma unroll
            for (int i = 0; i < 8; ++i) col[16 * i + tr] = acc[i][j];
        }
    }
    __syncthreads();  // the next stage reuses the shared area
}

template <int MODE, int TERMS>
__device__ void outer_update(float *A, int lda, int n, int K0, bool vec, Shared &sh, unsigned char *dyn)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int kend = K0 + W2;
    const int mb = n - K0;  // rows (positions) of the outer block and below
    // (a) the block's composed permutation P (position -> row, relative to K0) and the
    //     positions whose row changed
    short *P = reinterpret_cast<short *>(dyn);
    int *bch = reinterpret_cast<int *>(dyn + 2 * MAXN);
    for (int i = t; i < mb; i += BT) P[i] = (short)i;
    if (t == 0) sh.nchanged = 0;
    __syncthreads();
    for (int ip = 0; ip < W2 / NB; ++ip)
    {
        const int pidx = K0 / NB + ip, rel = ip * NB;
        short v = 0;
        if (t < sh.nchg[pidx]) v = P[rel + sh.src[pidx][t]];
        __syncthreads();
        if (t < sh.nchg[pidx]) P[rel + sh.chg[pidx][t]] = v;
        __syncthreads();
    }
    for (int p = t; p < mb; p += BT)
        if (P[p] != p) bch[atomicAdd(&sh.nchanged, 1)] = p;
    __syncthreads();
    const int nb = sh.nchanged;  // at most 2 NB per inner panel
    // (b) the interchanges on the trailing columns: a warp per column, BSWAP columns in flight
    {
        constexpr int PER = (W2 / NB) * 2 * NB / 32;  // changed positions per lane, at most
        int dst[PER], srcr[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j)
        {
            const int e = lane + 32 * j;
            dst[j] = e < nb ? bch[e] : -1;
            srcr[j] = e < nb ? P[dst[j]] : 0;
        }
        const int ntr = n - kend;
        for (int base = warp * BSWAP; base < ntr; base += NW * BSWAP)
        {
            float v[BSWAP][PER];
#pragma unroll
            for (int c = 0; c < BSWAP; ++c)
            {
                const float *col = A + (int64_t)(kend + min(base + c, ntr - 1)) * lda + K0;
#pragma unroll
                for (int j = 0; j < PER; ++j) v[c][j] = dst[j] >= 0 ? col[srcr[j]] : 0.0f;
            }
            __syncwarp();
#pragma unroll
            for (int c = 0; c < BSWAP; ++c)
            {
                if (base + c >= ntr) continue;
                float *col = A + (int64_t)(kend + base + c) * lda + K0;
#pragma unroll
                for (int j = 0; j < PER; ++j)
                    if (dst[j] >= 0) col[dst[j]] = v[c][j];
            }
        }
    }
    __syncthreads();
    // (c) U12 = L11^-1 A12.  Mixed modes: through X = L11^-1 on the tensor cores.  Plain: with the
    //     block's unit-lower L11 (staged), per 64-column tile held
    //     in shared memory: four threads per column, each owning eight consecutive rows of
    //     every 32-row chunk; chunk ci is solved (shuffles among the four), then applied to
    //     the rows of the later chunks, in ascending k for every element
    if (MODE != 0)
        mixed_outer_u12(A, lda, n, K0, sh, dyn);
    else
    {
    float *Lo = reinterpret_cast<float *>(dyn);
    float *Ub = Lo + (size_t)W2 * LOP;  // CT columns x LOP: Ub[col][row]
    staged_copy<16>(
        W2 * W2, [&](int e) { return A[(int64_t)(K0 + e / W2) * lda + K0 + e % W2]; },
        [&](int e, float v) { Lo[(e / W2) * LOP + e % W2] = v; });
    for (int j0 = kend; j0 < n; j0 += CT)
    {
        const int nc = min(CT, n - j0);
        staged_copy<16>(
            W2 * CT,
            [&](int e) { return e / W2 < nc ? A[(int64_t)(j0 + e / W2) * lda + K0 + e % W2] : 0.0f; },
            [&](int e, float v) { Ub[(e / W2) * LOP + e % W2] = v; });
        __syncthreads();
        {
            // thread (cc, part) owns rows 8 part .. 8 part + 7 of every chunk of column cc
            const int cc = t >> 2, part = t & 3;
            float *ucol = Ub + cc * LOP;
#pragma unroll 1
            for (int ci = 0; ci < W2 / 32; ++ci)
            {
                const unsigned z = sh.bz[ci];
                float v[8];
                {
                    const float4 p0 = *reinterpret_cast<const float4 *>(ucol + ci * 32 + 8 * part);
                    const float4 p1 = *reinterpret_cast<const float4 *>(ucol + ci * 32 + 8 * part + 4);
                    v[0] = p0.x, v[1] = p0.y, v[2] = p0.z, v[3] = p0.w, v[4] = p1.x, v[5] = p1.y, v[6] = p1.z, v[7] = p1.w;
                }
#pragma unroll
                for (int k = 0; k < 32; ++k)
                {
                    if ((z >> k) & 1u) continue;  // uniform
                    const float u = __shfl_sync(FULL, v[k & 7], (lane & ~3) | (k >> 3));
                    const float4 l0 = *reinterpret_cast<const float4 *>(Lo + (ci * 32 + k) * LOP + ci * 32 + 8 * part);
                    const float4 l1 = *reinterpret_cast<const float4 *>(Lo + (ci * 32 + k) * LOP + ci * 32 + 8 * part + 4);
                    const float lv[8] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y, l1.z, l1.w};
#pragma unroll
                    for (int s = 0; s < 8; ++s)
                        if (8 * part + s > k) v[s] = fma_rn(-lv[s], u, v[s]);
                }
                *reinterpret_cast<float4 *>(ucol + ci * 32 + 8 * part) = make_float4(v[0], v[1], v[2], v[3]);
                *reinterpret_cast<float4 *>(ucol + ci * 32 + 8 * part + 4) = make_float4(v[4], v[5], v[6], v[7]);
                __syncwarp();
#pragma unroll 1
                for (int cj = ci + 1; cj < W2 / 32; ++cj)
                {
                    float x[8];
                    {
                        const float4 p0 = *reinterpret_cast<const float4 *>(ucol + cj * 32 + 8 * part);
                        const float4 p1 = *reinterpret_cast<const float4 *>(ucol + cj * 32 + 8 * part + 4);
                        x[0] = p0.x, x[1] = p0.y, x[2] = p0.z, x[3] = p0.w, x[4] = p1.x, x[5] = p1.y, x[6] = p1.z, x[7] = p1.w;
                    }
#pragma unroll 4
                    for (int k4 = 0; k4 < 32; k4 += 4)
                    {
                        const float4 u4 = *reinterpret_cast<const float4 *>(ucol + ci * 32 + k4);
                        const float uu[4] = {u4.x, u4.y, u4.z, u4.w};
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                        {
                            const int k = k4 + e;
                            if ((z >> k) & 1u) continue;
                            const float4 l0 = *reinterpret_cast<const float4 *>(Lo + (ci * 32 + k) * LOP + cj * 32 + 8 * part);
                            const float4 l1 =
                                *reinterpret_cast<const float4 *>(Lo + (ci * 32 + k) * LOP + cj * 32 + 8 * part + 4);
                            const float lv[8] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y, l1.z, l1.w};
#pragma unroll
                            for (int s = 0; s < 8; ++s) x[s] = fma_rn(-lv[s], uu[e], x[s]);
                        }
                    }
                    *reinterpret_cast<float4 *>(ucol + cj * 32 + 8 * part) = make_float4(x[0], x[1], x[2], x[3]);
                    *reinterpret_cast<float4 *>(ucol + cj * 32 + 8 * part + 4) = make_float4(x[4], x[5], x[6], x[7]);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int e = t; e < W2 * CT; e += BT)
        {
            const int cc = e / W2, r = e % W2;
            if (cc < nc) A[(int64_t)(j0 + cc) * lda + K0 + r] = Ub[cc * LOP + r];
        }
        __syncthreads();
    }
    }
    // (d) A22 -= L21 U12, K = W2: a row tile of L21 staged once, then every column tile
    for (int r0 = W2; r0 < mb; r0 += RT)
    {
        if (MODE == 0)
        {
            float *Lt = reinterpret_cast<float *>(dyn);
            staged_copy<16>(
                W2 * RT,
                [&](int e) { return r0 + e % RT < mb ? A[(int64_t)(K0 + e / RT) * lda + K0 + r0 + e % RT] : 0.0f; },
                [&](int e, float v) { Lt[(e / RT) * LTP + e % RT] = v; });
        }
        else
        {
            __nv_bfloat16 *lh = reinterpret_cast<__nv_bfloat16 *>(dyn);
            __nv_bfloat16 *ll = lh + (size_t)RT * BHP;
            staged_copy<16>(
                W2 * RT,
                [&](int e) { return r0 + e % RT < mb ? A[(int64_t)(K0 + e / RT) * lda + K0 + r0 + e % RT] : 0.0f; },
                [&](int e, float a) {
                    const int k = e / RT, rr = e % RT;
                    const float v = ((sh.bz[k / 32] >> (k & 31)) & 1u) ? 0.0f : -a;
                    __nv_bfloat16 h, l;
                    split_bf16(v, h, l);
                    lh[(size_t)rr * BHP + k] = h;
                    if (TERMS > 1) ll[(size_t)rr * BHP + k] = l;
                });
        }
        for (int c0 = kend; c0 < n; c0 += CT)
        {
            const int nc = min(CT, n - c0);
            if (MODE == 0)
            {
                float *Ut = reinterpret_cast<float *>(dyn) + (size_t)W2 * LTP;
                staged_copy<16>(
                    W2 * CT,
                    [&](int e) { return e / W2 < nc ? A[(int64_t)(c0 + e / W2) * lda + K0 + e % W2] : 0.0f; },
                    [&](int e, float v) { Ut[(e % W2) * UTP + e / W2] = v; });
            }
            else
            {
                __nv_bfloat16 *uh = reinterpret_cast<__nv_bfloat16 *>(dyn) + (size_t)(TERMS > 1 ? 2 : 1) * RT * BHP;
                __nv_bfloat16 *ul = uh + (size_t)CT * BHP;
                staged_copy<16>(
                    W2 * CT,
                    [&](int e) { return e / W2 < nc ? A[(int64_t)(c0 + e / W2) * lda + K0 + e % W2] : 0.0f; },
                    [&](int e, float v) {
                        __nv_bfloat16 h, l;
                        split_bf16(v, h, l);
                        uh[(size_t)(e / W2) * BHP + e % W2] = h;
                        if (TERMS > 1) ul[(size_t)(e / W2) * BHP + e % W2] = l;
                    });
            }
            __syncthreads();
            if (MODE == 0)
            {
                float acc[8][4];
                plain_c_load(A, lda, mb, K0, c0, nc, r0, vec, acc);
                plain_outer_update(acc, reinterpret_cast<float *>(dyn), reinterpret_cast<float *>(dyn) + (size_t)W2 * LTP,
                                   sh.bz);
                plain_c_store(A, lda, mb, K0, c0, nc, r0, vec, acc);
            }
            else
            {
                const __nv_bfloat16 *lh = reinterpret_cast<const __nv_bfloat16 *>(dyn);
                const __nv_bfloat16 *ll = lh + (size_t)RT * BHP;
                const __nv_bfloat16 *uh = lh + (size_t)(TERMS > 1 ? 2 : 1) * RT * BHP;
                const __nv_bfloat16 *ul = uh + (size_t)CT * BHP;
                float acc[2][4][4];
                mixed_c_load(A, lda, mb, K0, c0, nc, r0, acc);
                mixed_outer_update<TERMS>(acc, lh, ll, uh, ul);
                mixed_c_store(A, lda, mb, K0, c0, nc, r0, acc);
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------------------
template <int MODE>  // 0 plain FP32, 1 BF16, 3 split BF16 (three products)
__global__ void __launch_bounds__(BT, 2) getrf_blocked_kernel(float *single, float *const *table, int first, int n,
                                                               int lda, int *ipiv, int *info, int count,
                                                               const float *const *src, int src_ld, int *perm_out,
                                                               short *lists_out)
{
    constexpr int TERMS = MODE == 1 ? 1 : 3;
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ Shared sh;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int lp = lp_pitch(n);
    // carve the dynamic area
    float *L = reinterpret_cast<float *>(dyn);  // plain: NB x lp; mixed: L11 NB x L11P
    float *us = L + (MODE == 0 ? (size_t)NB * lp : (size_t)NB * L11P);  // plain: 2 x NB x UP
    __nv_bfloat16 *lh = reinterpret_cast<__nv_bfloat16 *>(us);          // mixed: after L11
    __nv_bfloat16 *ll = lh + (size_t)n * HP;
    __nv_bfloat16 *uh = lh + (size_t)(TERMS > 1 ? 2 : 1) * n * HP;      // 2 x CT x HP
    __nv_bfloat16 *ul = uh + 2 * (size_t)CT * HP;
    const float *l11 = L;
    const int l11p = MODE == 0 ? lp : L11P;

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
        if (src)
        {
            // out of place: the matrix is first copied from its source slot
            const float *S = slot(src, q);
            if (!S)
            {
                if (t == 0) info[q] = -2;
                continue;
            }
            const bool v4 = vec && (reinterpret_cast<uintptr_t>(S) & 15u) == 0 && (src_ld & 3) == 0 && (n & 3) == 0;
            if (v4)
            {
                const int per = n / 4;
                for (int e = t; e < n * per; e += BT)
                {
                    const int c = e / per, r4 = (e % per) * 4;
                    *reinterpret_cast<float4 *>(A + (int64_t)c * lda + r4) =
                        __ldg(reinterpret_cast<const float4 *>(S + (int64_t)c * src_ld + r4));
                }
            }
            else
            {
                for (int e = t; e < n * n; e += BT)
                {
                    const int c = e / n, r = e % n;
                    A[(int64_t)c * lda + r] = S[(int64_t)c * src_ld + r];
                }
            }
            __syncthreads();
        }
        if (t == 0) sh.state = 0;
        for (int K0 = 0; K0 < n; K0 += W2)
        {
        const int kend = min(n, K0 + W2);
        for (int k0 = K0; k0 < kend; k0 += NB)
        {
            const int w = min(NB, n - k0);
            const int m = n - k0;
            if (t == 0)
            {
                sh.zmask = 0u;
                sh.nchanged = 0;
            }
            int pos[2];
            panel_factor<MODE == 0>(A, lda, n, k0, w, piv, piv != nullptr, sh, pos);
            // the permutation and the positions whose row changed
#pragma unroll
            for (int s = 0; s < 2; ++s)
                if (t + s * BT < m) sh.perm[pos[s]] = (short)(t + s * BT);
            __syncthreads();
            for (int p = t; p < m; p += BT)
                if (sh.perm[p] != p)
                {
                    const int at = atomicAdd(&sh.nchanged, 1);
                    if (at < 2 * NB) sh.changed[at] = p;
                }
            __syncthreads();
            const int nch = min(sh.nchanged, 2 * NB);
            {
                // kept for the epilogue, and written out for a solve over factors without the
                // left interchanges
                short *entry = lists_out ? lists_out + ((size_t)q * BLOCKED_PANELS + k0 / NB) * PANEL_LIST_SHORTS
                                         : nullptr;
                if (t < nch)
                {
                    const int p = sh.changed[t];
                    const short from = sh.perm[p];
                    sh.chg[k0 / NB][t] = (short)p;
                    sh.src[k0 / NB][t] = from;
                    if (entry)
                    {
                        entry[1 + t] = (short)p;
                        entry[1 + 2 * NB + t] = from;
                    }
                }
                if (t == 0)
                {
                    sh.nchg[k0 / NB] = nch;
                    if (entry) entry[0] = (short)nch;
                }
            }
            // (1) row interchanges on the panel and trailing columns: a warp per column,
            //     SWAP_COLS columns in flight, every source read before any destination is
            //     written
            {
                int p0 = -1, p1 = -1, s0 = 0, s1 = 0;
                if (lane < nch)
                {
                    p0 = sh.changed[lane];
                    s0 = sh.perm[p0];
                }
                if (lane + 32 < nch)
                {
                    p1 = sh.changed[lane + 32];
                    s1 = sh.perm[p1];
                }
                // every column of the outer block: the block's earlier panels (their L), the
                // panel and the block's later columns
                const int mc = kend - K0;
                for (int base = warp * SWAP_COLS; base < mc; base += NW * SWAP_COLS)
                {
                    float v0[SWAP_COLS], v1[SWAP_COLS];
#pragma unroll
                    for (int c = 0; c < SWAP_COLS; ++c)
                    {
                        const float *col = A + (int64_t)(K0 + min(base + c, mc - 1)) * lda + k0;
                        v0[c] = p0 >= 0 ? col[s0] : 0.0f;
                        v1[c] = p1 >= 0 ? col[s1] : 0.0f;
                    }
                    __syncwarp();
#pragma unroll
                    for (int c = 0; c < SWAP_COLS; ++c)
                    {
                        if (base + c < mc)
                        {
                            float *col = A + (int64_t)(K0 + base + c) * lda + k0;
                            if (p0 >= 0) col[p0] = v0[c];
                            if (p1 >= 0) col[p1] = v1[c];
                        }
                    }
                }
            }
            if (t == 0) sh.bz[(k0 - K0) / NB] = sh.zmask;
            __syncthreads();
            if (k0 + w >= kend) continue;  // last panel of the block: nothing inside it to update (w == NB below)
            // stage L from the panel, now in final order: plain FP32 L[k][p]; mixed FP32 L11
            // and the negated BF16 split of L21 (zero-pivot columns zeroed)
            {
                const unsigned zm = sh.zmask;
                const float *pan = A + (int64_t)k0 * lda + k0;
#pragma unroll
                for (int s = 0; s < 2; ++s)
                {
                    const int p = t + s * BT;
                    if (p >= m) continue;
                    float v[NB];
#pragma unroll
                    for (int c = 0; c < NB; ++c) v[c] = pan[(int64_t)c * lda + p];
                    if (MODE == 0)
                    {
#pragma unroll
                        for (int c = 0; c < NB; ++c) L[c * lp + p] = v[c];
                    }
                    else if (p < NB)
                    {
#pragma unroll
                        for (int c = 0; c < NB; ++c) L[c * L11P + p] = v[c];
                    }
                    else
                    {
                        __nv_bfloat16 h[NB], l[NB];
#pragma unroll
                        for (int c = 0; c < NB; ++c)
                        {
                            const float x = ((zm >> c) & 1u) ? 0.0f : -v[c];
                            split_bf16(x, h[c], l[c]);
                        }
                        uint4 *dh = reinterpret_cast<uint4 *>(lh + (size_t)p * HP);
                        uint4 *dl = reinterpret_cast<uint4 *>(ll + (size_t)p * HP);
#pragma unroll
                        for (int c = 0; c < NB; c += 8)
                        {
                            dh[c / 8] = *reinterpret_cast<const uint4 *>(&h[c]);
                            if (TERMS > 1) dl[c / 8] = *reinterpret_cast<const uint4 *>(&l[c]);
                        }
                    }
                }
            }
            __syncthreads();
            const unsigned zmask = sh.zmask;
            const int jt = k0 + NB;   // first trailing column
            const int ntr = kend - jt;  // the rest of the outer block
            // (2) U12 = L11^-1 A12: a thread per column, ascending k, zero pivots skipped
            for (int jc = t; jc < ntr; jc += BT)
            {
                float *col = A + (int64_t)(jt + jc) * lda + k0;
                float v[NB];
                if (vec)
                {
#pragma unroll
                    for (int i = 0; i < NB; i += 4)
                    {
                        const float4 a = *reinterpret_cast<const float4 *>(col + i);
                        v[i] = a.x, v[i + 1] = a.y, v[i + 2] = a.z, v[i + 3] = a.w;
                    }
                }
                else
                {
#pragma unroll
                    for (int i = 0; i < NB; ++i) v[i] = col[i];
                }
#pragma unroll
                for (int k = 0; k < NB; ++k)
                {
                    if ((zmask >> k) & 1u) continue;  // uniform
                    const float u = v[k];
#pragma unroll
                    for (int i4 = 0; i4 < NB; i4 += 4)
                    {
                        if (i4 + 3 <= k) continue;
                        const float4 l4 = *reinterpret_cast<const float4 *>(l11 + k * l11p + i4);
                        const float lv[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            if (i4 + e > k) v[i4 + e] = fma_rn(-lv[e], u, v[i4 + e]);
                    }
                }
                if (vec)
                {
#pragma unroll
                    for (int i = 0; i < NB; i += 4)
                        *reinterpret_cast<float4 *>(col + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
                }
                else
                {
#pragma unroll
                    for (int i = 0; i < NB; ++i) col[i] = v[i];
                }
            }
            __syncthreads();
            // (3) A22 -= L21 U12 over 128 x 64 tiles (positions NB..m-1)
            const int nct = (ntr + CT - 1) / CT;
            {
                float u[8];
                u_load(A, lda, k0, jt, min(CT, ntr), vec, u);
                u_store<MODE, TERMS>(u, us, uh, ul);
            }
            __syncthreads();
            // the C tile of the next (column tile, row tile) pair is loaded while the current
            // one is updated, across column-tile boundaries too
            float acc[MODE == 0 ? 32 : 32], nxt[32];
            if (MODE == 0)
                plain_c_load(A, lda, m, k0, jt, min(CT, ntr), NB, vec, *reinterpret_cast<float(*)[8][4]>(acc));
            else
                mixed_c_load(A, lda, m, k0, jt, min(CT, ntr), NB, *reinterpret_cast<float(*)[2][4][4]>(acc));
            for (int ct = 0; ct < nct; ++ct)
            {
                const int j0 = jt + ct * CT;
                const int nc = min(CT, kend - j0);
                const int buf = ct & 1;
                float u[8];
                if (ct + 1 < nct) u_load(A, lda, k0, j0 + CT, min(CT, kend - j0 - CT), vec, u);
                for (int r0 = NB; r0 < m; r0 += RT)
                {
                    const bool more_rows = r0 + RT < m;
                    const bool more = more_rows || ct + 1 < nct;
                    const int nj0 = more_rows ? j0 : j0 + CT;
                    const int nnc = min(CT, kend - nj0);
                    const int nr0 = more_rows ? r0 + RT : NB;
                    if (MODE == 0)
                    {
                        auto &ca = *reinterpret_cast<float(*)[8][4]>(acc);
                        auto &cn = *reinterpret_cast<float(*)[8][4]>(nxt);
                        if (more) plain_c_load(A, lda, m, k0, nj0, nnc, nr0, vec, cn);
                        plain_c_update(ca, L, lp, r0, zmask, us + (size_t)buf * NB * UP);
                        plain_c_store(A, lda, m, k0, j0, nc, r0, vec, ca);
                    }
                    else
                    {
                        auto &ca = *reinterpret_cast<float(*)[2][4][4]>(acc);
                        auto &cn = *reinterpret_cast<float(*)[2][4][4]>(nxt);
                        if (more) mixed_c_load(A, lda, m, k0, nj0, nnc, nr0, cn);
                        mixed_c_update<TERMS>(ca, n, r0, lh, ll, uh + (size_t)buf * CT * HP, ul + (size_t)buf * CT * HP);
                        mixed_c_store(A, lda, m, k0, j0, nc, r0, ca);
                    }
                    if (more)
                    {
#pragma unroll
                        for (int i = 0; i < 32; ++i) acc[i] = nxt[i];
                    }
                }
                if (ct + 1 < nct)
                    u_store<MODE, TERMS>(u, us + (size_t)(buf ^ 1) * NB * UP, uh + (size_t)(buf ^ 1) * CT * HP,
                                         ul + (size_t)(buf ^ 1) * CT * HP);
                __syncthreads();
            }
        }
        __syncthreads();
        if (kend < n) outer_update<MODE, TERMS>(A, lda, n, K0, vec, sh, dyn);
        __syncthreads();
        }
        const int npanel_all = (n + NB - 1) / NB;
        if (perm_out && piv)
        {
            // the composed permutation: position i of the factors holds original row P[i]
            short *P = reinterpret_cast<short *>(dyn);
            for (int i = t; i < n; i += BT) P[i] = (short)i;
            for (int p = 0; p < npanel_all; ++p)
            {
                __syncthreads();
                const int kp = p * NB;
                short v = 0;
                if (t < sh.nchg[p]) v = P[kp + sh.src[p][t]];
                __syncthreads();
                if (t < sh.nchg[p]) P[kp + sh.chg[p][t]] = v;
            }
            __syncthreads();
            for (int i = t; i < n; i += BT) perm_out[q * n + i] = P[i];
            __syncthreads();
        }
        else if (perm_out)
        {
            for (int i = t; i < n; i += BT) perm_out[q * n + i] = i;
        }
        __syncthreads();
        if (t == 0) info[q] = sh.state;
        __syncthreads();
    }
}

// The L columns of panel p take the row interchanges of the panels of later outer blocks
// (those of its own block were applied to the whole block as they were made):
// final[pos] = stored[T[pos]], T the interchanges ipiv[k], k >= kq (the next block's first
// column), applied in order to the identity.  One block per (matrix, panel); a warp per
// column.
__global__ void __launch_bounds__(BT) left_swaps_kernel(float *single, float *const *table, int first, int n, int lda,
                                                         const int *ipiv, int count)
{
    __shared__ short T[MAXN];
    __shared__ float stage[NW][MAXN];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t q = blockIdx.x;
    const int p = blockIdx.y;
    if (q >= count) return;
    float *A = table ? slot(table, first + q) : single;
    if (!A) return;
    const int *piv = ipiv + q * n;
    const int kq = (p * NB / W2 + 1) * W2;
    if (kq >= n) return;
    for (int i = kq + t; i < n; i += BT) T[i] = (short)i;
    __syncthreads();
    if (t == 0)
        for (int k = kq; k < n; ++k)
        {
            const int s = piv[k] - 1;
            if (s > k && s < n)
            {
                const short v = T[k];
                T[k] = T[s];
                T[s] = v;
            }
        }
    __syncthreads();
    for (int c = warp; c < NB; c += NW)
    {
        float *col = A + (int64_t)(p * NB + c) * lda;
        float v[MAXN / 32];
#pragma unroll
        for (int u = 0; u < MAXN / 32; ++u)
        {
            const int i = kq + lane + 32 * u;
            v[u] = i < n ? col[i] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < MAXN / 32; ++u)
        {
            const int i = kq + lane + 32 * u;
            if (i < n) stage[warp][i - kq] = v[u];
        }
        __syncwarp();
        for (int i = kq + lane; i < n; i += 32) col[i] = stage[warp][T[i] - kq];
        __syncwarp();
    }
}

template <int MODE>
cudaError_t launch_mode(const RealBatch &a, int *ipiv, int *info, const float *const *src, int src_ld, int *perm,
                        short *lists, cudaStream_t stream)
{
    const size_t smem = dyn_bytes(a.n, MODE);
    cudaError_t e = cudaFuncSetAttribute(getrf_blocked_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int64_t blocks = a.count < 148 * 2 ? a.count : 148 * 2;
    if (blocks < 1) blocks = 1;
    getrf_blocked_kernel<MODE><<<(unsigned)blocks, BT, smem, stream>>>(a.single, a.table, a.first, a.n, a.ld, ipiv,
                                                                       info, a.count, src, src_ld, perm, lists);
    const int npanel = (a.n + NB - 1) / NB;
    if (ipiv && !lists && npanel > 1)
    {
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        left_swaps_kernel<<<dim3((unsigned)a.count, (unsigned)(npanel - 1)), BT, 0, stream>>>(
            a.single, a.table, a.first, a.n, a.ld, ipiv, a.count);
    }
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_getrf_blocked(const RealBatch &a, int *ipiv, int *info, int mode, cudaStream_t stream,
                                 const float *const *src, int src_ld, int *perm, short *lists)
{
    if (a.n > MAXN || a.n < 1) return cudaErrorInvalidValue;
    switch (mode)
    {
        case 0:
            return launch_mode<0>(a, ipiv, info, src, src_ld, perm, lists, stream);
        case 1:
            return launch_mode<1>(a, ipiv, info, src, src_ld, perm, lists, stream);
        default:
            return launch_mode<3>(a, ipiv, info, src, src_ld, perm, lists, stream);
    }
}

}  // namespace ops_solver
