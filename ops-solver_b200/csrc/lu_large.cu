// lu_large.cu -- LU with partial pivoting of one large matrix (rows up to 8192) over the
// whole GPU: the drop-in for the reference's blocked single-matrix factorisation
// (src/sgetrf/real_lu_blocked_kernel.cpp:1469-1520, BlockedFactorLaunch::Run and its panel,
// swap/trsm, product and subtract kernels; host entry src/sgetrf/sgetrf_host.cpp:96-124).
//
// Right-looking, two-level: 32-column panels inside 128-column outer blocks.
//   * panel (a cluster of eight 1024-thread blocks, one panel row per thread): per column,
//     each block finds its candidate (warp reduction, block barrier), publishes it into
//     every block of the cluster through distributed shared memory, one cluster barrier,
//     and every block picks the same winner; rows are never moved during the panel, final
//     values are written to their rows' places and the changed positions are listed;
//   * interchanges: the panel's changed positions moved in every column of the matrix;
//   * inside the outer block: U12 = L11^-1 A12 and A22 -= L21 U12 on its columns only;
//   * once per outer block: U12 with the 128 x 128 L11 and one rank-128 update of the
//     trailing matrix (FP32 FFMA2 tiles, or split-BF16 tensor-core tiles in mixed mode).
// Plain mode keeps the oracle's per-element order -- every element receives fma(-l, u, a)
// in ascending k, zero-pivot columns skipped, IEEE division by the pivot -- so factors,
// pivots and info equal the unblocked order bit for bit.
#include <cooperative_groups.h>

#include "common.cuh"
#include "launch.h"

namespace cg = cooperative_groups;

namespace ops_solver
{
namespace
{
constexpr int LT = 1024;      // panel threads per block
constexpr int LNW = LT / 32;  // panel warps per block
constexpr int PW = 32;        // panel width
constexpr int CSZ = 8;        // blocks per panel cluster
constexpr int OB = 128;       // outer block
constexpr unsigned FULL = 0xffffffffu;
static_assert(LNW == 32, "the block winner is read one warp report per lane");

struct __align__(16) PanelShared
{
    float slot[2][LNW][PW];  // each warp's best row, double buffered by column parity
    uint2 key[2][LNW];       // each warp's (best key, its position)
    int krow[2][LNW];        // each warp's best row (panel-relative)
    float cand[2][CSZ][PW];  // each cluster block's candidate row (written by that block)
    uint4 ckey[2][CSZ];      // each cluster block's (key, position, row, 0)
    unsigned zmask;
    int first_zero;
};

// ---------------------------------------------------------------------------------------
// panel: rows k0 .. m-1, columns k0 .. k0+w-1 of A (positions relative to k0)
// ---------------------------------------------------------------------------------------
template <bool EXACT>
__global__ void __cluster_dims__(CSZ, 1, 1) __launch_bounds__(LT, 1)
    large_panel_kernel(float *A, int lda, int m, int k0, int w, int *ipiv, LargeStatus *st)
{
    constexpr int NP = PW / 2;
    __shared__ PanelShared sh;
    cg::cluster_group cluster = cg::this_cluster();
    const int c = (int)cluster.block_rank();
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int mr = m - k0;
    const int R = (mr + CSZ - 1) / CSZ;  // rows per block
    const int r0 = c * R;
    const int mine = max(0, min(R, mr - r0));  // rows of this block
    const bool active = warp * 32 < mine;
    const bool valid = t < mine;
    const int i = r0 + t;  // this thread's panel row
    int pos = i;
    float *pan = A + (int64_t)k0 * lda + k0;
    const bool pivoting = ipiv != nullptr;
    if (t == 0)
    {
        sh.zmask = 0u;
        sh.first_zero = 0;
    }
    f32x2 r[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p)
    {
        const float lo = (valid && 2 * p < w) ? pan[(int64_t)(2 * p) * lda + i] : 0.0f;
        const float hi = (valid && 2 * p + 1 < w) ? pan[(int64_t)(2 * p + 1) * lda + i] : 0.0f;
        r[p] = f2_pack(lo, hi);
    }
    for (int j0 = 0; j0 < w; j0 += 4)
    {
        const int wl = w - j0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
            const int j = j0 + u;
            if (j >= w) break;  // uniform across the cluster
            const int buf = j & 1;
            const float cur = (u & 1) ? f2_hi(r[u / 2]) : f2_lo(r[u / 2]);
            // (1) each warp's candidate
            if (active)
            {
                unsigned key;
                if (!valid)
                    key = 0u;
                else if (pivoting)
                    key = pos == j && cur != cur ? 0xffffffffu : (pos >= j ? pivot_key(cur) : 0u);
                else
                    key = pos == j ? 1u : 0u;
                const unsigned wmax = __reduce_max_sync(FULL, key);
                const unsigned wpos = __reduce_min_sync(FULL, valid && key == wmax ? (unsigned)pos : 0xffffffffu);
                if (valid && key == wmax && (unsigned)pos == wpos)
                {
                    ulonglong2 *dst = reinterpret_cast<ulonglong2 *>(sh.slot[buf][warp]);
#pragma unroll
                    for (int q = 0; q < NP / 2; ++q)
                        if (4 * q < wl) dst[q] = make_ulonglong2(r[2 * q], r[2 * q + 1]);
                    sh.krow[buf][warp] = i;
                }
                if (lane == 0) sh.key[buf][warp] = make_uint2(wmax, wpos);
            }
            else if (lane == 0)
                sh.key[buf][warp] = make_uint2(0u, 0xffffffffu);
            __syncthreads();
            // (2) warp 0: the block's candidate, published to every block of the cluster
            if (warp == 0)
            {
                const uint2 kw = sh.key[buf][lane];
                const unsigned gmax = __reduce_max_sync(FULL, kw.x);
                const unsigned gpos = __reduce_min_sync(FULL, kw.x == gmax ? kw.y : 0xffffffffu);
                const int gw = __ffs(__ballot_sync(FULL, kw.x == gmax && kw.y == gpos)) - 1;
                const int dest = lane >> 2, part = lane & 3;
                const float4 *src = reinterpret_cast<const float4 *>(sh.slot[buf][gw]) + 2 * part;
                float4 *rc = reinterpret_cast<float4 *>(cluster.map_shared_rank(&sh.cand[buf][c][0], dest)) + 2 * part;
                rc[0] = src[0];
                rc[1] = src[1];
                if (part == 0)
                {
                    uint4 *kc = cluster.map_shared_rank(&sh.ckey[buf][c], dest);
                    *kc = make_uint4(gmax, gpos, (unsigned)sh.krow[buf][gw], 0u);
                }
            }
            cluster.sync();
            // (3) the cluster's winner: largest key, then the smallest position
            const uint4 kc = lane < CSZ ? sh.ckey[buf][lane] : make_uint4(0u, 0xffffffffu, 0u, 0u);
            const unsigned gmax = __reduce_max_sync(FULL, kc.x);
            const unsigned gpos = __reduce_min_sync(FULL, kc.x == gmax ? kc.y : 0xffffffffu);
            const int gc = __ffs(__ballot_sync(FULL, kc.x == gmax && kc.y == gpos)) - 1;
            const int pr = (int)gpos;
            const float *prow = sh.cand[buf][gc];
            const int krow = (int)sh.ckey[buf][gc].z;
            if (c == 0)
            {
                if (pivoting && t == 0) ipiv[k0 + j] = k0 + pr + 1;
                if (t < w - j) pan[(int64_t)(j + t) * lda + krow] = prow[u + t];
            }
            pos = pos == j ? pr : (pos == pr ? j : pos);
            const float d = prow[u];
            const bool go = valid && pos > j;
            if (d == 0.0f)
            {
                if (c == 0 && t == 0)
                {
                    if (sh.first_zero == 0) sh.first_zero = k0 + j + 1;
                    sh.zmask |= 1u << j;
                }
                if (go) pan[(int64_t)j * lda + i] = cur;
            }
            else
            {
                const float l = go ? (EXACT ? div_rn(cur, d) : cur * __frcp_rn(d)) : 0.0f;
                if (go) pan[(int64_t)j * lda + i] = l;
                const f32x2 nl = f2_pack(-l, -l);
                const ulonglong2 *p2 = reinterpret_cast<const ulonglong2 *>(prow);
#pragma unroll
                for (int q = 0; q < NP / 2; ++q)
                {
                    if (4 * q + 3 <= u) continue;
                    if (4 * q >= wl) break;
                    const ulonglong2 v = p2[q];
                    if (4 * q + 1 > u && go) fma2(r[2 * q], nl, v.x);
                    if (go) fma2(r[2 * q + 1], nl, v.y);
                }
            }
        }
#pragma unroll
        for (int p = 0; p < NP - 2; ++p) r[p] = r[p + 2];
        r[NP - 2] = 0ull;
        r[NP - 1] = 0ull;
    }
    // the changed positions (at most 2 w): position pos now holds physical row i
    if (valid && pos != i)
    {
        const int at = atomicAdd(&st->nchg[k0 / PW], 1);
        if (at < 2 * PW) st->chg[k0 / PW][at] = make_int2(pos, i);
    }
    if (c == 0 && t == 0)
    {
        st->zmask[k0 / PW] = sh.zmask;
        if (sh.first_zero && st->info == 0) st->info = sh.first_zero;
    }
}

// ---------------------------------------------------------------------------------------
// the panel's interchanges on every column: a warp per column, all reads before writes
// ---------------------------------------------------------------------------------------
constexpr int SW_COLS = 8;  // columns per warp

__global__ void __launch_bounds__(256) large_swap_kernel(float *A, int lda, int ncols, int k0, int skip0, int skip1,
                                                         const LargeStatus *st)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = k0 / PW;
    const int nch = min(st->nchg[p], 2 * PW);
    int dst0 = -1, src0 = 0, dst1 = -1, src1 = 0;
    if (lane < nch)
    {
        const int2 e = st->chg[p][lane];
        dst0 = e.x;
        src0 = e.y;
    }
    if (lane + 32 < nch)
    {
        const int2 e = st->chg[p][lane + 32];
        dst1 = e.x;
        src1 = e.y;
    }
    const int base = (blockIdx.x * 8 + warp) * SW_COLS;
    float v0[SW_COLS], v1[SW_COLS];
#pragma unroll
    for (int q = 0; q < SW_COLS; ++q)
    {
        int col = base + q;
        col = col >= skip0 && col < skip1 ? -1 : col;  // the panel's own columns are handled separately
        const float *a = A + (int64_t)col * lda + k0;
        v0[q] = (col >= 0 && col < ncols && dst0 >= 0) ? a[src0] : 0.0f;
        v1[q] = (col >= 0 && col < ncols && dst1 >= 0) ? a[src1] : 0.0f;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < SW_COLS; ++q)
    {
        int col = base + q;
        if (col >= skip0 && col < skip1) continue;
        if (col >= ncols) continue;
        float *a = A + (int64_t)col * lda + k0;
        if (dst0 >= 0) a[dst0] = v0[q];
        if (dst1 >= 0) a[dst1] = v1[q];
    }
}

// ---------------------------------------------------------------------------------------
// U12 = L11^-1 A12 for a unit-lower W x W L11 at (K0, K0): 64 columns per block, four
// threads per column, each owning eight rows of every 32-row chunk (ascending k, zero-pivot
// columns skipped)
// ---------------------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) large_trsm_kernel(float *A, int lda, int K0, int c0, int ncols,
                                                         const LargeStatus *st)
{
    constexpr int P = W + 4;
    extern __shared__ __align__(16) float smem[];
    float *Lo = smem;                  // Lo[k][i] = L(K0 + i, K0 + k)
    float *Ub = smem + (size_t)W * P;  // Ub[col][row]
    const int t = threadIdx.x, lane = t & 31;
    const int j0 = c0 + blockIdx.x * 64;
    const int nc = min(64, c0 + ncols - j0);
    for (int e = t; e < W * W; e += 256) Lo[(e / W) * P + e % W] = A[(int64_t)(K0 + e / W) * lda + K0 + e % W];
    for (int e = t; e < W * 64; e += 256)
    {
        const int cc = e / W, rr = e % W;
        Ub[cc * P + rr] = cc < nc ? A[(int64_t)(j0 + cc) * lda + K0 + rr] : 0.0f;
    }
    __syncthreads();
    const int cc = t >> 2, part = t & 3;
    float *ucol = Ub + cc * P;
#pragma unroll 1
    for (int ci = 0; ci < W / 32; ++ci)
    {
        const unsigned z = st->zmask[K0 / PW + ci];
        float v[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) v[s] = ucol[ci * 32 + 8 * part + s];
#pragma unroll
        for (int k = 0; k < 32; ++k)
        {
            if ((z >> k) & 1u) continue;  // uniform
            const float u = __shfl_sync(FULL, v[k & 7], (lane & ~3) | (k >> 3));
#pragma unroll
            for (int s = 0; s < 8; ++s)
                if (8 * part + s > k) v[s] = fma_rn(-Lo[(ci * 32 + k) * P + ci * 32 + 8 * part + s], u, v[s]);
        }
#pragma unroll
        for (int s = 0; s < 8; ++s) ucol[ci * 32 + 8 * part + s] = v[s];
        __syncwarp();
#pragma unroll 1
        for (int cj = ci + 1; cj < W / 32; ++cj)
        {
            float x[8];
#pragma unroll
            for (int s = 0; s < 8; ++s) x[s] = ucol[cj * 32 + 8 * part + s];
#pragma unroll 4
            for (int k = 0; k < 32; ++k)
            {
                if ((z >> k) & 1u) continue;
                const float u = ucol[ci * 32 + k];
#pragma unroll
                for (int s = 0; s < 8; ++s) x[s] = fma_rn(-Lo[(ci * 32 + k) * P + cj * 32 + 8 * part + s], u, x[s]);
            }
#pragma unroll
            for (int s = 0; s < 8; ++s) ucol[cj * 32 + 8 * part + s] = x[s];
        }
        __syncwarp();
    }
    __syncthreads();
    for (int e = t; e < W * 64; e += 256)
    {
        const int c2 = e / W, rr = e % W;
        if (c2 < nc) A[(int64_t)(j0 + c2) * lda + K0 + rr] = Ub[c2 * P + rr];
    }
}

// ---------------------------------------------------------------------------------------
// C -= L21 U12 (plain, exact order): C = A[r0.., c0..] (rows x cols), L21 = A[r0.., K0..],
// U12 = A[K0.., c0..], K = KW.  128 x 128 tile per block, thread tile 8 x 8 (rows
// 4tr..+3 and 64+4tr..+3, columns 4tc..+3 and 64+4tc..+3), row pairs in FFMA2 registers;
// U is staged negated and duplicated, so every product is fma(l, -u, c) = fma(-l, u, c).
// ---------------------------------------------------------------------------------------
constexpr int GT = 128;   // tile
constexpr int GK = 16;    // k per stage
constexpr int GLP = GT + 4;
constexpr int GUP = GT + 2;  // pairs: consecutive k rows of a column fall on different banks
constexpr size_t GEMM_SMEM = 2 * GK * GLP * sizeof(float) + 2 * GK * GUP * sizeof(f32x2);

__global__ void __launch_bounds__(256, 2) large_gemm_kernel(float *A, int lda, int r0, int rows, int c0, int cols,
                                                            int K0, int KW, const LargeStatus *st)
{
    extern __shared__ __align__(16) unsigned char gsm[];
    auto Ls = reinterpret_cast<float(*)[GK][GLP]>(gsm);                                  // Ls[buf][k][row]
    auto Us = reinterpret_cast<f32x2(*)[GK][GUP]>(gsm + 2 * GK * GLP * sizeof(float));  // Us[buf][k][col] = (-u, -u)
    const int t = threadIdx.x, tr = t & 15, tc = t >> 4;
    const int rb = r0 + blockIdx.x * GT, cb = c0 + blockIdx.y * GT;
    const int nr = min(GT, r0 + rows - rb), ncl = min(GT, c0 + cols - cb);
    // any zero pivot among the KW columns: those k are skipped (uniform per k)
    unsigned zany = 0u;
    for (int p = 0; p < KW / PW; ++p) zany |= st->zmask[K0 / PW + p];
    f32x2 acc[4][8];  // acc[ip][jc]: rows (2ip, 2ip+1) of the thread's 8, column jc
    const int rr[8] = {4 * tr, 4 * tr + 1, 4 * tr + 2, 4 * tr + 3, 64 + 4 * tr, 65 + 4 * tr, 66 + 4 * tr, 67 + 4 * tr};
    const int cc[8] = {4 * tc, 4 * tc + 1, 4 * tc + 2, 4 * tc + 3, 64 + 4 * tc, 65 + 4 * tc, 66 + 4 * tc, 67 + 4 * tc};
    // 16-byte accesses when the tile's rows are all present and aligned
    const bool vec = nr == GT && (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0 && (rb & 3) == 0;
#pragma unroll
    for (int jc = 0; jc < 8; ++jc)
    {
        const bool cv = cc[jc] < ncl;
        const float *col = A + (int64_t)(cb + min(cc[jc], ncl - 1)) * lda + rb;
        if (vec)
        {
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const ulonglong2 v = cv ? *reinterpret_cast<const ulonglong2 *>(col + 64 * h + 4 * tr)
                                        : make_ulonglong2(0ull, 0ull);
                acc[2 * h][jc] = v.x;
                acc[2 * h + 1][jc] = v.y;
            }
        }
        else
        {
#pragma unroll
            for (int ip = 0; ip < 4; ++ip)
            {
                const float lo = cv && rr[2 * ip] < nr ? col[rr[2 * ip]] : 0.0f;
                const float hi = cv && rr[2 * ip + 1] < nr ? col[rr[2 * ip + 1]] : 0.0f;
                acc[ip][jc] = f2_pack(lo, hi);
            }
        }
    }
    auto stage = [&](int buf, int kb) {
        // L: GK columns x 128 rows; U: GK rows x 128 columns
        for (int e = t; e < GK * GT; e += 256)
        {
            const int k = e / GT, x = e % GT;
            Ls[buf][k][x] = x < nr ? A[(int64_t)(K0 + kb + k) * lda + rb + x] : 0.0f;
        }
        for (int e = t; e < GK * GT; e += 256)
        {
            const int x = e / GK, k = e % GK;
            const float u = x < ncl ? A[(int64_t)(cb + x) * lda + K0 + kb + k] : 0.0f;
            Us[buf][k][x] = f2_pack(-u, -u);
        }
    };
    stage(0, 0);
    __syncthreads();
    for (int kb = 0; kb < KW; kb += GK)
    {
        const int buf = (kb / GK) & 1;
        if (kb + GK < KW) stage(buf ^ 1, kb + GK);
        const unsigned z = zany ? (st->zmask[(K0 + kb) / PW] >> ((K0 + kb) % PW)) : 0u;
#pragma unroll 4
        for (int k = 0; k < GK; ++k)
        {
            if ((z >> k) & 1u) continue;  // uniform: a zero-pivot column takes no part
            const ulonglong2 a0 = *reinterpret_cast<const ulonglong2 *>(&Ls[buf][k][4 * tr]);
            const ulonglong2 a1 = *reinterpret_cast<const ulonglong2 *>(&Ls[buf][k][64 + 4 * tr]);
            const ulonglong2 b0 = *reinterpret_cast<const ulonglong2 *>(&Us[buf][k][4 * tc]);
            const ulonglong2 b1 = *reinterpret_cast<const ulonglong2 *>(&Us[buf][k][4 * tc + 2]);
            const ulonglong2 b2 = *reinterpret_cast<const ulonglong2 *>(&Us[buf][k][64 + 4 * tc]);
            const ulonglong2 b3 = *reinterpret_cast<const ulonglong2 *>(&Us[buf][k][64 + 4 * tc + 2]);
            const f32x2 a[4] = {a0.x, a0.y, a1.x, a1.y};
            const f32x2 b[8] = {b0.x, b0.y, b1.x, b1.y, b2.x, b2.y, b3.x, b3.y};
#pragma unroll
            for (int ip = 0; ip < 4; ++ip)
#pragma unroll
                for (int jc = 0; jc < 8; ++jc) fma2(acc[ip][jc], a[ip], b[jc]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int jc = 0; jc < 8; ++jc)
    {
        if (cc[jc] >= ncl) continue;
        float *col = A + (int64_t)(cb + cc[jc]) * lda + rb;
        if (vec)
        {
#pragma unroll
            for (int h = 0; h < 2; ++h)
                *reinterpret_cast<ulonglong2 *>(col + 64 * h + 4 * tr) = make_ulonglong2(acc[2 * h][jc], acc[2 * h + 1][jc]);
        }
        else
        {
#pragma unroll
            for (int ip = 0; ip < 4; ++ip)
            {
                if (rr[2 * ip] < nr) col[rr[2 * ip]] = f2_lo(acc[ip][jc]);
                if (rr[2 * ip + 1] < nr) col[rr[2 * ip + 1]] = f2_hi(acc[ip][jc]);
            }
        }
    }
}

}  // namespace

// One matrix, m x n, m <= LARGE_MAX_ROWS.  Plain mode only for now (mode 0).
cudaError_t launch_getrf_large(float *A, int m, int n, int lda, int *ipiv, int *info, LargeStatus *st,
                               cudaStream_t stream)
{
    if (m > LARGE_MAX_ROWS || n > LARGE_MAX_COLS) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(st, 0, sizeof(LargeStatus), stream);
    if (e != cudaSuccess) return e;
    const int kmin = std::min(m, n);
    static bool attr = false;
    if (!attr)
    {
        e = cudaFuncSetAttribute(large_trsm_kernel<OB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((OB * (OB + 4) + 64 * (OB + 4)) * sizeof(float)));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(large_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    for (int K0 = 0; K0 < kmin; K0 += OB)
    {
        const int kend = std::min(kmin, K0 + OB);
        const int bend = std::min(n, K0 + OB);  // the outer block's columns
        for (int k0 = K0; k0 < kend; k0 += PW)
        {
            const int w = std::min(PW, kmin - k0);
            large_panel_kernel<true><<<CSZ, LT, 0, stream>>>(A, lda, m, k0, w, ipiv, st);
            // interchanges on every column but the panel's (which holds final values by row)
            large_swap_kernel<<<(n + 8 * SW_COLS - 1) / (8 * SW_COLS), 256, 0, stream>>>(A, lda, n, k0, -1, -1, st);
            const int jt = k0 + w;
            if (jt < bend && k0 + w < m)
            {
                large_trsm_kernel<PW><<<(bend - jt + 63) / 64, 256, (PW * (PW + 4) + 64 * (PW + 4)) * sizeof(float),
                                        stream>>>(A, lda, k0, jt, bend - jt, st);
                dim3 g((m - jt + GT - 1) / GT, (bend - jt + GT - 1) / GT);
                large_gemm_kernel<<<g, 256, GEMM_SMEM, stream>>>(A, lda, jt, m - jt, jt, bend - jt, k0, PW, st);
            }
        }
        if (bend < n && kend < m)
        {
            const int W = kend - K0;  // OB except at the end, where no columns remain
            if (W == OB)
            {
                large_trsm_kernel<OB><<<(n - bend + 63) / 64, 256, (OB * (OB + 4) + 64 * (OB + 4)) * sizeof(float),
                                        stream>>>(A, lda, K0, bend, n - bend, st);
                dim3 g((m - kend + GT - 1) / GT, (n - bend + GT - 1) / GT);
                large_gemm_kernel<<<g, 256, GEMM_SMEM, stream>>>(A, lda, kend, m - kend, bend, n - bend, K0, OB, st);
            }
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaMemcpyAsync(info, &st->info, sizeof(int), cudaMemcpyDeviceToDevice, stream);
}

}  // namespace ops_solver
