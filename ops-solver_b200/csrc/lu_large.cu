// lu_large.cu -- LU with partial pivoting of one large matrix (rows up to 8192) over the
// whole GPU: the drop-in for the reference's blocked single-matrix factorisation
// (src/sgetrf/real_lu_blocked_kernel.cpp:1469-1520, BlockedFactorLaunch::Run and its panel,
// swap/trsm, product and subtract kernels; host entry src/sgetrf/sgetrf_host.cpp:96-124).
//
// Right-looking, two-level: 32-column panels inside 128-column outer blocks.
//   * panel (a cluster of sixteen 256-thread blocks, or eight where sixteen cannot be placed;
//     up to two / four panel rows per thread): per column,
//     each block finds its candidate (warp reduction, block barrier), publishes it into
//     every block of the cluster through distributed shared memory, one cluster barrier,
//     and every block picks the same winner; rows are never moved during the panel, final
//     values are written to their rows' places and the changed positions are listed;
//   * interchanges: the panel's changed positions moved in every column of the matrix;
//   * inside the outer block: U12 = L11^-1 A12 and A22 -= L21 U12 on its columns only;
//   * once per outer block: U12 with the 128 x 128 L11 and one rank-128 update of the
//     trailing matrix (FP32 FFMA2 tiles; in mixed mode split-BF16 products on the tcgen05
//     tensor cores with the accumulator in tensor memory, lu_large_umma.cu).
// Plain mode keeps the oracle's per-element order -- every element receives fma(-l, u, a)
// in ascending k, zero-pivot columns skipped, IEEE division by the pivot -- so factors,
// pivots and info equal the unblocked order bit for bit.
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "device_once.h"
#include "launch.h"

namespace cg = cooperative_groups;

namespace ops_solver
{
namespace
{
constexpr int LT = 256;       // panel threads per block (one block per SM: up to 255 registers)
constexpr int LNW = LT / 32;  // panel warps per block
constexpr int PW = 32;        // panel width
// blocks per panel cluster: 16 where the GPU can place it, else 8 (panel_cluster_size)
constexpr int OB = 128;       // outer block
constexpr unsigned FULL = 0xffffffffu;
static_assert(32 % LNW == 0, "the block winner is read one warp report per lane group");

// Cluster exchange: every block's candidate (row and key, 144 bytes) goes to every block of
// the cluster with st.async, which completes the bytes on the receiver's mbarrier for that
// column parity; a block waits on its own barrier only (no cluster-wide barrier per column,
// so the column's global stores are never fenced).  Waits are bounded: a wait that runs out
// sets the status's error flag, and from then on no panel waits again (the factors are
// invalid and reported so), which keeps the whole factorisation's run time bounded.
constexpr unsigned CAND_BYTES = PW * sizeof(float) + sizeof(uint4);
constexpr long long WAIT_LIMIT = 1ll << 16;  // try_wait rounds (each suspends for a while)

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned cluster_addr(unsigned local, unsigned rank)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_async_v4(unsigned raddr, float4 v, unsigned rbar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(raddr),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(rbar)
                 : "memory");
}
__device__ __forceinline__ void st_async_v4u(unsigned raddr, uint4 v, unsigned rbar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(raddr),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(rbar)
                 : "memory");
}
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

template <int CS>
struct __align__(16) PanelShared
{
    float slot[2][LNW][PW];  // each warp's best row, double buffered by column parity
    uint2 key[2][LNW];       // each warp's (best key, its position)
    int krow[2][LNW];        // each warp's best row (panel-relative)
    float cand[2][CS][PW];   // each cluster block's candidate row (written by that block)
    uint4 ckey[2][CS];       // each cluster block's (key, position, row, 0)
    unsigned long long bar[2];  // per column parity: the cluster's candidates have landed
    unsigned zmask;
    int first_zero;
};

// ---------------------------------------------------------------------------------------
// panel: rows k0 .. m-1, columns k0 .. k0+w-1 of A (positions relative to k0)
// ---------------------------------------------------------------------------------------
template <bool EXACT, int NR, int CS>
__global__ void __launch_bounds__(LT, 1)
    large_panel_kernel(float *A, int lda, int m, int k0, int w, int *ipiv, LargeStatus *st)
{
    constexpr int NP = PW / 2;
    constexpr unsigned STEP_BYTES = CS * CAND_BYTES;
    constexpr int PL = 32 / CS;   // lanes of warp 0 per destination block
    constexpr int PER = PW / PL;  // candidate values each of them sends
    static_assert(PER % 4 == 0 && PER >= 4, "candidate values go out in 16-byte pieces: at least four blocks per cluster");
    __shared__ PanelShared<CS> sh;
    cg::cluster_group cluster = cg::this_cluster();
    const int c = (int)cluster.block_rank();
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int mr = m - k0;
    const int R = (mr + CS - 1) / CS;  // rows per block, at most NR * LT
    const int r0 = c * R;
    const int mine = max(0, min(R, mr - r0));  // rows of this block
    const bool active = warp * 32 < mine;      // warp-uniform: its first row is present
    float *pan = A + (int64_t)k0 * lda + k0;
    const bool pivoting = ipiv != nullptr;
    if (t == 0)
    {
        sh.zmask = 0u;
        sh.first_zero = 0;
        mbar_init(smem_addr(&sh.bar[0]), 1);
        mbar_init(smem_addr(&sh.bar[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cluster.sync();  // every block's barriers exist before any candidate is sent
    bool ok = st->error == 0;  // the same in every block: written only by earlier launches
    // thread t holds rows r0 + t + s LT (s < NR), columns in pairs, rotated by four columns
    f32x2 r[NR][NP];
    bool valid[NR];
    int pos[NR];
#pragma unroll
    for (int s = 0; s < NR; ++s)
    {
        const int i = r0 + t + s * LT;
        valid[s] = t + s * LT < mine;
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
        const int wl = w - j0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
            const int j = j0 + u;
            if (j >= w) break;  // uniform across the cluster
            const int buf = j & 1;
            float cur[NR];
#pragma unroll
            for (int s = 0; s < NR; ++s) cur[s] = (u & 1) ? f2_hi(r[s][u / 2]) : f2_lo(r[s][u / 2]);
            // this column's barrier phase: expect the cluster's candidates (the phase two
            // columns back is complete, this thread waited for it)
            if (t == 0) mbar_expect(smem_addr(&sh.bar[buf]), STEP_BYTES);
            // (1) each warp's candidate
            if (active)
            {
                unsigned key[NR];
                unsigned kmax = 0u;
#pragma unroll
                for (int s = 0; s < NR; ++s)
                {
                    if (!valid[s])
                        key[s] = 0u;
                    else if (pivoting)
                        key[s] = pos[s] == j && cur[s] != cur[s] ? 0xffffffffu : (pos[s] >= j ? pivot_key(cur[s]) : 0u);
                    else
                        key[s] = pos[s] == j ? 1u : 0u;
                    kmax = max(kmax, key[s]);
                }
                const unsigned wmax = __reduce_max_sync(FULL, kmax);
                unsigned cand = 0xffffffffu;
#pragma unroll
                for (int s = 0; s < NR; ++s)
                    if (valid[s] && key[s] == wmax) cand = min(cand, (unsigned)pos[s]);
                const unsigned wpos = __reduce_min_sync(FULL, cand);
#pragma unroll
                for (int s = 0; s < NR; ++s)
                    if (valid[s] && key[s] == wmax && (unsigned)pos[s] == wpos)
                    {
                        ulonglong2 *dst = reinterpret_cast<ulonglong2 *>(sh.slot[buf][warp]);
#pragma unroll
                        for (int q = 0; q < NP / 2; ++q)
                            if (4 * q < wl) dst[q] = make_ulonglong2(r[s][2 * q], r[s][2 * q + 1]);
                        sh.krow[buf][warp] = r0 + t + s * LT;
                    }
                if (lane == 0) sh.key[buf][warp] = make_uint2(wmax, wpos);
            }
            else if (lane == 0)
                sh.key[buf][warp] = make_uint2(0u, 0xffffffffu);
            __syncthreads();
            // (2) warp 0: the block's candidate, sent to every block of the cluster
            if (warp == 0)
            {
                const uint2 kw = sh.key[buf][lane & (LNW - 1)];
                const unsigned gmax = __reduce_max_sync(FULL, kw.x);
                const unsigned gpos = __reduce_min_sync(FULL, kw.x == gmax ? kw.y : 0xffffffffu);
                const int gw = __ffs(__ballot_sync(FULL, kw.x == gmax && kw.y == gpos)) - 1;
                const unsigned dest = lane / PL, part = lane % PL;
                const float4 *src = reinterpret_cast<const float4 *>(sh.slot[buf][gw]) + (PER / 4) * part;
                const unsigned rbar = cluster_addr(smem_addr(&sh.bar[buf]), dest);
                const unsigned rc = cluster_addr(smem_addr(&sh.cand[buf][c][PER * part]), dest);
#pragma unroll
                for (int v = 0; v < PER / 4; ++v) st_async_v4(rc + 16 * v, src[v], rbar);
                if (part == 0)
                    st_async_v4u(cluster_addr(smem_addr(&sh.ckey[buf][c]), dest),
                                 make_uint4(gmax, gpos, (unsigned)sh.krow[buf][gw], 0u), rbar);
            }
            if (ok && !mbar_wait(smem_addr(&sh.bar[buf]), (unsigned)(j >> 1) & 1u)) ok = false;
            // (3) the cluster's winner: largest key, then the smallest position
            const uint4 kc = lane < CS ? sh.ckey[buf][lane] : make_uint4(0u, 0xffffffffu, 0u, 0u);
            const unsigned gmax = __reduce_max_sync(FULL, kc.x);
            const unsigned gpos = __reduce_min_sync(FULL, kc.x == gmax ? kc.y : 0xffffffffu);
            const int gc = __ffs(__ballot_sync(FULL, kc.x == gmax && kc.y == gpos)) - 1;
            const int pr = (int)gpos;
            const float *prow = sh.cand[buf][gc];
            if (c == 0)
            {
                const int krow = (int)sh.ckey[buf][gc].z;
                if (pivoting && t == 0) ipiv[k0 + j] = k0 + pr + 1;
                if (t < w - j) pan[(int64_t)(j + t) * lda + krow] = prow[u + t];
            }
            const float d = prow[u];
            bool go[NR];
#pragma unroll
            for (int s = 0; s < NR; ++s)
            {
                pos[s] = pos[s] == j ? pr : (pos[s] == pr ? j : pos[s]);
                go[s] = valid[s] && pos[s] > j;
            }
            if (d == 0.0f)
            {
                if (c == 0 && t == 0)
                {
                    if (sh.first_zero == 0) sh.first_zero = k0 + j + 1;
                    sh.zmask |= 1u << j;
                }
#pragma unroll
                for (int s = 0; s < NR; ++s)
                    if (go[s]) pan[(int64_t)j * lda + r0 + t + s * LT] = cur[s];
            }
            else
            {
                // the reciprocal serves both: the refined modes multiply by it, the plain mode
                // divides through it (div_by: IEEE-exact)
                const float rinv = __frcp_rn(d);
                const bool dok = div_range(d);
                f32x2 nl[NR];
#pragma unroll
                for (int s = 0; s < NR; ++s)
                {
                    const float l = go[s] ? (EXACT ? div_by(cur[s], d, rinv, dok) : cur[s] * rinv) : 0.0f;
                    if (go[s]) pan[(int64_t)j * lda + r0 + t + s * LT] = l;
                    nl[s] = f2_pack(-l, -l);
                }
                const ulonglong2 *p2 = reinterpret_cast<const ulonglong2 *>(prow);
#pragma unroll
                for (int q = 0; q < NP / 2; ++q)
                {
                    if (4 * q + 3 <= u) continue;
                    if (4 * q >= wl) break;
                    const ulonglong2 v = p2[q];
#pragma unroll
                    for (int s = 0; s < NR; ++s)
                    {
                        if (4 * q + 1 > u && go[s]) fma2(r[s][2 * q], nl[s], v.x);
                        if (go[s]) fma2(r[s][2 * q + 1], nl[s], v.y);
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < NR; ++s)
        {
#pragma unroll
            for (int p = 0; p < NP - 2; ++p) r[s][p] = r[s][p + 2];
            r[s][NP - 2] = 0ull;
            r[s][NP - 1] = 0ull;
        }
    }
    __syncthreads();
    if (!ok) st->error = 1;
    cluster.sync();  // no block leaves while candidates may still be addressed to it
    // the changed positions (at most 2 w): position pos now holds physical row i
#pragma unroll
    for (int s = 0; s < NR; ++s)
    {
        const int i = r0 + t + s * LT;
        if (valid[s] && pos[s] != i)
        {
            const int at = atomicAdd(&st->nchg[k0 / PW], 1);
            if (at < 2 * PW) st->chg[k0 / PW][at] = make_int2(pos[s], i);
        }
    }
    if (c == 0 && t == 0)
    {
        st->zmask[k0 / PW] = sh.zmask;
        if (sh.first_zero && st->info == 0) st->info = sh.first_zero;
    }
}

// ---------------------------------------------------------------------------------------
// interchanges.  A panel's changed positions are moved at once only in its outer block's
// columns; the columns to the right take the outer block's four panels composed, once,
// before its U12 solve, and the L columns to the left take all later panels composed in one
// pass at the end (nothing reads them in between, so the result is LAPACK's).
// ---------------------------------------------------------------------------------------
constexpr int SW_COLS = 4;  // columns per warp

// Columns [c0, c1): panel k0's changed positions, a warp per column, all reads before writes.
__global__ void __launch_bounds__(256) large_swap_kernel(float *A, int lda, int c0, int c1, int k0,
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
    const int base = c0 + (blockIdx.x * 8 + warp) * SW_COLS;
    float v0[SW_COLS], v1[SW_COLS];
#pragma unroll
    for (int q = 0; q < SW_COLS; ++q)
    {
        const int col = base + q;
        const float *a = A + (int64_t)min(col, c1 - 1) * lda + k0;
        v0[q] = (col < c1 && dst0 >= 0) ? a[src0] : 0.0f;
        v1[q] = (col < c1 && dst1 >= 0) ? a[src1] : 0.0f;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < SW_COLS; ++q)
    {
        const int col = base + q;
        if (col >= c1) continue;
        float *a = A + (int64_t)col * lda + k0;
        if (dst0 >= 0) a[dst0] = v0[q];
        if (dst1 >= 0) a[dst1] = v1[q];
    }
}

// P[i] (i < m - R0): the row, relative to R0, that ends at position R0 + i after panels
// p0 .. p1-1 (in order); every panel's changed positions are relative to its own k0 >= R0.
__device__ void compose_panels(short *P, int m, int R0, int p0, int p1, const LargeStatus *st)
{
    const int t = threadIdx.x;
    for (int i = t; i < m - R0; i += blockDim.x) P[i] = (short)i;
    __syncthreads();
    for (int p = p0; p < p1; ++p)
    {
        const int rel = p * PW - R0;
        const int nch = min(st->nchg[p], 2 * PW);
        int2 e = make_int2(0, 0);
        short v = 0;
        if (t < nch)
        {
            e = st->chg[p][t];
            v = P[rel + e.y];
        }
        __syncthreads();
        if (t < nch) P[rel + e.x] = v;
        __syncthreads();
    }
}

// Columns [c0, c1), rows from K0: the outer block's panels (at most 4 x 64 moved positions).
constexpr int BS_PER = 4 * 2 * PW / 32;  // moved positions per lane, at most
__global__ void __launch_bounds__(256) large_block_swap_kernel(float *A, int lda, int m, int K0, int npan, int c0,
                                                               int c1, const LargeStatus *st)
{
    __shared__ short P[LARGE_MAX_ROWS];
    __shared__ int ld[4 * 2 * PW], ls[4 * 2 * PW];
    __shared__ int nl;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    compose_panels(P, m, K0, K0 / PW, K0 / PW + npan, st);
    if (t == 0) nl = 0;
    __syncthreads();
    for (int i = t; i < m - K0; i += 256)
        if (P[i] != i)
        {
            const int at = atomicAdd(&nl, 1);
            if (at < 4 * 2 * PW)
            {
                ld[at] = i;
                ls[at] = P[i];
            }
        }
    __syncthreads();
    const int nb = min(nl, 4 * 2 * PW);
    int dst[BS_PER], srcr[BS_PER];
#pragma unroll
    for (int j = 0; j < BS_PER; ++j)
    {
        const int e = lane + 32 * j;
        dst[j] = e < nb ? ld[e] : -1;
        srcr[j] = e < nb ? ls[e] : 0;
    }
    for (int col = c0 + blockIdx.x * 8 + warp; col < c1; col += gridDim.x * 8)
    {
        float *a = A + (int64_t)col * lda + K0;
        float v[BS_PER];
#pragma unroll
        for (int j = 0; j < BS_PER; ++j) v[j] = dst[j] >= 0 ? a[srcr[j]] : 0.0f;
        __syncwarp();
#pragma unroll
        for (int j = 0; j < BS_PER; ++j)
            if (dst[j] >= 0) a[dst[j]] = v[j];
        __syncwarp();
    }
}

// The L columns of panel blockIdx.x take the interchanges of every panel of the later outer
// blocks (its own block's later panels reached them through the block's column swaps): the
// composed permutation, each column gathered through a shared buffer.
__global__ void __launch_bounds__(256) large_left_swap_kernel(float *A, int lda, int m, int npanels,
                                                              const LargeStatus *st)
{
    __shared__ short P[LARGE_MAX_ROWS];
    __shared__ float buf[LARGE_MAX_ROWS];
    const int t = threadIdx.x;
    const int p = blockIdx.x;
    const int q0 = (p / (OB / PW) + 1) * (OB / PW);  // the next outer block's first panel
    const int R0 = q0 * PW;                          // rows moved by those panels start here
    if (q0 >= npanels || R0 >= m) return;            // uniform
    compose_panels(P, m, R0, q0, npanels, st);
    for (int c = p * PW; c < (p + 1) * PW; ++c)
    {
        float *a = A + (int64_t)c * lda + R0;
        for (int i = t; i < m - R0; i += 256) buf[i] = a[i];
        __syncthreads();
        for (int i = t; i < m - R0; i += 256)
            if (P[i] != i) a[i] = buf[P[i]];
        __syncthreads();
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
    const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0 && (K0 & 3) == 0;
    stage_tile(Lo, P, A + (int64_t)K0 * lda + K0, lda, W, W, vec);
    stage_tile(Ub, P, A + (int64_t)j0 * lda + K0, lda, W, nc, vec);  // columns past nc are never stored
    tile_wait();
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
    // staging: L by cp.async (16-byte chunks when aligned), U through registers (it is
    // negated and duplicated on the way), the next stage's loads in flight during this one's
    // products
    const bool lvec = vec && ((K0 & 3) == 0);
    auto stage_l = [&](int buf, int kb) {
        if (lvec)
        {
            for (int e = t; e < GK * GT / 4; e += 256)
            {
                const int k = e / (GT / 4), x = (e % (GT / 4)) * 4;
                const unsigned d = (unsigned)__cvta_generic_to_shared(&Ls[buf][k][x]);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d),
                             "l"(A + (int64_t)(K0 + kb + k) * lda + rb + x)
                             : "memory");
            }
        }
        else
        {
            for (int e = t; e < GK * GT; e += 256)
            {
                const int k = e / GT, x = e % GT;
                Ls[buf][k][x] = x < nr ? A[(int64_t)(K0 + kb + k) * lda + rb + x] : 0.0f;
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    constexpr int UPT = GK * GT / 256;  // U values per thread and stage
    float ureg[UPT];
    auto load_u = [&](int kb) {
#pragma unroll
        for (int q = 0; q < UPT; ++q)
        {
            const int e = t + q * 256, x = e / GK, k = e % GK;
            ureg[q] = x < ncl ? A[(int64_t)(cb + x) * lda + K0 + kb + k] : 0.0f;
        }
    };
    auto store_u = [&](int buf) {
#pragma unroll
        for (int q = 0; q < UPT; ++q)
        {
            const int e = t + q * 256, x = e / GK, k = e % GK;
            Us[buf][k][x] = f2_pack(-ureg[q], -ureg[q]);
        }
    };
    stage_l(0, 0);
    load_u(0);
    store_u(0);
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    for (int kb = 0; kb < KW; kb += GK)
    {
        const int buf = (kb / GK) & 1;
        const bool more = kb + GK < KW;
        if (more)
        {
            stage_l(buf ^ 1, kb + GK);
            load_u(kb + GK);
        }
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
        if (more) store_u(buf ^ 1);
        asm volatile("cp.async.wait_all;" ::: "memory");
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

// ---------------------------------------------------------------------------------------
// Mixed modes: C -= L21 U12 on the tensor cores (mma.sync m16n8k16 BF16, FP32 accumulate),
// L21 and U12 split into BF16 halves (TERMS 3: hi*hi + hi*lo + lo*hi; TERMS 1: hi*hi).  A
// 128 x 128 tile per block, warp (wm, wn) = (warp & 3, warp >> 2) owns 32 rows x 64 columns;
// K in chunks of 32 staged through registers (the next chunk's loads in flight during this
// chunk's products).  Zero-pivot columns of L are zeroed, so they take no part.
// ---------------------------------------------------------------------------------------
constexpr int MKC = 32;        // k per chunk
constexpr int MHP = MKC + 8;   // BF16 pitch (80 bytes: ldmatrix rows on distinct banks)

__device__ __forceinline__ void ldsm4(unsigned (&d)[4], const void *p)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3])
                 : "r"(a));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void split2(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

template <int TERMS>
__global__ void __launch_bounds__(256, 1) large_gemm_mixed_kernel(float *A, int lda, int r0, int rows, int c0,
                                                                  int cols, int K0, int KW, const LargeStatus *st)
{
    constexpr int NA = TERMS > 1 ? 2 : 1;  // halves kept
    extern __shared__ __align__(16) unsigned char msm[];
    __nv_bfloat16 *lh = reinterpret_cast<__nv_bfloat16 *>(msm);  // [row][k] (negated L)
    __nv_bfloat16 *ll = lh + GT * MHP;
    __nv_bfloat16 *uh = lh + NA * GT * MHP;                       // [col][k]
    __nv_bfloat16 *ul = uh + GT * MHP;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int rb = r0 + blockIdx.x * GT, cb = c0 + blockIdx.y * GT;
    const int nr = min(GT, r0 + rows - rb), ncl = min(GT, c0 + cols - cb);
    const int wr = (warp & 3) * 32, wc = (warp >> 2) * 64;
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
                const int cj = wc + ni * 8 + q * 2 + (e & 1);
                acc[mi][ni][e] = (row < nr && cj < ncl) ? A[(int64_t)(cb + cj) * lda + rb + row] : 0.0f;
            }
    // staging: thread t takes 16 L values (row x = e % 128, k = e / 128) and 16 U values
    // (column x = e / 32, k = e % 32) of each chunk
    constexpr int PER = GT * MKC / 256;
    float lv[PER], uv[PER];
    auto load = [&](int kb) {
        const unsigned z = st->zmask[(K0 + kb) / PW] >> ((K0 + kb) % PW);
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int e = t + u * 256;
            const int x = e % GT, k = e / GT;
            lv[u] = (x < nr && !((z >> k) & 1u)) ? A[(int64_t)(K0 + kb + k) * lda + rb + x] : 0.0f;
            const int xc = e / MKC, kc = e % MKC;
            uv[u] = xc < ncl ? A[(int64_t)(cb + xc) * lda + K0 + kb + kc] : 0.0f;
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int e = t + u * 256;
            const int x = e % GT, k = e / GT;
            __nv_bfloat16 h, l;
            split2(-lv[u], h, l);
            lh[x * MHP + k] = h;
            if (TERMS > 1) ll[x * MHP + k] = l;
            const int xc = e / MKC, kc = e % MKC;
            split2(uv[u], h, l);
            uh[xc * MHP + kc] = h;
            if (TERMS > 1) ul[xc * MHP + kc] = l;
        }
    };
    load(0);
    for (int kb = 0; kb < KW; kb += MKC)
    {
        __syncthreads();  // the previous chunk's products are done with the tiles
        store();
        __syncthreads();
        if (kb + MKC < KW) load(kb + MKC);
#pragma unroll
        for (int ks = 0; ks < MKC / 16; ++ks)
        {
            unsigned ah[2][4], al[2][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
            {
                const int row = wr + mi * 16 + (lane & 15);
                const int kk = ks * 16 + (lane >> 4) * 8;
                ldsm4(ah[mi], lh + row * MHP + kk);
                if (TERMS > 1) ldsm4(al[mi], ll + row * MHP + kk);
            }
#pragma unroll
            for (int np = 0; np < 4; ++np)
            {
                const int mt = lane >> 3, rr = lane & 7;
                const int col = wc + np * 16 + (mt >> 1) * 8 + rr;
                const int kk = ks * 16 + (mt & 1) * 8;
                unsigned bh[4], bl[4];
                ldsm4(bh, uh + col * MHP + kk);
                if (TERMS > 1) ldsm4(bl, ul + col * MHP + kk);
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ni = np * 2 + h;
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
                    {
                        if (TERMS > 1)
                        {
                            mma16816(acc[mi][ni], al[mi], bh[2 * h], bh[2 * h + 1]);
                            mma16816(acc[mi][ni], ah[mi], bl[2 * h], bl[2 * h + 1]);
                        }
                        mma16816(acc[mi][ni], ah[mi], bh[2 * h], bh[2 * h + 1]);
                    }
                }
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
                const int cj = wc + ni * 8 + q * 2 + (e & 1);
                if (row < nr && cj < ncl) A[(int64_t)(cb + cj) * lda + rb + row] = acc[mi][ni][e];
            }
}

template <int TERMS>
constexpr size_t mixed_gemm_smem()
{
    return (size_t)2 * (TERMS > 1 ? 2 : 1) * GT * MHP * sizeof(__nv_bfloat16);
}

// info = the first zero pivot, or LARGE_WAIT_ERROR when a panel's bounded wait ran out
__global__ void large_info_kernel(int *info, const LargeStatus *st) { *info = st->error ? LARGE_WAIT_ERROR : st->info; }

}  // namespace

namespace
{
template <bool EXACT, int NR, int CS>
cudaError_t panel_launch_cs(float *A, int lda, int m, int k0, int w, int *ipiv, LargeStatus *st, cudaStream_t stream)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CS);
    cfg.blockDim = dim3(LT);
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CS;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, large_panel_kernel<EXACT, NR, CS>, A, lda, m, k0, w, ipiv, st);
}

// The cluster size: 16 blocks (two panel rows per thread at 8192) when the device can place
// such a cluster of this kernel, otherwise the portable 8.
int query_cluster_size()
{
    int cs = 8;
    const void *fn = reinterpret_cast<const void *>(large_panel_kernel<true, 2, 16>);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
        cudaFuncSetAttribute(reinterpret_cast<const void *>(large_panel_kernel<false, 2, 16>),
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
        cudaFuncSetAttribute(reinterpret_cast<const void *>(large_panel_kernel<true, 1, 16>),
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
        cudaFuncSetAttribute(reinterpret_cast<const void *>(large_panel_kernel<false, 1, 16>),
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(16);
        cfg.blockDim = dim3(LT);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 16;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) == cudaSuccess && clusters >= 1) cs = 16;
    }
    cudaGetLastError();  // a refused query leaves no error behind
    return cs;
}

// ... asked once per device (the non-portable size attribute is set per device).
int panel_cluster_size()
{
    static std::atomic<int> cache[ONCE_MAX_DEVICES];
    return value_per_device(cache, query_cluster_size);
}

template <bool EXACT>
cudaError_t panel_launch(float *A, int lda, int m, int k0, int w, int *ipiv, LargeStatus *st, cudaStream_t stream)
{
    const int cs = panel_cluster_size();
    const int per = ((m - k0 + cs - 1) / cs + LT - 1) / LT;  // rows per thread
    if (cs == 16)
        return per <= 1 ? panel_launch_cs<EXACT, 1, 16>(A, lda, m, k0, w, ipiv, st, stream)
                        : panel_launch_cs<EXACT, 2, 16>(A, lda, m, k0, w, ipiv, st, stream);
    if (per <= 1) return panel_launch_cs<EXACT, 1, 8>(A, lda, m, k0, w, ipiv, st, stream);
    if (per == 2) return panel_launch_cs<EXACT, 2, 8>(A, lda, m, k0, w, ipiv, st, stream);
    if (per == 3) return panel_launch_cs<EXACT, 3, 8>(A, lda, m, k0, w, ipiv, st, stream);
    return panel_launch_cs<EXACT, 4, 8>(A, lda, m, k0, w, ipiv, st, stream);
}

void gemm_launch(int mode, float *A, int lda, int r0, int rows, int c0, int cols, int K0, int KW, LargeStatus *st,
                 cudaStream_t stream)
{
    dim3 g((rows + GT - 1) / GT, (cols + GT - 1) / GT);
    if (mode == 0)
        large_gemm_kernel<<<g, 256, GEMM_SMEM, stream>>>(A, lda, r0, rows, c0, cols, K0, KW, st);
    else if (mode == 1)
        large_gemm_mixed_kernel<1><<<g, 256, mixed_gemm_smem<1>(), stream>>>(A, lda, r0, rows, c0, cols, K0, KW, st);
    else
        large_gemm_mixed_kernel<3><<<g, 256, mixed_gemm_smem<3>(), stream>>>(A, lda, r0, rows, c0, cols, K0, KW, st);
}
}  // namespace

// One matrix, m x n, n <= m <= LARGE_MAX_ROWS; mode 0 plain FP32 (the oracle's order), 1 BF16,
// 3 split BF16 trailing updates (pivot search by packed key, reciprocal multiply).
namespace
{
// Look-ahead streams of one device: the panel chain runs on a high-priority stream, the bulk
// of each outer block's trailing update on a low-priority one, forked from and joined back to
// the caller's stream with events (capturable).  Created on first use, kept for the process;
// calls from several host threads enqueue one at a time (their work then runs in order).
struct LookAhead
{
    cudaStream_t hi = nullptr, lo = nullptr;
    cudaEvent_t fork = nullptr, part_a = nullptr, part_b = nullptr, join_hi = nullptr, join_lo = nullptr;
};
cudaError_t look_ahead(LookAhead *&out)
{
    static LookAhead devs[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    LookAhead &la = devs[dev];
    if (!la.hi)
    {
        int least = 0, greatest = 0;
        e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&la.hi, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&la.lo, cudaStreamNonBlocking, least);
        cudaEvent_t *evs[5] = {&la.fork, &la.part_a, &la.part_b, &la.join_hi, &la.join_lo};
        for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(evs[i], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    out = &la;
    return cudaSuccess;
}
}  // namespace

cudaError_t launch_getrf_large(float *A, int m, int n, int lda, int *ipiv, int *info, LargeStatus *st, int mode,
                               cudaStream_t stream, void *umma_scratch)
{
    if (m > LARGE_MAX_ROWS || n > LARGE_MAX_COLS) return cudaErrorInvalidValue;
    const int kmin = std::min(m, n);
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        cudaError_t r = cudaFuncSetAttribute(large_trsm_kernel<OB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)((OB * (OB + 4) + 64 * (OB + 4)) * sizeof(float)));
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(large_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        return r;
    });
    if (e != cudaSuccess) return e;
    static std::mutex enqueue;
    std::lock_guard<std::mutex> lock(enqueue);
    LookAhead *la = nullptr;
    e = look_ahead(la);
    if (e != cudaSuccess) return e;
    cudaStream_t hs = la->hi, ls = la->lo;
    e = cudaEventRecord(la->fork, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hs, la->fork, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ls, la->fork, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(st, 0, sizeof(LargeStatus), hs);
    if (e != cudaSuccess) return e;
    const bool tcgen = mode != 0 && umma_scratch;
    for (int K0 = 0; K0 < kmin; K0 += OB)
    {
        const int kend = std::min(kmin, K0 + OB);
        const int bend = std::min(n, K0 + OB);  // the outer block's columns
        for (int k0 = K0; k0 < kend; k0 += PW)
        {
            const int w = std::min(PW, kmin - k0);
            e = mode == 0 ? panel_launch<true>(A, lda, m, k0, w, ipiv, st, hs)
                          : panel_launch<false>(A, lda, m, k0, w, ipiv, st, hs);
            if (e != cudaSuccess) return e;
            // the outer block's columns (the panel's included: it holds final values by row)
            large_swap_kernel<<<(bend - K0 + 8 * SW_COLS - 1) / (8 * SW_COLS), 256, 0, hs>>>(A, lda, K0, bend, k0, st);
            const int jt = k0 + w;
            if (jt < bend && k0 + w < m)
            {
                large_trsm_kernel<PW><<<(bend - jt + 63) / 64, 256, (PW * (PW + 4) + 64 * (PW + 4)) * sizeof(float),
                                        hs>>>(A, lda, k0, jt, bend - jt, st);
                gemm_launch(mode, A, lda, jt, m - jt, jt, bend - jt, k0, PW, st, hs);
            }
        }
        if (bend < n)
        {
            // the previous block's update of these columns is complete; then this block's
            // interchanges on the columns to its right, its U12, and its update: the next
            // block's columns on the high-priority stream (its panels follow at once), the
            // rest on the low-priority stream while those panels run
            e = cudaStreamWaitEvent(hs, la->part_b, 0);
            if (e != cudaSuccess) return e;
            large_block_swap_kernel<<<std::min(148, (n - bend + 7) / 8), 256, 0, hs>>>(
                A, lda, m, K0, (kend - K0 + PW - 1) / PW, bend, n, st);
            if (kend < m && kend - K0 == OB)
            {
                large_trsm_kernel<OB><<<(n - bend + 63) / 64, 256, (OB * (OB + 4) + 64 * (OB + 4)) * sizeof(float),
                                        hs>>>(A, lda, K0, bend, n - bend, st);
                const int split = std::min(n, bend + OB);
                if (tcgen)
                {
                    e = launch_umma_split(A, lda, m, n, K0, kend, bend, st, umma_scratch, hs);
                    if (e == cudaSuccess)
                        e = launch_umma_range(A, lda, m, n, kend, bend, bend, split, mode == 1 ? 1 : 3, st,
                                              umma_scratch, hs);
                }
                else
                    gemm_launch(mode, A, lda, kend, m - kend, bend, split - bend, K0, OB, st, hs);
                if (e == cudaSuccess) e = cudaEventRecord(la->part_a, hs);
                if (e == cudaSuccess && split < n)
                {
                    e = cudaStreamWaitEvent(ls, la->part_a, 0);
                    if (e == cudaSuccess)
                    {
                        if (tcgen)
                            e = launch_umma_range(A, lda, m, n, kend, bend, split, n, mode == 1 ? 1 : 3, st,
                                                  umma_scratch, ls);
                        else
                            gemm_launch(mode, A, lda, kend, m - kend, split, n - split, K0, OB, st, ls);
                    }
                    if (e == cudaSuccess) e = cudaEventRecord(la->part_b, ls);
                }
                if (e != cudaSuccess) return e;
            }
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    e = cudaStreamWaitEvent(hs, la->part_b, 0);
    if (e != cudaSuccess) return e;
    // every panel's L columns take the later panels' interchanges
    const int npanels = (kmin + PW - 1) / PW;
    if (npanels > 1) large_left_swap_kernel<<<npanels - 1, 256, 0, hs>>>(A, lda, m, npanels, st);
    large_info_kernel<<<1, 1, 0, hs>>>(info, st);
    // join both streams back into the caller's
    e = cudaEventRecord(la->join_hi, hs);
    if (e == cudaSuccess) e = cudaEventRecord(la->join_lo, ls);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, la->join_hi, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, la->join_lo, 0);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace ops_solver
