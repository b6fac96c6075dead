// qr.cu -- the real QR family: Householder factorisation (Sgeqrf), application of Q or Q^T
// from either side (Sormqr), explicit Q (Sorgqr) and least squares (SSgels).
//
// Reflectors follow LAPACK's convention, as the reference's CPU golden does
// (src/sgeqrf/kernel/householder.hpp:55-141, Larfg): beta = -sign(alpha) ||x||,
// tau = (beta - alpha) / beta, v = x2 / (alpha - beta), tau = 0 for an all-zero x2.  The
// schedule is this build's: 32-column panels, the slarft block factor T, and block
// application C -= V op(T) (V^T C).  Every reduction over rows is a "lane sum": row r feeds
// lane r mod 32 (an FMA chain in ascending row order), and a warp butterfly
// (v += shfl_xor(v, off), off = 16 .. 1) combines the lanes, so the results do not depend
// on the grid and the CPU oracle restates them exactly:
//   qr_panel_kernel /    one block factors a panel in shared memory, or an eight-block cluster
//   qr_cluster_panel_kernel   a taller one: per column, warp 0 sums the squares and the other
//                        warps the products with their columns at once, then the reflector
//   qr_gram_kernel /     T of the panel (forward, columnwise): the reflector products one warp
//   qr_tri_kernel        per pair across the grid, then slarft's recurrence in one warp
//   qr_apply_kernel      one warp per column (left) or row (right) of C: W = V^T c by lane
//                        sums over 128-row chunks of V double-buffered in shared memory,
//                        W2 = op(T) W, then c -= V W2 with an FMA chain over the reflectors
//   qr_trsv_kernel       R X = Y, one block per right-hand side, 32-column blocks from the bottom
//   xlarft_gram_kernel / xlarft_tri_kernel   Xlarft: the reflector products over 32 x 32
//                        blocks, then slarft's recurrence on a packed triangle (k <= 256)
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "device_once.h"
#include "launch_qr.h"
#include "lookahead.h"

namespace ops_solver
{
namespace
{
constexpr int NB = 32;
constexpr int PANEL_THREADS = 1024;
constexpr int APPLY_WARPS = 8;

__device__ __forceinline__ float lane_fold(float p)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) p = add_rn(p, __shfl_xor_sync(0xffffffffu, p, off));
    return p;
}

// Panel columns [k, k + kb) of rows [k, m), staged in shared memory (pitch m - k).  Per column
// c, every reduction over the rows below c is taken at once from the column as it stands:
// warp 0 forms sumsq = sum x_i^2 and warp w >= 1 forms S_j = sum x_i A(i, j) for column
// j = c + w (lane sums), in parallel.  After one barrier every thread forms beta, tau and
// scale = 1 / (alpha - beta) (the same operations on the same values, so no second barrier);
// warp w applies w_j = tau fma(scale, S_j, A(c, j)) with v_i = x_i scale (v_c = 1) formed on
// the fly; column c itself is scaled, and beta stored, during the next column's reductions.
constexpr int PANEL_SMEM_FLOATS = 50 * 1024;

__global__ void __launch_bounds__(PANEL_THREADS) qr_panel_kernel(float *A, int lda, int m, int k, int kb, float *tau)
{
    extern __shared__ float sp[];
    __shared__ float s_sumsq, s_alpha, s_S[NB];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int H = m - k;
    auto at = [&](int j, int row) -> float & { return sp[(j - k) * H + (row - k)]; };
    for (int idx = tid; idx < H * kb; idx += PANEL_THREADS) sp[idx] = A[(int64_t)(k + idx / H) * lda + k + idx % H];
    __syncthreads();
    bool prev_apply = false;
    float prev_scale = 0.0f, prev_beta = 0.0f;
    for (int c = k; c < k + kb; ++c)
    {
        if (prev_apply)  // column c - 1 becomes its reflector, beta its diagonal entry
        {
            if (tid == 0) at(c - 1, c - 1) = prev_beta;
            for (int row = c + tid; row < m; row += PANEL_THREADS) at(c - 1, row) = mul_rn(at(c - 1, row), prev_scale);
        }
        const int j = c + warp;
        if (m - c > 1 && j < k + kb)
        {
            float p = 0.0f;
#pragma unroll 4
            for (int row = c + 1 + lane; row < m; row += 32) p = fma_rn(at(c, row), at(j, row), p);
            const float part = lane_fold(p);
            if (lane == 0)
            {
                if (warp == 0)
                {
                    s_sumsq = part;
                    s_alpha = at(c, c);
                }
                else
                    s_S[warp] = part;
            }
        }
        __syncthreads();
        // every thread forms the reflector's scalars (the same operations on the same values)
        float t = 0.0f, scale = 0.0f, beta = 0.0f;
        const bool apply = m - c > 1 && s_sumsq != 0.0f;
        if (apply)
        {
            const float alpha = s_alpha;
            const float norm = sqrt_rn(add_rn(mul_rn(alpha, alpha), s_sumsq));
            beta = alpha >= 0.0f ? -norm : norm;
            t = div_rn(sub_rn(beta, alpha), beta);
            scale = div_rn(1.0f, sub_rn(alpha, beta));
        }
        if (tid == 0) tau[c] = t;
        if (apply && warp >= 1 && j < k + kb)
        {
            const float w = mul_rn(t, fma_rn(scale, s_S[warp], at(j, c)));
            __syncwarp();
            if (lane == 0) at(j, c) = fma_rn(-w, 1.0f, at(j, c));
#pragma unroll 4
            for (int row = c + 1 + lane; row < m; row += 32)
                at(j, row) = fma_rn(-w, mul_rn(at(c, row), scale), at(j, row));
        }
        prev_apply = apply;
        prev_scale = scale;
        prev_beta = beta;
        __syncthreads();
    }
    if (prev_apply)
    {
        if (tid == 0) at(k + kb - 1, k + kb - 1) = prev_beta;
        for (int row = k + kb + tid; row < m; row += PANEL_THREADS)
            at(k + kb - 1, row) = mul_rn(at(k + kb - 1, row), prev_scale);
    }
    __syncthreads();
    for (int idx = tid; idx < H * kb; idx += PANEL_THREADS) A[(int64_t)(k + idx / H) * lda + k + idx % H] = sp[idx];
}

// Rows per block of a panel spread over a cluster (0: the panel fits one block, or is too
// tall for eight): ceil((m - k) / 8) rounded up to a multiple of 32.  The CPU oracle reduces
// with the same segments.
__host__ __device__ inline int panel_seg(int H, int kb, int budget)
{
    if ((int64_t)H * kb <= budget) return 0;
    const int seg = ((H + 7) / 8 + 31) & ~31;
    return (int64_t)seg * kb <= budget ? seg : 0;
}

// A tall panel over a cluster of ceil((m - k) / seg) blocks: block g holds rows
// [k + g seg, k + (g + 1) seg) of the kb columns in shared memory and runs the one-block
// schedule on them.  The reductions are lane sums per block, folded and published (with the
// rows of column c's diagonal entry, which block 0 holds) in shared memory double-buffered
// by column parity; after one cluster barrier per column every block adds the published
// totals in ascending block order through distributed shared memory, so all blocks derive
// the same reflector and the same column weights.
__global__ void __launch_bounds__(PANEL_THREADS) qr_cluster_panel_kernel(float *A, int lda, int m, int k, int kb,
                                                                         int seg, float *tau)
{
    namespace cg = cooperative_groups;
    extern __shared__ float sp[];  // sp[(j - k) * seg + (row - r0)]
    __shared__ float pub_sumsq[2], pub_S[2][NB], pub_row[2][NB];
    cg::cluster_group cluster = cg::this_cluster();
    const int g = (int)cluster.block_rank(), G = (int)cluster.num_blocks();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = k + g * seg, r1 = min(m, r0 + seg);
    const int rows = max(0, r1 - r0);
    auto at = [&](int j, int row) -> float & { return sp[(j - k) * seg + (row - r0)]; };
    // the blocks' totals in ascending block order: lane q fetches block q's, every lane adds
    auto total = [&](float *mine) -> float
    {
        const float part = lane < G ? *cluster.map_shared_rank(mine, lane) : 0.0f;
        float sum = __shfl_sync(0xffffffffu, part, 0);
        for (int q = 1; q < G; ++q) sum = add_rn(sum, __shfl_sync(0xffffffffu, part, q));
        return sum;
    };
    for (int idx = tid; idx < rows * kb; idx += PANEL_THREADS)
        sp[(idx / rows) * seg + idx % rows] = A[(int64_t)(k + idx / rows) * lda + r0 + idx % rows];
    __syncthreads();
    bool prev_apply = false;
    float prev_scale = 0.0f, prev_beta = 0.0f;
    for (int c = k; c < k + kb; ++c)
    {
        const int par = c & 1, owner = (c - k) / seg;
        if (prev_apply)  // column c - 1 becomes its reflector, beta its diagonal entry
        {
            if (tid == 0 && c - 1 >= r0 && c - 1 < r1) at(c - 1, c - 1) = prev_beta;
            for (int row = max(r0, c) + tid; row < r1; row += PANEL_THREADS)
                at(c - 1, row) = mul_rn(at(c - 1, row), prev_scale);
        }
        const int j = c + warp;
        if (j < k + kb)
        {
            float p = 0.0f;
#pragma unroll 4
            for (int row = max(r0, c + 1) + lane; row < r1; row += 32) p = fma_rn(at(c, row), at(j, row), p);
            const float part = lane_fold(p);
            if (lane == 0)
            {
                if (warp == 0)
                    pub_sumsq[par] = part;
                else
                    pub_S[par][warp] = part;
                if (g == owner) pub_row[par][warp] = at(j, c);
            }
        }
        cluster.sync();
        // every warp forms the reflector's scalars (the same operations on the same values)
        const float sumsq = total(&pub_sumsq[par]);
        const bool apply = m - c > 1 && sumsq != 0.0f;
        float t = 0.0f, scale = 0.0f, beta = 0.0f;
        if (apply)
        {
            const float alpha = *cluster.map_shared_rank(&pub_row[par][0], owner);
            const float norm = sqrt_rn(add_rn(mul_rn(alpha, alpha), sumsq));
            beta = alpha >= 0.0f ? -norm : norm;
            t = div_rn(sub_rn(beta, alpha), beta);
            scale = div_rn(1.0f, sub_rn(alpha, beta));
        }
        if (tid == 0 && g == 0) tau[c] = t;
        if (apply && warp >= 1 && j < k + kb)
        {
            const float S = total(&pub_S[par][warp]);
            const float acj = *cluster.map_shared_rank(&pub_row[par][warp], owner);
            const float w = mul_rn(t, fma_rn(scale, S, acj));
            if (lane == 0 && g == owner) at(j, c) = fma_rn(-w, 1.0f, acj);
#pragma unroll 4
            for (int row = max(r0, c + 1) + lane; row < r1; row += 32)
                at(j, row) = fma_rn(-w, mul_rn(at(c, row), scale), at(j, row));
        }
        prev_apply = apply;
        prev_scale = scale;
        prev_beta = beta;
        __syncthreads();
    }
    if (prev_apply)
    {
        if (tid == 0 && k + kb - 1 >= r0 && k + kb - 1 < r1) at(k + kb - 1, k + kb - 1) = prev_beta;
        for (int row = max(r0, k + kb) + tid; row < r1; row += PANEL_THREADS)
            at(k + kb - 1, row) = mul_rn(at(k + kb - 1, row), prev_scale);
    }
    cluster.sync();  // no block leaves while another may still read what it published
    for (int idx = tid; idx < rows * kb; idx += PANEL_THREADS)
        A[(int64_t)(k + idx / rows) * lda + r0 + idx % rows] = sp[(idx / rows) * seg + idx % rows];
}

// The reflector Gram products of a panel for slarft: d(i, r) = -tau_i (v_r . v_i) for r < i,
// one warp per pair, each a lane sum in ascending rows, stored below T's diagonal
// (T[r * NB + i]); qr_tri_kernel then forms T's upper triangle from them.
constexpr int GRAM_WARPS = 8;

__global__ void __launch_bounds__(GRAM_WARPS * 32) qr_gram_kernel(const float *A, int lda, int nq, int k, int kb,
                                                                  const float *tau, float *T)
{
    const int lane = threadIdx.x & 31;
    const int pr = blockIdx.x * GRAM_WARPS + (threadIdx.x >> 5);
    if (pr >= kb * (kb - 1) / 2) return;
    int i = 1, r = pr;
    while (r >= i)
    {
        r -= i;
        ++i;
    }
    const float *vr = A + (int64_t)(k + r) * lda, *vi = A + (int64_t)(k + i) * lda;
    const int first = k + i;
    constexpr int U = 16;
    float p = 0.0f;
    for (int base = first & ~31; base < nq; base += 32 * U)
    {
        float a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int row = base + 32 * u + lane;
            const bool ok = row >= first && row < nq;
            a[u] = ok ? vr[row] : 0.0f;
            b[u] = ok ? (row == first ? 1.0f : vi[row]) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int row = base + 32 * u + lane;
            if (row >= first && row < nq) p = fma_rn(a[u], b[u], p);
        }
    }
    const float dot = lane_fold(p);
    if (lane == 0) T[r * NB + i] = mul_rn(-tau[k + i], dot);
}

// T (kb x kb upper, column-major, ld NB): T(i, i) = tau_i, T(0:i, i) = T(0:i, 0:i) d(i, 0:i)
// (an FMA chain in ascending q), a zero column where tau_i = 0.  Lane r keeps row r of T in
// registers.
__global__ void __launch_bounds__(32) qr_tri_kernel(int k, int kb, const float *tau, float *T)
{
    __shared__ float d[NB][NB];  // d[i][q] = d(i, q)
    const int r = threadIdx.x;
    for (int i = 0; i < kb; ++i)
        if (r < i) d[i][r] = T[r * NB + i];
    __syncwarp();
    float tr[NB];  // tr[q] = T(r, q)
#pragma unroll
    for (int i = 0; i < NB; ++i)
    {
        tr[i] = 0.0f;
        if (i < kb)
        {
            const float ti = tau[k + i];
            if (ti != 0.0f)
            {
                if (r == i)
                    tr[i] = ti;
                else if (r < i)
                {
                    float acc = 0.0f;
#pragma unroll
                    for (int q = 0; q < i; ++q)
                        if (q >= r) acc = fma_rn(tr[q], d[i][q], acc);
                    tr[i] = acc;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i)
        if (i < kb && r <= i) T[i * NB + r] = tr[i];
}

// C = C - V op(T) (V^T C) (LEFT: one warp per column of C, reflector index = C's row) or
// C = C - (C V) op(T) V^T (RIGHT: one warp per row of C, reflector index = C's column).
// LOWER_CHAIN: W2[i] = sum_{q <= i} T(q, i) W[q] (op(T) = T^T for LEFT, T for RIGHT);
// otherwise W2[i] = sum_{q >= i} T(i, q) W[q].
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <bool RIGHT, bool LOWER_CHAIN>
__global__ void __launch_bounds__(APPLY_WARPS * 32, 3) qr_apply_kernel(const float *V, int ldv, int nq, int k, int kb,
                                                                       const float *T, float *C, int64_t ldc,
                                                                       int count)
{
    constexpr int ROWS = 128;   // four 32-row chunks of V per pass
    constexpr int VP = NB + 4;  // row pitch: 16-byte aligned rows, conflict-free 128-bit reads
    constexpr int CU = ROWS / 32;
    // V is double-buffered: the next pass's rows are copied (cp.async) while this pass computes.
    // The raw reflector store is staged; the unit diagonal and the zeros above it are applied
    // when the first 32 rows are read.
    __shared__ __align__(16) float vs[2][ROWS][VP];
    __shared__ float ts[NB * NB];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j = blockIdx.x * APPLY_WARPS + warp;  // column (LEFT) or row (RIGHT) of C
    const bool live = j < count;
    for (int idx = tid; idx < NB * NB; idx += APPLY_WARPS * 32) ts[idx] = T[idx];
    auto cat = [&](int row) -> float * { return RIGHT ? C + (int64_t)row * ldc + j : C + (int64_t)j * ldc + row; };
    auto stage = [&](int base0, int b)
    {
        if (base0 < nq)
            for (int idx = tid; idx < ROWS * kb; idx += APPLY_WARPS * 32)
            {
                const int rr = idx % ROWS, i = idx / ROWS, row = base0 + rr;
                if (row < nq) cp_async4(&vs[b][rr][i], V + (int64_t)(k + i) * ldv + row);
            }
        cp_async_commit();
    };
    auto load_c = [&](int base0, float *c)
    {
#pragma unroll
        for (int u = 0; u < CU; ++u)
        {
            const int row = base0 + 32 * u + lane;
            c[u] = live && row >= k && row < nq ? *cat(row) : 0.0f;
        }
    };
    const int first = k & ~31;
    float p[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) p[i] = 0.0f;
    float c[CU];
    stage(first, 0);
    load_c(first, c);
    int b = 0;
    for (int base0 = first; base0 < nq; base0 += ROWS, b ^= 1)
    {
        stage(base0 + ROWS, b ^ 1);
        float cn[CU];
        load_c(base0 + ROWS, cn);
        cp_async_wait_prior();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u)  // chunks in ascending row order
        {
            const int row = base0 + 32 * u + lane;
            if (live && kb == NB && row >= k + NB && row < nq)  // below every reflector's unit entry
            {
#pragma unroll
                for (int i = 0; i < NB; i += 4)
                {
                    const float4 v = *reinterpret_cast<const float4 *>(&vs[b][32 * u + lane][i]);
                    p[i] = fma_rn(v.x, c[u], p[i]);
                    p[i + 1] = fma_rn(v.y, c[u], p[i + 1]);
                    p[i + 2] = fma_rn(v.z, c[u], p[i + 2]);
                    p[i + 3] = fma_rn(v.w, c[u], p[i + 3]);
                }
            }
            else if (live && row >= k && row < nq)
            {
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    if (i < kb && row >= k + i)
                        p[i] = fma_rn(row == k + i ? 1.0f : vs[b][32 * u + lane][i], c[u], p[i]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u) c[u] = cn[u];
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) p[i] = lane_fold(p[i]);
    float w2[NB];  // W2 = op(T) W, lane i forming entry i, then shared across the warp
    {
        float acc = 0.0f;
#pragma unroll
        for (int q = 0; q < NB; ++q)
        {
            if (LOWER_CHAIN)
            {
                if (q <= lane && lane < kb) acc = fma_rn(ts[lane * NB + q], p[q], acc);
            }
            else
            {
                if (q >= lane && q < kb) acc = fma_rn(ts[q * NB + lane], p[q], acc);
            }
        }
#pragma unroll
        for (int i = 0; i < NB; ++i) w2[i] = __shfl_sync(0xffffffffu, acc, i);
    }
    stage(first, 0);
    load_c(first, c);
    b = 0;
    for (int base0 = first; base0 < nq; base0 += ROWS, b ^= 1)
    {
        stage(base0 + ROWS, b ^ 1);
        float cn[CU];
        load_c(base0 + ROWS, cn);
        cp_async_wait_prior();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u)
        {
            const int row = base0 + 32 * u + lane;
            if (live && kb == NB && row >= k + NB && row < nq)
            {
                float x = c[u];
#pragma unroll
                for (int i = 0; i < NB; i += 4)
                {
                    const float4 v = *reinterpret_cast<const float4 *>(&vs[b][32 * u + lane][i]);
                    x = fma_rn(-v.x, w2[i], x);
                    x = fma_rn(-v.y, w2[i + 1], x);
                    x = fma_rn(-v.z, w2[i + 2], x);
                    x = fma_rn(-v.w, w2[i + 3], x);
                }
                *cat(row) = x;
            }
            else if (live && row >= k && row < nq)
            {
                float x = c[u];
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    if (i < kb && i <= row - k) x = fma_rn(-(row == k + i ? 1.0f : vs[b][32 * u + lane][i]), w2[i], x);
                *cat(row) = x;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u) c[u] = cn[u];
    }
}

// R X = Y for one right-hand side per block, in 32-column blocks from the bottom: warp 0
// solves the diagonal block with the right-hand side in its lanes (x_p = x_p / R_pp, then
// x_i -= R_ip x_p, p descending, R's block columns preloaded in registers), then every
// thread applies the block's columns to the rows above it, p descending.  Each x_i receives
// its updates in descending p, as a column sweep would.
__global__ void __launch_bounds__(1024) qr_trsv_kernel(const float *R, int ldr, int n, const float *Y, int ldy,
                                                       float *X, int ldx)
{
    extern __shared__ float xs[];
    const int j = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < n; i += blockDim.x) xs[i] = Y[(int64_t)j * ldy + i];
    __syncthreads();
    for (int c0 = (n - 1) & ~31; c0 >= 0; c0 -= 32)
    {
        const int cw = min(32, n - c0);
        if (tid < 32)
        {
            float r[32];
#pragma unroll
            for (int q = 0; q < 32; ++q)
                r[q] = lane < cw && q < cw ? R[(int64_t)(c0 + q) * ldr + c0 + lane] : 1.0f;
            float x = lane < cw ? xs[c0 + lane] : 0.0f;
#pragma unroll
            for (int q = 31; q >= 0; --q)
            {
                if (q < cw && lane == q) x = div_rn(x, r[q]);
                const float xp = __shfl_sync(0xffffffffu, x, q);
                if (q < cw && lane < q) x = fma_rn(-r[q], xp, x);
            }
            if (lane < cw) xs[c0 + lane] = x;
        }
        __syncthreads();
        for (int i = tid; i < c0; i += blockDim.x)
        {
            float x = xs[i];
            for (int q = cw - 1; q >= 0; --q) x = fma_rn(-R[(int64_t)(c0 + q) * ldr + i], xs[c0 + q], x);
            xs[i] = x;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += blockDim.x) X[(int64_t)j * ldx + i] = xs[i];
}

// Reflector products for Xlarft: G(r, i) = lane sum over the rows both reflectors share of
// v_r . v_i, for the pairs r < i (forward: v_i's unit at row i, rows [i, n)) or r > i
// (backward: unit at row n-k+i, rows [0, n-k+i]).  Block (rb, ib) covers r in [32 rb, +32),
// i in [32 ib, +32); warp w owns i = 32 ib + w, lane t's accumulator t owns r = 32 rb + t;
// 32-row chunks of both column blocks are staged in shared memory.
template <bool BACKWARD>
__global__ void __launch_bounds__(1024) xlarft_gram_kernel(const float *V, int ldv, int n, int k, float *G)
{
    __shared__ float vr[32][33], vi[32][33];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    if (BACKWARD ? r0 + 31 <= i0 : r0 >= i0 + 31) return;  // no pair of this block is referenced
    const int i = i0 + warp;
    const int unit_i = BACKWARD ? n - k + i : i;
    int lo, hi;  // rows any pair of the block reads
    if (BACKWARD)
    {
        lo = 0;
        hi = min(n - 1, n - k + min(i0 + 31, k - 1));
    }
    else
    {
        lo = i0 & ~31;
        hi = n - 1;
    }
    float p[32];
#pragma unroll
    for (int t = 0; t < 32; ++t) p[t] = 0.0f;
    for (int base = lo & ~31; base <= hi; base += 32)
    {
        __syncthreads();
        {
            const int rr = tid & 31, cc = tid >> 5, row = base + rr;
            const int cr = r0 + cc, ci = i0 + cc;
            vr[rr][cc] = row < n && cr < k ? V[(int64_t)cr * ldv + row] : 0.0f;
            float x = 0.0f;
            if (row < n && ci < k)
            {
                const int u = BACKWARD ? n - k + ci : ci;
                x = row == u ? 1.0f : V[(int64_t)ci * ldv + row];
            }
            vi[rr][cc] = x;
        }
        __syncthreads();
        const int row = base + lane;
        const bool in_rows = i < k && row < n && (BACKWARD ? row <= unit_i : row >= unit_i);
        if (in_rows)
        {
            const float x = vi[lane][warp];
#pragma unroll
            for (int t = 0; t < 32; ++t)
            {
                const int r = r0 + t;
                if (r < k && (BACKWARD ? r > i : r < i)) p[t] = fma_rn(vr[lane][t], x, p[t]);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < 32; ++t)
    {
        const float dot = lane_fold(p[t]);
        const int r = r0 + t;
        if (lane == 0 && i < k && r < k && (BACKWARD ? r > i : r < i)) G[(int64_t)i * k + r] = dot;
    }
}

// slarft's recurrence, one block: forward, for i ascending, T(r, i) = sum_{q=r}^{i-1} T(r, q)
// d_q (r < i); backward, for i descending, T(r, i) = sum_{q=i+1}^{r} T(r, q) d_q (r > i); d_q =
// -tau_i G(q, i), every sum an FMA chain in ascending q.  The referenced triangle of T is kept
// packed in shared memory and written out at the end.
template <bool BACKWARD>
__global__ void __launch_bounds__(256) xlarft_tri_kernel(const float *G, int k, const float *tau, float *T, int ldt)
{
    extern __shared__ float tp[];  // packed triangle, column by column
    __shared__ float d[256];
    const int tid = threadIdx.x;
    // forward: column i holds rows 0..i at i(i+1)/2; backward: rows i..k-1 at i k - i(i-1)/2
    auto at = [&](int r, int c) -> float & {
        return BACKWARD ? tp[c * k - c * (c - 1) / 2 + (r - c)] : tp[c * (c + 1) / 2 + r];
    };
    for (int s = 0; s < k; ++s)
    {
        const int i = BACKWARD ? k - 1 - s : s;
        const float ti = tau[i];
        for (int q = tid; q < k; q += blockDim.x)
            d[q] = (BACKWARD ? q > i : q < i) ? mul_rn(-ti, G[(int64_t)i * k + q]) : 0.0f;
        __syncthreads();
        for (int r = tid; r < k; r += blockDim.x)
        {
            if (BACKWARD ? r < i : r > i) continue;
            float val;
            if (ti == 0.0f)
                val = 0.0f;
            else if (r == i)
                val = ti;
            else
            {
                float acc = 0.0f;
                if (BACKWARD)
                    for (int q = i + 1; q <= r; ++q) acc = fma_rn(at(r, q), d[q], acc);
                else
                    for (int q = r; q < i; ++q) acc = fma_rn(at(r, q), d[q], acc);
                val = acc;
            }
            at(r, i) = val;
        }
        __syncthreads();
    }
    for (int c = 0; c < k; ++c)
        for (int r = tid; r < k; r += blockDim.x)
            if (BACKWARD ? r >= c : r <= c) T[(int64_t)c * ldt + r] = at(r, c);
}

__global__ void qr_identity_kernel(float *A, int lda, int m, int n)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m * n) return;
    const int r = (int)(idx % m), c = (int)(idx / m);
    A[(int64_t)c * lda + r] = r == c ? 1.0f : 0.0f;
}

cudaError_t apply_block(bool right, bool lower_chain, const float *V, int ldv, int nq, int k, int kb, const float *T,
                        float *C, int64_t ldc, int count, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((count + APPLY_WARPS - 1) / APPLY_WARPS);
    if (right && lower_chain)
        qr_apply_kernel<true, true><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    else if (right)
        qr_apply_kernel<true, false><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    else if (lower_chain)
        qr_apply_kernel<false, true><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    else
        qr_apply_kernel<false, false><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    return cudaGetLastError();
}
// T of the panel's kb reflectors: the Gram products over the grid, then the recurrence.
cudaError_t larft(const float *A, int lda, int nq, int k, int kb, const float *tau, float *T, cudaStream_t stream)
{
    const int pairs = kb * (kb - 1) / 2;
    if (pairs > 0)
    {
        qr_gram_kernel<<<(pairs + GRAM_WARPS - 1) / GRAM_WARPS, GRAM_WARPS * 32, 0, stream>>>(A, lda, nq, k, kb, tau,
                                                                                             T);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    qr_tri_kernel<<<1, 32, 0, stream>>>(k, kb, tau, T);
    return cudaGetLastError();
}
}  // namespace

static std::atomic<unsigned long long> g_qr_attr{0};

cudaError_t launch_sgeqrf(float *A, int lda, int m, int n, float *tau, float *T, cudaStream_t stream)
{
    const int lim = std::min(m, n);
    cudaError_t e = once_per_device(g_qr_attr,
                                    []
                                    {
                                        cudaError_t r = cudaFuncSetAttribute(
                                            qr_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            PANEL_SMEM_FLOATS * (int)sizeof(float));
                                        if (r == cudaSuccess)
                                            r = cudaFuncSetAttribute(qr_cluster_panel_kernel,
                                                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                     PANEL_SMEM_FLOATS * (int)sizeof(float));
                                        return r;
                                    });
    // Look-ahead (panels on a high-priority stream beside the wide update) once the trailing
    // matrix is wide and tall enough to keep the rest of the GPU busy.
    Lookahead la;
    // No look-ahead while the stream is being captured: it would create a stream and events.
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess)
    {
        cudaGetLastError();
        capture = cudaStreamCaptureStatusActive;
    }
    bool ahead = e == cudaSuccess && capture == cudaStreamCaptureStatusNone && m >= 512 && n > 3 * NB;
    if (ahead && la.open(stream) != cudaSuccess)
    {
        la.abandon();  // no private stream to be had: factor on the caller's stream alone
        ahead = false;
    }
    cudaStream_t ps = ahead ? la.panel : stream;
    for (int k = 0; k < lim && e == cudaSuccess; k += NB)
    {
        const int kb = std::min(NB, lim - k);
        const int64_t panel_floats = (int64_t)(m - k) * kb;
        const int seg = panel_seg(m - k, kb, PANEL_SMEM_FLOATS);
        if (panel_floats <= PANEL_SMEM_FLOATS)
        {
            qr_panel_kernel<<<1, PANEL_THREADS, (size_t)panel_floats * sizeof(float), ps>>>(A, lda, m, k, kb, tau);
            e = cudaGetLastError();
        }
        else if (seg > 0)
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)((m - k + seg - 1) / seg));
            cfg.blockDim = dim3(PANEL_THREADS);
            cfg.dynamicSmemBytes = (size_t)seg * kb * sizeof(float);
            cfg.stream = ps;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cfg.gridDim.x;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            e = cudaLaunchKernelEx(&cfg, qr_cluster_panel_kernel, A, lda, m, k, kb, seg, tau);
        }
        else  // taller than eight blocks hold (m > 12,800): not reached, the entries cap m at 8,192
            e = cudaErrorInvalidValue;
        if (e == cudaSuccess && k + kb < n)
        {
            float *Tk = T + (size_t)((k / NB) & 1) * QR_T_FLOATS;  // panel p's T, read by its wide update
            e = larft(A, lda, m, k, kb, tau, Tk, ps);
            const int next = ahead ? std::min(NB, n - k - kb) : n - k - kb;
            // the previous wide update has reached the next panel's columns
            if (e == cudaSuccess && ahead && k > 0) e = la.to_panel(stream);
            if (e == cudaSuccess)
                e = apply_block(false, true, A, lda, m, k, kb, Tk, A + (int64_t)(k + kb) * lda, lda, next, ps);
            const int rest = n - k - kb - next;
            if (e == cudaSuccess && rest > 0)
            {
                e = la.to_main(stream);  // T and the reflectors are ready
                if (e == cudaSuccess)
                    e = apply_block(false, true, A, lda, m, k, kb, Tk, A + (int64_t)(k + kb + next) * lda, lda, rest,
                                    stream);
            }
        }
    }
    if (ahead)
    {
        const cudaError_t c = la.close(stream);
        if (e == cudaSuccess) e = c;
    }
    return e;
}

cudaError_t launch_sormqr(int side, int trans, int m, int n, int k, const float *A, int lda, const float *tau,
                          float *C, int ldc, float *T, cudaStream_t stream)
{
    const bool right = side != 0, tr = trans != 0;
    const int nq = right ? n : m, count = right ? m : n;
    const int npan = (k + NB - 1) / NB;
    const bool forward = !right == tr;  // Q^T from the left and Q from the right take H(1) first
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < npan && e == cudaSuccess; ++s)
    {
        const int pi = forward ? s : npan - 1 - s;
        const int k0 = pi * NB, kb = std::min(NB, k - k0);
        e = larft(A, lda, nq, k0, kb, tau, T, stream);
        // op(T) = T^T (lower chain) for Q^T from the left and for Q from the right
        if (e == cudaSuccess) e = apply_block(right, right ? !tr : tr, A, lda, nq, k0, kb, T, C, ldc, count, stream);
    }
    return e;
}

cudaError_t launch_sorgqr(int m, int n, int k, float *A, int lda, const float *tau, float *work, cudaStream_t stream)
{
    float *v = work, *T = work + (size_t)m * k;
    cudaError_t e = cudaSuccess;
    if (k > 0)
        e = cudaMemcpy2DAsync(v, (size_t)m * sizeof(float), A, (size_t)lda * sizeof(float), (size_t)m * sizeof(float),
                              k, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess)
    {
        const int64_t total = (int64_t)m * n;
        qr_identity_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(A, lda, m, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && k > 0) e = launch_sormqr(0, 0, m, n, k, v, m, tau, A, lda, T, stream);
    return e;
}

size_t sgels_work_floats(int m, int n, int nrhs)
{
    auto up = [](size_t x) { return (x + 63) & ~size_t(63); };
    return up((size_t)std::max(n, 1)) + up((size_t)m * nrhs) + up(QR_GEQRF_T_FLOATS);
}

cudaError_t launch_sgels(int m, int n, int nrhs, float *A, int lda, const float *B, int ldb, float *X, int ldx,
                         float *work, cudaStream_t stream)
{
    auto up = [](size_t x) { return (x + 63) & ~size_t(63); };
    float *tau = work, *Y = tau + up((size_t)std::max(n, 1)), *T = Y + up((size_t)m * nrhs);
    cudaError_t e = cudaMemcpy2DAsync(Y, (size_t)m * sizeof(float), B, (size_t)ldb * sizeof(float),
                                      (size_t)m * sizeof(float), nrhs, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess) e = launch_sgeqrf(A, lda, m, n, tau, T, stream);
    if (e == cudaSuccess) e = launch_sormqr(0, 1, m, nrhs, n, A, lda, tau, Y, m, T, stream);
    if (e == cudaSuccess)
    {
        qr_trsv_kernel<<<nrhs, 1024, (size_t)n * sizeof(float), stream>>>(A, lda, n, Y, m, X, ldx);
        e = cudaGetLastError();
    }
    return e;
}
}  // namespace ops_solver

namespace ops_solver
{
size_t xlarft_work_bytes(int k) { return (size_t)k * k * sizeof(float); }

cudaError_t launch_xlarft(int backward, int n, int k, const float *V, int ldv, const float *tau, float *T, int ldt,
                          float *G, cudaStream_t stream)
{
    if (n <= 0 || k <= 0) return cudaSuccess;
    if (k > 256) return cudaErrorInvalidValue;
    const int kb = (k + 31) / 32;
    dim3 grid(kb, kb);
    const size_t tri = (size_t)k * (k + 1) / 2 * sizeof(float);
    cudaError_t e;
    if (backward)
    {
        e = cudaFuncSetAttribute(xlarft_tri_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri);
        if (e != cudaSuccess) return e;
        xlarft_gram_kernel<true><<<grid, 1024, 0, stream>>>(V, ldv, n, k, G);
        xlarft_tri_kernel<true><<<1, 256, tri, stream>>>(G, k, tau, T, ldt);
    }
    else
    {
        e = cudaFuncSetAttribute(xlarft_tri_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri);
        if (e != cudaSuccess) return e;
        xlarft_gram_kernel<false><<<grid, 1024, 0, stream>>>(V, ldv, n, k, G);
        xlarft_tri_kernel<false><<<1, 256, tri, stream>>>(G, k, tau, T, ldt);
    }
    return cudaGetLastError();
}
}  // namespace ops_solver
