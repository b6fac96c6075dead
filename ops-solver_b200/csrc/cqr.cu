// cqr.cu -- the complex QR family: Cgeqrf, Cunmqr, Cungqr and CCgels (complex64).
//
// Reflectors follow LAPACK clarfg, as the reference's kernel does
// (src/cgeqrf/arch35/cgeqrf_reflector_simd.h:89-170): beta = -copysign(||(alpha; x)||, Re alpha),
// tau = ((beta - Re alpha) / beta, -(Im alpha / beta)), v = x / (alpha - beta), tau = 0 when
// x is zero and alpha real; Q = H(1)...H(k), H = I - tau v v^H.  The schedule is the real
// family's (qr.cu): 32-column panels, lane sums over rows (row r into lane r mod 32, a warp
// butterfly per component), slarft's T, block application.  The complex products are fixed
// FMA sequences (cq_* below) that the CPU oracle restates.
#include <cooperative_groups.h>
#include <limits.h>

#include <algorithm>
#include <atomic>

#include "complex_lu.cuh"
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
constexpr int PANEL_SMEM_ELEMS = 25 * 1024;  // complex elements of a panel kept in shared memory

// acc += conj(v) a
__device__ __forceinline__ float2 cq_conjdot(float2 acc, float2 v, float2 a)
{
    return make_float2(fma_rn(v.y, a.y, fma_rn(v.x, a.x, acc.x)), fma_rn(-v.y, a.x, fma_rn(v.x, a.y, acc.y)));
}
// acc += c v
__device__ __forceinline__ float2 cq_dot(float2 acc, float2 c, float2 v)
{
    return make_float2(fma_rn(-c.y, v.y, fma_rn(c.x, v.x, acc.x)), fma_rn(c.y, v.x, fma_rn(c.x, v.y, acc.y)));
}
// x - y conj(v)
__device__ __forceinline__ float2 cq_submulc(float2 x, float2 y, float2 v)
{
    return make_float2(fma_rn(-y.y, v.y, fma_rn(-y.x, v.x, x.x)), fma_rn(y.x, v.y, fma_rn(-y.y, v.x, x.y)));
}
__device__ __forceinline__ float2 cq_mul(float2 a, float2 b)
{
    return make_float2(fma_rn(-a.y, b.y, mul_rn(a.x, b.x)), fma_rn(a.y, b.x, mul_rn(a.x, b.y)));
}
__device__ __forceinline__ float2 cq_mulc(float2 a, float2 b)
{
    return make_float2(fma_rn(a.y, b.y, mul_rn(a.x, b.x)), fma_rn(-a.y, b.x, mul_rn(a.x, b.y)));
}
// acc + a b
__device__ __forceinline__ float2 cq_fma(float2 a, float2 b, float2 acc)
{
    return make_float2(fma_rn(-a.y, b.y, fma_rn(a.x, b.x, acc.x)), fma_rn(a.y, b.x, fma_rn(a.x, b.y, acc.y)));
}
// acc + conj(a) b
__device__ __forceinline__ float2 cq_fmac(float2 a, float2 b, float2 acc)
{
    return make_float2(fma_rn(a.y, b.y, fma_rn(a.x, b.x, acc.x)), fma_rn(-a.y, b.x, fma_rn(a.x, b.y, acc.y)));
}

__device__ __forceinline__ float fold1(float p)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) p = add_rn(p, __shfl_xor_sync(0xffffffffu, p, off));
    return p;
}
__device__ __forceinline__ float2 fold2(float2 p) { return make_float2(fold1(p.x), fold1(p.y)); }

__device__ __forceinline__ bool czero2(float2 v) { return v.x == 0.0f && v.y == 0.0f; }

// Panel columns [k, k + kb) of rows [k, m), in shared memory (SMEM) or, for panels taller
// than eight blocks hold, in A.  Per column c, every reduction over the rows below c is taken
// at once from the column as it stands: warp 0 forms sumsq = sum |x_i|^2 and warp w >= 1
// forms S_j = sum conj(x_i) A(i, j) for column j = c + w, in parallel.  After one barrier
// every thread forms beta, tau, d = alpha - beta, den = |d|^2 and g = d / den (cq_scalars);
// warp w applies w_j = conj(tau) (A(c, j) + g S_j) with v_i = x_i / d formed on the fly;
// column c itself is divided, and beta stored, during the next column's reductions.
__device__ __forceinline__ float2 cq_reflect(float2 x, float dr, float di, float den)
{
    return make_float2(div_rn(add_rn(mul_rn(x.x, dr), mul_rn(x.y, di)), den),
                       div_rn(sub_rn(mul_rn(x.y, dr), mul_rn(x.x, di)), den));
}

// Scalars of column c's reflector from sumsq and alpha (every thread forms them identically).
struct CqScalars
{
    bool apply;
    float beta, dr, di, den;
    float2 t, g;
};

__device__ __forceinline__ CqScalars cq_scalars(float sumsq, float2 al)
{
    CqScalars r{};
    r.apply = !(sumsq == 0.0f && al.y == 0.0f);
    r.t = make_float2(0.0f, 0.0f);
    if (r.apply)
    {
        const float norm = sqrt_rn(add_rn(add_rn(mul_rn(al.x, al.x), mul_rn(al.y, al.y)), sumsq));
        r.beta = -copysignf(norm, al.x);
        r.t = make_float2(div_rn(sub_rn(r.beta, al.x), r.beta), -div_rn(al.y, r.beta));
        r.dr = sub_rn(al.x, r.beta);
        r.di = al.y;
        r.den = add_rn(mul_rn(r.dr, r.dr), mul_rn(r.di, r.di));
        r.g = make_float2(div_rn(r.dr, r.den), div_rn(r.di, r.den));
    }
    return r;
}

template <bool SMEM>
__global__ void __launch_bounds__(PANEL_THREADS) cq_panel_kernel(float2 *A, int lda, int m, int k, int kb, float2 *tau)
{
    extern __shared__ float2 sp[];
    __shared__ float2 s_S[NB], s_alpha;
    __shared__ float s_sumsq;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int H = m - k;
    auto at = [&](int j, int row) -> float2 & {
        return SMEM ? sp[(int64_t)(j - k) * H + (row - k)] : A[(int64_t)j * lda + row];
    };
    if (SMEM)
    {
        for (int idx = tid; idx < H * kb; idx += PANEL_THREADS) sp[idx] = A[(int64_t)(k + idx / H) * lda + k + idx % H];
        __syncthreads();
    }
    CqScalars prev{};
    prev.apply = false;
    for (int c = k; c < k + kb; ++c)
    {
        if (prev.apply)  // column c - 1 becomes its reflector, beta its diagonal entry
        {
            if (tid == 0) at(c - 1, c - 1) = make_float2(prev.beta, 0.0f);
            for (int row = c + tid; row < m; row += PANEL_THREADS)
                at(c - 1, row) = cq_reflect(at(c - 1, row), prev.dr, prev.di, prev.den);
        }
        const int j = c + warp;
        if (warp == 0)
        {
            float p = 0.0f;
#pragma unroll 4
            for (int row = c + 1 + lane; row < m; row += 32)
            {
                const float2 x = at(c, row);
                p = fma_rn(x.y, x.y, fma_rn(x.x, x.x, p));
            }
            const float part = fold1(p);
            if (lane == 0)
            {
                s_sumsq = part;
                s_alpha = at(c, c);
            }
        }
        else if (j < k + kb)
        {
            float2 p = make_float2(0.0f, 0.0f);
#pragma unroll 4
            for (int row = c + 1 + lane; row < m; row += 32) p = cq_conjdot(p, at(c, row), at(j, row));
            const float2 part = fold2(p);
            if (lane == 0) s_S[warp] = part;
        }
        __syncthreads();
        const CqScalars r = cq_scalars(s_sumsq, s_alpha);
        if (tid == 0) tau[c] = r.t;
        if (r.apply && warp >= 1 && j < k + kb)
        {
            const float2 w = cq_mulc(r.t, cq_fma(r.g, s_S[warp], at(j, c)));
            __syncwarp();
            if (lane == 0) at(j, c) = clu::csubmul(at(j, c), make_float2(1.0f, 0.0f), w);
#pragma unroll 4
            for (int row = c + 1 + lane; row < m; row += 32)
                at(j, row) = clu::csubmul(at(j, row), cq_reflect(at(c, row), r.dr, r.di, r.den), w);
        }
        prev = r;
        __syncthreads();
    }
    if (prev.apply)
    {
        if (tid == 0) at(k + kb - 1, k + kb - 1) = make_float2(prev.beta, 0.0f);
        for (int row = k + kb + tid; row < m; row += PANEL_THREADS)
            at(k + kb - 1, row) = cq_reflect(at(k + kb - 1, row), prev.dr, prev.di, prev.den);
    }
    if (SMEM)
    {
        __syncthreads();
        for (int idx = tid; idx < H * kb; idx += PANEL_THREADS) A[(int64_t)(k + idx / H) * lda + k + idx % H] = sp[idx];
    }
}

// Rows per block of a panel spread over a cluster (0: the panel fits one block, or is too
// tall for eight), as in the real family; the CPU oracle reduces with the same segments.
__host__ __device__ inline int panel_seg(int H, int kb, int budget)
{
    if ((int64_t)H * kb <= budget) return 0;
    const int seg = ((H + 7) / 8 + 31) & ~31;
    return (int64_t)seg * kb <= budget ? seg : 0;
}

// A tall panel over a cluster of ceil((m - k) / seg) blocks, block g holding rows
// [k + g seg, k + (g + 1) seg) in shared memory and running the one-block schedule on them;
// the per-block lane sums (and block 0's row of diagonal entries) are published in shared
// memory double-buffered by column parity and, after one cluster barrier per column, added
// in ascending block order by every block through distributed shared memory.
__global__ void __launch_bounds__(PANEL_THREADS) cq_cluster_panel_kernel(float2 *A, int lda, int m, int k, int kb,
                                                                         int seg, float2 *tau)
{
    namespace cg = cooperative_groups;
    extern __shared__ float2 sp[];  // sp[(j - k) * seg + (row - r0)]
    __shared__ float pub_sumsq[2];
    __shared__ float2 pub_S[2][NB], pub_row[2][NB];
    cg::cluster_group cluster = cg::this_cluster();
    const int g = (int)cluster.block_rank(), G = (int)cluster.num_blocks();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = k + g * seg, r1 = min(m, r0 + seg);
    const int rows = max(0, r1 - r0);
    auto at = [&](int j, int row) -> float2 & { return sp[(j - k) * seg + (row - r0)]; };
    // the blocks' totals in ascending block order: lane q fetches block q's, every lane adds
    auto total1 = [&](float *mine) -> float
    {
        const float part = lane < G ? *cluster.map_shared_rank(mine, lane) : 0.0f;
        float sum = __shfl_sync(0xffffffffu, part, 0);
        for (int q = 1; q < G; ++q) sum = add_rn(sum, __shfl_sync(0xffffffffu, part, q));
        return sum;
    };
    auto total2 = [&](float2 *mine) -> float2
    {
        const float2 part = lane < G ? *cluster.map_shared_rank(mine, lane) : make_float2(0.0f, 0.0f);
        float2 sum = make_float2(__shfl_sync(0xffffffffu, part.x, 0), __shfl_sync(0xffffffffu, part.y, 0));
        for (int q = 1; q < G; ++q)
            sum = make_float2(add_rn(sum.x, __shfl_sync(0xffffffffu, part.x, q)),
                              add_rn(sum.y, __shfl_sync(0xffffffffu, part.y, q)));
        return sum;
    };
    for (int idx = tid; idx < rows * kb; idx += PANEL_THREADS)
        sp[(idx / rows) * seg + idx % rows] = A[(int64_t)(k + idx / rows) * lda + r0 + idx % rows];
    __syncthreads();
    CqScalars prev{};
    prev.apply = false;
    for (int c = k; c < k + kb; ++c)
    {
        const int par = c & 1, owner = (c - k) / seg;
        if (prev.apply)  // column c - 1 becomes its reflector, beta its diagonal entry
        {
            if (tid == 0 && c - 1 >= r0 && c - 1 < r1) at(c - 1, c - 1) = make_float2(prev.beta, 0.0f);
            for (int row = max(r0, c) + tid; row < r1; row += PANEL_THREADS)
                at(c - 1, row) = cq_reflect(at(c - 1, row), prev.dr, prev.di, prev.den);
        }
        const int j = c + warp;
        if (warp == 0)
        {
            float p = 0.0f;
#pragma unroll 4
            for (int row = max(r0, c + 1) + lane; row < r1; row += 32)
            {
                const float2 x = at(c, row);
                p = fma_rn(x.y, x.y, fma_rn(x.x, x.x, p));
            }
            const float part = fold1(p);
            if (lane == 0) pub_sumsq[par] = part;
        }
        else if (j < k + kb)
        {
            float2 p = make_float2(0.0f, 0.0f);
#pragma unroll 4
            for (int row = max(r0, c + 1) + lane; row < r1; row += 32) p = cq_conjdot(p, at(c, row), at(j, row));
            const float2 part = fold2(p);
            if (lane == 0) pub_S[par][warp] = part;
        }
        if (j < k + kb && lane == 0 && g == owner) pub_row[par][warp] = at(j, c);
        cluster.sync();
        const CqScalars r = cq_scalars(total1(&pub_sumsq[par]), *cluster.map_shared_rank(&pub_row[par][0], owner));
        if (tid == 0 && g == 0) tau[c] = r.t;
        if (r.apply && warp >= 1 && j < k + kb)
        {
            const float2 S = total2(&pub_S[par][warp]);
            const float2 acj = *cluster.map_shared_rank(&pub_row[par][warp], owner);
            const float2 w = cq_mulc(r.t, cq_fma(r.g, S, acj));
            if (lane == 0 && g == owner) at(j, c) = clu::csubmul(acj, make_float2(1.0f, 0.0f), w);
#pragma unroll 4
            for (int row = max(r0, c + 1) + lane; row < r1; row += 32)
                at(j, row) = clu::csubmul(at(j, row), cq_reflect(at(c, row), r.dr, r.di, r.den), w);
        }
        prev = r;
        __syncthreads();
    }
    if (prev.apply)
    {
        if (tid == 0 && k + kb - 1 >= r0 && k + kb - 1 < r1) at(k + kb - 1, k + kb - 1) = make_float2(prev.beta, 0.0f);
        for (int row = max(r0, k + kb) + tid; row < r1; row += PANEL_THREADS)
            at(k + kb - 1, row) = cq_reflect(at(k + kb - 1, row), prev.dr, prev.di, prev.den);
    }
    cluster.sync();  // no block leaves while another may still read what it published
    for (int idx = tid; idx < rows * kb; idx += PANEL_THREADS)
        A[(int64_t)(k + idx / rows) * lda + r0 + idx % rows] = sp[(idx / rows) * seg + idx % rows];
}

// The reflector products of a panel for T: d(i, r) = -tau_i (v_r^H v_i) for r < i, one warp
// per pair, each a lane sum in ascending rows, stored below T's diagonal (T[r * NB + i]);
// cq_tri_kernel then forms T's upper triangle from them.
constexpr int GRAM_WARPS = 8;

__global__ void __launch_bounds__(GRAM_WARPS * 32) cq_gram_kernel(const float2 *A, int lda, int nq, int k, int kb,
                                                                  const float2 *tau, float2 *T)
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
    const float2 *vr = A + (int64_t)(k + r) * lda, *vi = A + (int64_t)(k + i) * lda;
    const int first = k + i;
    constexpr int U = 8;
    float2 p = make_float2(0.0f, 0.0f);
    for (int base = first & ~31; base < nq; base += 32 * U)
    {
        float2 a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int row = base + 32 * u + lane;
            const bool ok = row >= first && row < nq;
            a[u] = ok ? vr[row] : make_float2(0.0f, 0.0f);
            b[u] = ok ? (row == first ? make_float2(1.0f, 0.0f) : vi[row]) : make_float2(0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const int row = base + 32 * u + lane;
            if (row >= first && row < nq) p = cq_conjdot(p, a[u], b[u]);
        }
    }
    const float2 dot = fold2(p);
    if (lane == 0)
    {
        const float2 ti = tau[k + i];
        T[r * NB + i] = cq_mul(make_float2(-ti.x, -ti.y), dot);
    }
}

// T (kb x kb upper, ld NB): T(i, i) = tau_i, T(0:i, i) = T(0:i, 0:i) d(i, 0:i) (a chain in
// ascending q), a zero column where tau_i = 0.  Lane r keeps row r of T in registers.
__global__ void __launch_bounds__(32) cq_tri_kernel(int k, int kb, const float2 *tau, float2 *T)
{
    __shared__ float2 d[NB][NB];  // d[i][q] = d(i, q)
    const int r = threadIdx.x;
    for (int i = 0; i < kb; ++i)
        if (r < i) d[i][r] = T[r * NB + i];
    __syncwarp();
    float2 tr[NB];  // tr[q] = T(r, q)
#pragma unroll
    for (int i = 0; i < NB; ++i)
    {
        tr[i] = make_float2(0.0f, 0.0f);
        if (i < kb)
        {
            const float2 ti = tau[k + i];
            if (!czero2(ti))
            {
                if (r == i)
                    tr[i] = ti;
                else if (r < i)
                {
                    float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                    for (int q = 0; q < i; ++q)
                        if (q >= r) acc = cq_fma(tr[q], d[i][q], acc);
                    tr[i] = acc;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i)
        if (i < kb && r <= i) T[i * NB + r] = tr[i];
}

// LEFT: C = (I - V op(T) V^H) C, one warp per column of C; RIGHT: C = C (I - V op(T) V^H), one
// warp per row.  HERM selects op(T) = T^H (LEFT: Q^H C; RIGHT: C Q^H), else T.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <bool RIGHT, bool HERM>
__global__ void __launch_bounds__(APPLY_WARPS * 32) cq_apply_kernel(const float2 *V, int ldv, int nq, int k, int kb,
                                                                    const float2 *T, float2 *C, int64_t ldc, int count)
{
    constexpr int ROWS = 64;
    constexpr int CU = ROWS / 32;
    // V double-buffered (the next pass copied by cp.async while this one computes), raw: the
    // unit diagonal and the zeros above it are applied when the first 32 rows are read.
    __shared__ __align__(16) float2 vs[2][ROWS][NB + 2];  // even pitch: 128-bit reads of two entries
    __shared__ float2 ts[NB * NB];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j = blockIdx.x * APPLY_WARPS + warp;
    const bool live = j < count;
    for (int idx = tid; idx < NB * NB; idx += APPLY_WARPS * 32) ts[idx] = T[idx];
    auto cat = [&](int row) -> float2 * { return RIGHT ? C + (int64_t)row * ldc + j : C + (int64_t)j * ldc + row; };
    auto stage = [&](int base0, int b)
    {
        if (base0 < nq)
            for (int idx = tid; idx < ROWS * kb; idx += APPLY_WARPS * 32)
            {
                const int rr = idx % ROWS, i = idx / ROWS, row = base0 + rr;
                if (row < nq) cp_async8(&vs[b][rr][i], V + (int64_t)(k + i) * ldv + row);
            }
        cp_async_commit();
    };
    auto load_c = [&](int base0, float2 *c)
    {
#pragma unroll
        for (int u = 0; u < CU; ++u)
        {
            const int row = base0 + 32 * u + lane;
            c[u] = live && row >= k && row < nq ? *cat(row) : make_float2(0.0f, 0.0f);
        }
    };
    const float2 one = make_float2(1.0f, 0.0f);
    float2 p[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) p[i] = make_float2(0.0f, 0.0f);
    const int first = k & ~31;
    float2 c[CU];
    stage(first, 0);
    load_c(first, c);
    int b = 0;
    for (int base0 = first; base0 < nq; base0 += ROWS, b ^= 1)
    {
        stage(base0 + ROWS, b ^ 1);
        float2 cn[CU];
        load_c(base0 + ROWS, cn);
        cp_async_wait_prior();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u)
        {
            const int row = base0 + 32 * u + lane;
            if (live && kb == NB && row >= k + NB && row < nq)  // below every reflector's unit entry
            {
#pragma unroll
                for (int i = 0; i < NB; i += 2)
                {
                    const float4 v2 = *reinterpret_cast<const float4 *>(&vs[b][32 * u + lane][i]);
                    const float2 va = make_float2(v2.x, v2.y), vb = make_float2(v2.z, v2.w);
                    p[i] = RIGHT ? cq_dot(p[i], c[u], va) : cq_conjdot(p[i], va, c[u]);
                    p[i + 1] = RIGHT ? cq_dot(p[i + 1], c[u], vb) : cq_conjdot(p[i + 1], vb, c[u]);
                }
            }
            else if (live && row >= k && row < nq)
            {
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    if (i < kb && row >= k + i)
                    {
                        const float2 v = row == k + i ? one : vs[b][32 * u + lane][i];
                        p[i] = RIGHT ? cq_dot(p[i], c[u], v) : cq_conjdot(p[i], v, c[u]);
                    }
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u) c[u] = cn[u];
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) p[i] = fold2(p[i]);
    float2 w2[NB];  // W2 = op(T) W, lane i forming entry i, then shared across the warp
    {
        // lower chain (sum over q <= i of T(q, i)): LEFT with T^H, RIGHT with T
        constexpr bool LOWER = RIGHT ? !HERM : HERM;
        float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < NB; ++q)
        {
            if (LOWER)
            {
                if (q <= lane && lane < kb)
                    acc = HERM ? cq_fmac(ts[lane * NB + q], p[q], acc) : cq_fma(ts[lane * NB + q], p[q], acc);
            }
            else
            {
                if (q >= lane && q < kb)
                    acc = HERM ? cq_fmac(ts[q * NB + lane], p[q], acc) : cq_fma(ts[q * NB + lane], p[q], acc);
            }
        }
#pragma unroll
        for (int i = 0; i < NB; ++i)
            w2[i] = make_float2(__shfl_sync(0xffffffffu, acc.x, i), __shfl_sync(0xffffffffu, acc.y, i));
    }
    stage(first, 0);
    load_c(first, c);
    b = 0;
    for (int base0 = first; base0 < nq; base0 += ROWS, b ^= 1)
    {
        stage(base0 + ROWS, b ^ 1);
        float2 cn[CU];
        load_c(base0 + ROWS, cn);
        cp_async_wait_prior();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u)
        {
            const int row = base0 + 32 * u + lane;
            if (live && kb == NB && row >= k + NB && row < nq)
            {
                float2 x = c[u];
#pragma unroll
                for (int i = 0; i < NB; i += 2)
                {
                    const float4 v2 = *reinterpret_cast<const float4 *>(&vs[b][32 * u + lane][i]);
                    const float2 va = make_float2(v2.x, v2.y), vb = make_float2(v2.z, v2.w);
                    x = RIGHT ? cq_submulc(x, w2[i], va) : clu::csubmul(x, va, w2[i]);
                    x = RIGHT ? cq_submulc(x, w2[i + 1], vb) : clu::csubmul(x, vb, w2[i + 1]);
                }
                *cat(row) = x;
            }
            else if (live && row >= k && row < nq)
            {
                float2 x = c[u];
#pragma unroll
                for (int i = 0; i < NB; ++i)
                    if (i < kb && i <= row - k)
                    {
                        const float2 v = row == k + i ? one : vs[b][32 * u + lane][i];
                        x = RIGHT ? cq_submulc(x, w2[i], v) : clu::csubmul(x, v, w2[i]);
                    }
                *cat(row) = x;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < CU; ++u) c[u] = cn[u];
    }
}

// R X = Y for one right-hand side per block; R's diagonal is real.  Every block first looks
// for a zero diagonal entry: the first one (one-based) goes to info and X is left untouched.
// Then 32-column blocks from the bottom: warp 0 solves the diagonal block with the
// right-hand side in its lanes (x_p = x_p / R_pp componentwise, then x_i -= R_ip x_p, p
// descending), and every thread applies the block's columns to the rows above it, p
// descending, so each x_i receives its updates in descending p.
__global__ void __launch_bounds__(512) cq_trsv_kernel(const float2 *R, int ldr, int n, const float2 *Y, int ldy,
                                                       float2 *X, int ldx, int *info)
{
    extern __shared__ float2 xs[];
    __shared__ int s_zero;
    const int j = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) s_zero = n;
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x)
        if (czero2(R[(int64_t)i * ldr + i])) atomicMin(&s_zero, i);
    __syncthreads();
    const int zero = s_zero;
    if (zero < n)
    {
        if (j == 0 && tid == 0) *info = zero + 1;
        return;
    }
    for (int i = tid; i < n; i += blockDim.x) xs[i] = Y[(int64_t)j * ldy + i];
    __syncthreads();
    for (int c0 = (n - 1) & ~31; c0 >= 0; c0 -= 32)
    {
        const int cw = min(32, n - c0);
        if (tid < 32)
        {
            float2 r[32];
#pragma unroll
            for (int q = 0; q < 32; ++q)
                r[q] = lane < cw && q < cw ? R[(int64_t)(c0 + q) * ldr + c0 + lane] : make_float2(1.0f, 0.0f);
            float2 x = lane < cw ? xs[c0 + lane] : make_float2(0.0f, 0.0f);
#pragma unroll
            for (int q = 31; q >= 0; --q)
            {
                if (q < cw && lane == q) x = make_float2(div_rn(x.x, r[q].x), div_rn(x.y, r[q].x));
                const float2 xp = make_float2(__shfl_sync(0xffffffffu, x.x, q), __shfl_sync(0xffffffffu, x.y, q));
                if (q < cw && lane < q) x = clu::csubmul(x, r[q], xp);
            }
            if (lane < cw) xs[c0 + lane] = x;
        }
        __syncthreads();
        for (int i = tid; i < c0; i += blockDim.x)
        {
            float2 x = xs[i];
            for (int q = cw - 1; q >= 0; --q) x = clu::csubmul(x, R[(int64_t)(c0 + q) * ldr + i], xs[c0 + q]);
            xs[i] = x;
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += blockDim.x) X[(int64_t)j * ldx + i] = xs[i];
}

// Input screening: the smallest code among the regions holding a NaN or an infinity goes to
// *flag (atomicMin over an initial INT_MAX).  A region with strict set is a reflector store:
// only the entries below its diagonal are inputs.
struct FiniteRegion
{
    const float2 *p;
    int rows, cols;
    int64_t ld;
    int strict, code;
};

__global__ void cq_finite_kernel(FiniteRegion r0, FiniteRegion r1, FiniteRegion r2, int *flag)
{
    const FiniteRegion rs[3] = {r0, r1, r2};
    int found = INT_MAX;
#pragma unroll
    for (int q = 0; q < 3; ++q)
    {
        const FiniteRegion r = rs[q];
        if (!r.p || r.rows <= 0 || r.cols <= 0) continue;
        const int64_t total = (int64_t)r.rows * r.cols;
        for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
             idx += (int64_t)gridDim.x * blockDim.x)
        {
            const int row = (int)(idx % r.rows), col = (int)(idx / r.rows);
            if (r.strict && row <= col) continue;
            const float2 v = r.p[(int64_t)col * r.ld + row];
            if (!isfinite(v.x) || !isfinite(v.y)) found = min(found, r.code);
        }
    }
    // the warp's smallest code, one atomic per warp
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) found = min(found, __shfl_xor_sync(0xffffffffu, found, off));
    if ((threadIdx.x & 31) == 0 && found != INT_MAX) atomicMin(flag, found);
}

__global__ void cq_identity_kernel(float2 *A, int lda, int m, int n)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m * n) return;
    const int r = (int)(idx % m), c = (int)(idx / m);
    A[(int64_t)c * lda + r] = make_float2(r == c ? 1.0f : 0.0f, 0.0f);
}

cudaError_t cq_larft(const float2 *A, int lda, int nq, int k, int kb, const float2 *tau, float2 *T,
                     cudaStream_t stream)
{
    const int pairs = kb * (kb - 1) / 2;
    if (pairs > 0)
    {
        cq_gram_kernel<<<(pairs + GRAM_WARPS - 1) / GRAM_WARPS, GRAM_WARPS * 32, 0, stream>>>(A, lda, nq, k, kb, tau,
                                                                                             T);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    cq_tri_kernel<<<1, 32, 0, stream>>>(k, kb, tau, T);
    return cudaGetLastError();
}

cudaError_t cq_apply(bool right, bool herm, const float2 *V, int ldv, int nq, int k, int kb, const float2 *T,
                     float2 *C, int64_t ldc, int count, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((count + APPLY_WARPS - 1) / APPLY_WARPS);
    if (right && herm)
        cq_apply_kernel<true, true><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    else if (right)
        cq_apply_kernel<true, false><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    else if (herm)
        cq_apply_kernel<false, true><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    else
        cq_apply_kernel<false, false><<<grid, APPLY_WARPS * 32, 0, stream>>>(V, ldv, nq, k, kb, T, C, ldc, count);
    return cudaGetLastError();
}

std::atomic<unsigned long long> g_cq_attr{0};
}  // namespace

cudaError_t launch_cgeqrf(float2 *A, int lda, int m, int n, float2 *tau, float2 *T, cudaStream_t stream)
{
    cudaError_t e = once_per_device(g_cq_attr,
                                    []
                                    {
                                        cudaError_t r = cudaFuncSetAttribute(
                                            cq_panel_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            PANEL_SMEM_ELEMS * (int)sizeof(float2));
                                        if (r == cudaSuccess)
                                            r = cudaFuncSetAttribute(cq_cluster_panel_kernel,
                                                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                                     PANEL_SMEM_ELEMS * (int)sizeof(float2));
                                        return r;
                                    });
    const int lim = std::min(m, n);
    // Look-ahead (panels on a high-priority stream beside the wide update), as the real family.
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
        const int64_t elems = (int64_t)(m - k) * kb;
        const int seg = panel_seg(m - k, kb, PANEL_SMEM_ELEMS);
        if (elems <= PANEL_SMEM_ELEMS)
            cq_panel_kernel<true><<<1, PANEL_THREADS, (size_t)elems * sizeof(float2), ps>>>(A, lda, m, k, kb, tau);
        else if (seg > 0)
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)((m - k + seg - 1) / seg));
            cfg.blockDim = dim3(PANEL_THREADS);
            cfg.dynamicSmemBytes = (size_t)seg * kb * sizeof(float2);
            cfg.stream = ps;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cfg.gridDim.x;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            e = cudaLaunchKernelEx(&cfg, cq_cluster_panel_kernel, A, lda, m, k, kb, seg, tau);
        }
        else
            cq_panel_kernel<false><<<1, PANEL_THREADS, 0, ps>>>(A, lda, m, k, kb, tau);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess && k + kb < n)
        {
            float2 *Tk = T + (size_t)((k / NB) & 1) * QR_T_FLOATS;  // panel p's T, read by its wide update
            e = cq_larft(A, lda, m, k, kb, tau, Tk, ps);
            const int next = ahead ? std::min(NB, n - k - kb) : n - k - kb;
            // the previous wide update has reached the next panel's columns
            if (e == cudaSuccess && ahead && k > 0) e = la.to_panel(stream);
            if (e == cudaSuccess)
                e = cq_apply(false, true, A, lda, m, k, kb, Tk, A + (int64_t)(k + kb) * lda, lda, next, ps);
            const int rest = n - k - kb - next;
            if (e == cudaSuccess && rest > 0)
            {
                e = la.to_main(stream);  // T and the reflectors are ready
                if (e == cudaSuccess)
                    e = cq_apply(false, true, A, lda, m, k, kb, Tk, A + (int64_t)(k + kb + next) * lda, lda, rest,
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

cudaError_t launch_cunmqr(int side, int herm, int m, int n, int k, const float2 *A, int lda, const float2 *tau,
                          float2 *C, int ldc, float2 *T, cudaStream_t stream)
{
    const bool right = side != 0, h = herm != 0;
    const int nq = right ? n : m, count = right ? m : n;
    const int npan = (k + NB - 1) / NB;
    const bool forward = !right == h;
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < npan && e == cudaSuccess; ++s)
    {
        const int pi = forward ? s : npan - 1 - s;
        const int k0 = pi * NB, kb = std::min(NB, k - k0);
        e = cq_larft(A, lda, nq, k0, kb, tau, T, stream);
        if (e == cudaSuccess) e = cq_apply(right, h, A, lda, nq, k0, kb, T, C, ldc, count, stream);
    }
    return e;
}

cudaError_t launch_cungqr(int m, int n, int k, float2 *A, int lda, const float2 *tau, float2 *work, cudaStream_t stream)
{
    float2 *v = work, *T = work + (size_t)m * k;
    cudaError_t e = cudaSuccess;
    if (k > 0)
        e = cudaMemcpy2DAsync(v, (size_t)m * sizeof(float2), A, (size_t)lda * sizeof(float2),
                              (size_t)m * sizeof(float2), k, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess)
    {
        const int64_t total = (int64_t)m * n;
        cq_identity_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(A, lda, m, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && k > 0) e = launch_cunmqr(0, 0, m, n, k, v, m, tau, A, lda, T, stream);
    return e;
}

size_t cgels_work_elems(int m, int n, int nrhs)
{
    auto up = [](size_t x) { return (x + 31) & ~size_t(31); };
    return up((size_t)std::max(n, 1)) + up((size_t)m * nrhs) + up(QR_GEQRF_T_FLOATS);
}

cudaError_t launch_cgels(int m, int n, int nrhs, float2 *A, int lda, const float2 *B, int ldb, float2 *X, int ldx,
                         float2 *work, int *info, cudaStream_t stream)
{
    auto up = [](size_t x) { return (x + 31) & ~size_t(31); };
    float2 *tau = work, *Y = tau + up((size_t)std::max(n, 1)), *T = Y + up((size_t)m * nrhs);
    cudaError_t e = cudaMemcpy2DAsync(Y, (size_t)m * sizeof(float2), B, (size_t)ldb * sizeof(float2),
                                      (size_t)m * sizeof(float2), nrhs, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess) e = launch_cgeqrf(A, lda, m, n, tau, T, stream);
    if (e == cudaSuccess) e = launch_cunmqr(0, 1, m, nrhs, n, A, lda, tau, Y, m, T, stream);
    if (e == cudaSuccess)
    {
        cq_trsv_kernel<<<nrhs, 512, (size_t)n * sizeof(float2), stream>>>(A, lda, n, Y, m, X, ldx, info);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_cq_finite(const CqRegion *regions, int count, int *flag, cudaStream_t stream)
{
    FiniteRegion r[3] = {};
    int64_t most = 0;
    for (int q = 0; q < count && q < 3; ++q)
    {
        r[q] = {static_cast<const float2 *>(regions[q].p), regions[q].rows, regions[q].cols, regions[q].ld,
                regions[q].strict, regions[q].code};
        most = std::max<int64_t>(most, (int64_t)regions[q].rows * regions[q].cols);
    }
    const int64_t blocks = std::min<int64_t>(std::max<int64_t>((most + 255) / 256, 1), 148 * 8);
    cq_finite_kernel<<<(unsigned)blocks, 256, 0, stream>>>(r[0], r[1], r[2], flag);
    return cudaGetLastError();
}
}  // namespace ops_solver
