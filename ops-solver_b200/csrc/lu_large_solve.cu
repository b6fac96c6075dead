// lu_large_solve.cu -- P A = L U solves of one large matrix over the whole GPU (the solve
// half of the reference's single-matrix path: src/sgetrs/sgetrs_kernel.cpp:76-80 laswp,
// custom_trsm, custom_trsm_upper).
//
// X (n x nrhs, column-major) first takes the pivots (the LAPACK swap sequence composed into
// one gather), then one launch per 128-row block and sweep: every block of the launch solves
// the diagonal 128 x 128 triangle for all right-hand sides in shared memory (redundantly, it
// is small) and then subtracts the block's contribution from one 128-row strip of the rows
// still to come.  Every element of X receives its updates as fma(-l, x, acc) in ascending k
// (forward) or descending k (backward, after the IEEE division by U(k,k)), which is the
// oracle's sgetrs order bit for bit.
#include "common.cuh"
#include "device_once.h"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int SB = 128;  // rows per block
constexpr int ST = 256;  // threads
constexpr int SBP4 = SB + 4;  // shared pitch of the staged 128 x 128 tiles (16-byte rows)

// perm[i] = the original row that ends at position i after the swaps ipiv[0..n-1].
// Two phases instead of one serial chain of n swaps.  (1) A warp per chunk of 32 swaps
// composes the chunk into a list of moves "position p takes the row that was at position q
// before the chunk": lane l holds position k0 + l and, when it is the first lane naming it,
// its swap's target outside the chunk; each swap exchanges two such slots by shuffles.
// (2) One warp applies the chunks' lists in order to the identity.  An out-of-range pivot
// (below its own index or past n) counts as no swap and sets *bad = 1 (the solve is skipped).
constexpr int PERM_CHUNK = 32;
constexpr int PERM_MAX_CHUNKS = LARGE_MAX_COLS / PERM_CHUNK;
constexpr size_t PERM_SMEM = (size_t)LARGE_MAX_COLS * sizeof(short) +
                             (size_t)PERM_MAX_CHUNKS * 2 * PERM_CHUNK * sizeof(int) + PERM_MAX_CHUNKS * sizeof(int);

__global__ void __launch_bounds__(1024) large_perm_kernel(const int *ipiv, int n, int *perm, int *bad)
{
    extern __shared__ __align__(16) unsigned char psm[];
    short *P = reinterpret_cast<short *>(psm);
    int *moves = reinterpret_cast<int *>(P + LARGE_MAX_COLS);  // per chunk: (position << 16) | source
    int *count = moves + PERM_MAX_CHUNKS * 2 * PERM_CHUNK;
    __shared__ int bflag;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nch = (n + PERM_CHUNK - 1) / PERM_CHUNK;
    if (t == 0) bflag = 0;
    __syncthreads();
    for (int c = warp; c < nch; c += blockDim.x / 32)
    {
        const int k0 = c * PERM_CHUNK, kend = min(n, k0 + PERM_CHUNK);
        const int k = k0 + lane;
        int r = k < n ? ipiv[k] - 1 : k;
        if (k < n && (r < k || r >= n))
        {
            bflag = 1;
            r = k;
        }
        const bool outside = r >= kend;
        const unsigned same = __match_any_sync(0xffffffffu, r);
        const bool ownb = outside && lane == __ffs(same) - 1;  // this lane's slot B holds position r
        int srca = k, srcb = r;
        for (int j = 0; j < kend - k0; ++j)
        {
            const int bpos = __shfl_sync(0xffffffffu, r, j);
            const int owner = __ffs(__ballot_sync(0xffffffffu, ownb && r == bpos)) - 1;  // -1 inside the chunk
            const int va = __shfl_sync(0xffffffffu, srca, j);
            const bool in = bpos < kend;
            const int vin = __shfl_sync(0xffffffffu, srca, in ? bpos - k0 : 0);
            const int vout = __shfl_sync(0xffffffffu, srcb, in ? 0 : owner);
            const int vb = in ? vin : vout;
            if (lane == j) srca = vb;
            if (in && lane == bpos - k0) srca = va;
            if (!in && lane == owner) srcb = va;
        }
        const bool ma = k < kend && srca != k, mb = ownb && srcb != r;
        const unsigned ba = __ballot_sync(0xffffffffu, ma), bb = __ballot_sync(0xffffffffu, mb);
        const unsigned below = (1u << lane) - 1u;
        int *list = moves + (size_t)c * 2 * PERM_CHUNK;
        if (ma) list[__popc(ba & below)] = (k << 16) | srca;
        if (mb) list[__popc(ba) + __popc(bb & below)] = (r << 16) | srcb;
        if (lane == 0) count[c] = __popc(ba) + __popc(bb);
    }
    for (int i = t; i < n; i += blockDim.x) P[i] = (short)i;
    __syncthreads();
    if (warp == 0)
    {
        for (int c = 0; c < nch; ++c)
        {
            const int cnt = count[c];
            const int *list = moves + (size_t)c * 2 * PERM_CHUNK;
            int m0 = -1, m1 = -1;
            short v0 = 0, v1 = 0;
            if (lane < cnt)
            {
                m0 = list[lane];
                v0 = P[m0 & 0xffff];
            }
            if (lane + 32 < cnt)
            {
                m1 = list[lane + 32];
                v1 = P[m1 & 0xffff];
            }
            __syncwarp();
            if (m0 >= 0) P[m0 >> 16] = v0;
            if (m1 >= 0) P[m1 >> 16] = v1;
            __syncwarp();
        }
    }
    __syncthreads();
    if (t == 0) *bad = bflag;
    for (int i = t; i < n; i += blockDim.x) perm[i] = P[i];
}

// Y = X permuted (Y[i] = X[perm[i]]) for every right-hand side; Y is scratch (n x nrhs, ld n).
// X is X1, or slot 0 of the table Xt.
__global__ void large_gather_kernel(const float *X1, const float *const *Xt, int ldx, int n, int nrhs, const int *perm,
                                    float *Y)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * nrhs) return;
    const float *X = Xt ? slot(Xt, 0) : X1;
    const int r = (int)(e / n), i = (int)(e % n);
    Y[(int64_t)r * n + i] = X[(int64_t)r * ldx + (perm ? perm[i] : i)];
}

// X = Y, unless a pivot was out of range (X is then left as it was and info, if given, is
// the reference's -6) or a sweep's bounded wait ran out (info LARGE_WAIT_ERROR); 0 otherwise
__global__ void large_scatter_kernel(float *X1, float *const *Xt, int ldx, int n, int nrhs, const float *Y,
                                     const int *bad, int *info)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int bv = bad ? *bad : 0;
    const bool b = bv != 0;
    if (e == 0 && info) *info = bv == 1 ? -6 : (bv ? LARGE_WAIT_ERROR : 0);
    if (b || e >= (int64_t)n * nrhs) return;
    float *X = Xt ? slot(Xt, 0) : X1;
    const int r = (int)(e / n), i = (int)(e % n);
    X[(int64_t)r * ldx + i] = Y[(int64_t)r * n + i];
}

// One block step of a sweep over Y (n x nrhs, ld n).  FORWARD: diagonal block b of the unit
// lower L, then strips below; backward: diagonal block b of U (divisions), then strips above.
// Grid: 1 + the strips to update; block 0 also writes the solved block back.
template <bool FORWARD>
__global__ void __launch_bounds__(ST) large_sweep_kernel(const float *A1, const float *const *At, int lda, int n,
                                                          float *Y, int nrhs, int b, const int *bad)
{
    if (bad && *bad) return;  // uniform: nothing is solved with invalid pivots
    const float *A = At ? slot(At, 0) : A1;
    extern __shared__ __align__(16) float sm[];
    float *D = sm;                   // D[k][i] = A(b0 + i, b0 + k), pitch SBP4
    float *xs = D + SB * SBP4;       // xs[r][i]: the block's solution, pitch SB
    float *S = xs + LARGE_SOLVE_MAX_RHS * SB;  // S[k][i]: the strip's columns, pitch SBP4
    const int t = threadIdx.x;
    const int b0 = b * SB, w = min(SB, n - b0);
    const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0 && w == SB;
    stage_tile(D, SBP4, A + (int64_t)b0 * lda + b0, lda, w, w, vec);
    stage_tile(xs, SB, Y + b0, n, w, nrhs, (n & 3) == 0 && w == SB);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // the strip's columns are fetched while the diagonal block is solved
    const int s = FORWARD ? b + blockIdx.x : b - blockIdx.x;
    const int s0 = s * SB, sw = min(SB, n - s0);
    if (blockIdx.x > 0) stage_tile(S, SBP4, A + (int64_t)b0 * lda + s0, lda, sw, w, vec && sw == SB);
    __syncthreads();
    // the diagonal block in 32-row sub-blocks: each sub-block's triangle by one warp per two
    // right-hand sides (a lane per row, the solved entry broadcast by shuffle), then the
    // block's remaining rows take that sub-block's columns; per element still ascending k
    // (forward) or descending k after the division (backward)
    {
        const int lane = t & 31, warp = t >> 5;
        const int nsub = (w + 31) / 32;
        for (int si = 0; si < nsub; ++si)
        {
            const int cb = 32 * (FORWARD ? si : nsub - 1 - si), cw = min(32, w - cb);
            const int ra = warp, rb2 = warp + ST / 32;  // this warp's right-hand sides
            float *xa = xs + ra * SB + cb, *xb = xs + rb2 * SB + cb;
            const bool la = ra < nrhs, lb = rb2 < nrhs;  // warp-uniform
            float va = la && lane < cw ? xa[lane] : 0.0f;
            float vb = lb && lane < cw ? xb[lane] : 0.0f;
            if (!la && !lb)
            {
                // no right-hand side in this warp (and no dummy divisions: a zero dividend
                // takes the division's slow path)
            }
            else if (FORWARD)
            {
                for (int k = 0; k < cw; ++k)
                {
                    const float ka = __shfl_sync(0xffffffffu, va, k), kb = __shfl_sync(0xffffffffu, vb, k);
                    if (lane > k && lane < cw)
                    {
                        const float l = D[(cb + k) * SBP4 + cb + lane];
                        va = fma_rn(-l, ka, va);
                        vb = fma_rn(-l, kb, vb);
                    }
                }
            }
            else
            {
                // each lane's divisor is its own diagonal entry: reciprocal ahead of the chain
                const float dl = lane < cw ? D[(cb + lane) * SBP4 + cb + lane] : 1.0f;
                const float yl = div_prepare(dl);
                const bool okl = div_range(dl);
                for (int k = cw - 1; k >= 0; --k)
                {
                    if (lane == k)
                    {
                        va = div_by(va, dl, yl, okl);
                        if (lb) vb = div_by(vb, dl, yl, okl);
                    }
                    const float ka = __shfl_sync(0xffffffffu, va, k), kb = __shfl_sync(0xffffffffu, vb, k);
                    if (lane < k)
                    {
                        const float u = D[(cb + k) * SBP4 + cb + lane];
                        va = fma_rn(-u, ka, va);
                        vb = fma_rn(-u, kb, vb);
                    }
                }
            }
            if (la && lane < cw) xa[lane] = va;
            if (lb && lane < cw) xb[lane] = vb;
            __syncthreads();
            // the rest of the block: rows after the sub-block (forward) or before it (backward)
            const int r0 = FORWARD ? cb + cw : 0, r1 = FORWARD ? w : cb;
            const int nrow = r1 - r0;
            for (int e = t; e < nrow * nrhs; e += ST)
            {
                const int i = r0 + e % nrow, r = e / nrow;
                float *x = xs + r * SB;
                float acc = x[i];
                for (int kk = 0; kk < cw; ++kk)
                {
                    const int k = FORWARD ? kk : cw - 1 - kk;
                    acc = fma_rn(-D[(cb + k) * SBP4 + i], x[cb + k], acc);
                }
                x[i] = acc;
            }
            __syncthreads();
        }
    }
    if (blockIdx.x == 0)
    {
        for (int e = t; e < nrhs * SB; e += ST)
        {
            const int r = e / SB, i = e % SB;
            if (i < w) Y[(int64_t)r * n + b0 + i] = xs[r * SB + i];
        }
        return;
    }
    // a strip of 128 rows below (forward) or above (backward): Y[rows] -= A[rows, block] x
    // thread: row s0 + (t % 128), right-hand sides (t / 128), +2, ... (at most eight)
    constexpr int RPT = LARGE_SOLVE_MAX_RHS / (ST / SB);
    const int i = t % SB, r0 = t / SB;
    tile_wait();  // the strip (each thread its own copies), then everyone's
    __syncthreads();
    float acc[RPT];
    if (i >= sw) return;
#pragma unroll
    for (int q = 0; q < RPT; ++q)
    {
        const int r = r0 + q * (ST / SB);
        acc[q] = r < nrhs ? Y[(int64_t)r * n + s0 + i] : 0.0f;
    }
    for (int kk = 0; kk < w; ++kk)
    {
        const int k = FORWARD ? kk : w - 1 - kk;
        const float l = S[k * SBP4 + i];
#pragma unroll
        for (int q = 0; q < RPT; ++q) acc[q] = fma_rn(-l, xs[(r0 + q * (ST / SB)) * SB + k], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q)
    {
        const int r = r0 + q * (ST / SB);
        if (r < nrhs) Y[(int64_t)r * n + s0 + i] = acc[q];
    }
}


// Inverses of the 128 x 128 diagonal blocks of the factors, for the refinement's solves (whose
// results need not follow the oracle's order): block (b, which) inverts the unit-lower L
// block (which 0) or the upper U block (which 1) of diagonal block b, thread j computing
// column j by substitution against e_j in shared memory.  Stored column-major per (b, which);
// a ragged last block of order w is inverted as w x w (the rest of the 128 x 128 identity).
__global__ void __launch_bounds__(SB, 1) large_diag_inverse(const float *A, int lda, int n, float *inv)
{
    extern __shared__ __align__(16) float dsm[];
    float *T = dsm;              // T[k][i] = A(b0 + i, b0 + k), pitch SBP4
    float *Y = dsm + SB * SBP4;  // Y[j][i]: column j of the inverse, pitch SBP4
    const int b = blockIdx.x, which = blockIdx.y, j = threadIdx.x;
    const int b0 = b * SB, w = min(SB, n - b0);
    const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0 && w == SB;
    stage_tile(T, SBP4, A + (int64_t)b0 * lda + b0, lda, w, w, vec);
    tile_wait();
    __syncthreads();
    float *y = Y + j * SBP4;
    for (int i = 0; i < SB; ++i) y[i] = 0.0f;
    if (j >= w)
        y[j] = 1.0f;
    else if (which == 0)
    {
        y[j] = 1.0f;
        for (int i = j + 1; i < w; ++i)
        {
            float acc = 0.0f;
            for (int k = j; k < i; ++k) acc = fma_rn(-T[k * SBP4 + i], y[k], acc);
            y[i] = acc;
        }
    }
    else
    {
        y[j] = 1.0f / T[j * SBP4 + j];
        for (int i = j - 1; i >= 0; --i)
        {
            float acc = 0.0f;
            for (int k = i + 1; k <= j; ++k) acc = fma_rn(-T[k * SBP4 + i], y[k], acc);
            y[i] = acc / T[i * SBP4 + i];
        }
    }
    __syncthreads();
    float *dst = inv + ((size_t)b * 2 + which) * SB * SB;
    for (int e = threadIdx.x; e < SB * SB; e += SB) dst[e] = Y[(e / SB) * SBP4 + e % SB];
}

// The same sweep as one cooperative launch: block s owns 128-row strip s for the whole sweep.
// It applies the finished blocks b in order (forward: b < s ascending; backward: b > s
// descending), each as soon as block b has published its solution (flag[b] == epoch), with
// the next factor tile streaming into a second buffer meanwhile, then solves its own diagonal
// block and publishes it.  Per element the order is that of the per-block sweep (bit-identical results).  Waits
// are bounded: one that runs out sets *bad to 2 and the block goes on (the solve is then
// reported failed, never hangs).  All blocks are resident (cooperative launch), so every
// flag is eventually set.
constexpr long long FLAG_WAIT = 1ll << 22;
static_assert(SB == 16 * (ST / 32) && LARGE_SOLVE_MAX_RHS == 16, "a warp's 16 rows, a lane's four rows and two right-hand sides");

template <bool FORWARD>
__global__ void __launch_bounds__(ST, 1) large_sweep_coop(const float *A1, const float *const *At, int lda, int n,
                                                           float *Y, int nrhs, int *flags, int epoch, int *bad,
                                                           const float *dinv)
{
    extern __shared__ __align__(16) float sm[];
    float *D = sm;                            // this strip's diagonal block, pitch SBP4
    float *Lbuf = D + SB * SBP4;              // two factor tiles: the one applied, the next one
    float *xs = Lbuf + 2 * SB * SBP4;         // this strip's right-hand sides, xs[r][i]
    float *xb = xs + LARGE_SOLVE_MAX_RHS * SB;  // the applied block's solution
    __shared__ int stop;
    if (*bad == 1) return;  // uniform: invalid pivots, nothing is solved
    const float *A = At ? slot(At, 0) : A1;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nb = gridDim.x;
    const int sidx = blockIdx.x;
    const int s = FORWARD ? sidx : nb - 1 - sidx;  // the strip; forward strips start at the top
    const int s0 = s * SB, sw = min(SB, n - s0);
    const bool vec = (reinterpret_cast<uintptr_t>(A) & 15u) == 0 && (lda & 3) == 0;
    if (dinv)  // the diagonal block's inverse (128 x 128, column-major, 16-byte aligned)
        stage_tile(D, SBP4, dinv + ((size_t)s * 2 + (FORWARD ? 0 : 1)) * SB * SB, SB, SB, SB, true);
    else
        stage_tile(D, SBP4, A + (int64_t)s0 * lda + s0, lda, sw, sw, vec && sw == SB);
    stage_tile(xs, SB, Y + s0, n, sw, nrhs, (n & 3) == 0 && sw == SB);
    if (t == 0) stop = 0;
    const int nprev = FORWARD ? s : nb - 1 - s;  // blocks applied before this strip's own
    auto block_of = [&](int q) { return FORWARD ? q : nb - 1 - q; };
    auto stage_block = [&](int q)
    {
        const int b = block_of(q);
        stage_tile(Lbuf + (size_t)(q & 1) * SB * SBP4, SBP4, A + (int64_t)(b * SB) * lda + s0, lda, sw,
                   min(SB, n - b * SB), vec && sw == SB);
    };
    if (nprev > 0) stage_block(0);
    tile_wait();
    __syncthreads();
    // register blocking: warp w owns rows 16w .. 16w + 15 of the strip for every right-hand
    // side, lane l rows 16w + 4(l % 4) .. + 3 and the right-hand sides 2(l / 4), 2(l / 4) + 1,
    // so that each warp reads a factor tile's rows once (the lanes of a row quad share the
    // loads) and the applied solution is kept k-major, xb[k][r].  Per element the updates still
    // run in the sweep's order; the columns past nrhs compute on junk and are never stored.
    const int row4 = 16 * warp + 4 * (lane & 3), rp = 2 * (lane >> 2);
    for (int q = 0; q < nprev; ++q)
    {
        const int b = block_of(q), b0 = b * SB, bw = min(SB, n - b0);
        if (q + 1 < nprev) stage_block(q + 1);  // the next tile streams in during this one
        // block b's solution
        if (t == 0)
        {
            long long it = 0;
            while (true)
            {
                int f;
                asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(f) : "l"(flags + b) : "memory");
                if (f == epoch) break;
                if (++it > FLAG_WAIT)
                {
                    atomicExch(bad, 2);
                    stop = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        __syncthreads();
        if (stop) break;  // uniform
        for (int e = t; e < nrhs * SB; e += ST)
        {
            const int r = e / SB, k = e % SB;
            xb[k * LARGE_SOLVE_MAX_RHS + r] = k < bw ? __ldcg(Y + (int64_t)r * n + b0 + k) : 0.0f;
        }
        if (q + 1 < nprev)
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        else
            tile_wait();
        __syncthreads();
        // this strip minus L(s, b) x_b (or U(s, b) x_b), ascending (descending) k
        const float *L = Lbuf + (size_t)(q & 1) * SB * SBP4;
        {
            float4 a0 = *reinterpret_cast<const float4 *>(xs + rp * SB + row4);
            float4 a1 = *reinterpret_cast<const float4 *>(xs + (rp + 1) * SB + row4);
#pragma unroll 8
            for (int kk = 0; kk < bw; ++kk)
            {
                const int k = FORWARD ? kk : bw - 1 - kk;
                const float4 l = *reinterpret_cast<const float4 *>(L + k * SBP4 + row4);
                const float2 x = *reinterpret_cast<const float2 *>(xb + k * LARGE_SOLVE_MAX_RHS + rp);
                a0.x = fma_rn(-l.x, x.x, a0.x);
                a0.y = fma_rn(-l.y, x.x, a0.y);
                a0.z = fma_rn(-l.z, x.x, a0.z);
                a0.w = fma_rn(-l.w, x.x, a0.w);
                a1.x = fma_rn(-l.x, x.y, a1.x);
                a1.y = fma_rn(-l.y, x.y, a1.y);
                a1.z = fma_rn(-l.z, x.y, a1.z);
                a1.w = fma_rn(-l.w, x.y, a1.w);
            }
            *reinterpret_cast<float4 *>(xs + rp * SB + row4) = a0;
            *reinterpret_cast<float4 *>(xs + (rp + 1) * SB + row4) = a1;
        }
        __syncthreads();
    }
    tile_wait();  // nothing of a stopped sweep is left in flight
    if (dinv)
    {
        // x = inv xs (ascending k from zero): xs goes k-major into xb, the product back into xs
        for (int e = t; e < LARGE_SOLVE_MAX_RHS * SB; e += ST)
        {
            const int r = e / SB, k = e % SB;
            xb[k * LARGE_SOLVE_MAX_RHS + r] = r < nrhs ? xs[r * SB + k] : 0.0f;
        }
        __syncthreads();
        float4 a0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), a1 = a0;
#pragma unroll 8
        for (int k = 0; k < sw; ++k)
        {
            const float4 d = *reinterpret_cast<const float4 *>(D + k * SBP4 + row4);
            const float2 x = *reinterpret_cast<const float2 *>(xb + k * LARGE_SOLVE_MAX_RHS + rp);
            a0.x = fma_rn(d.x, x.x, a0.x);
            a0.y = fma_rn(d.y, x.x, a0.y);
            a0.z = fma_rn(d.z, x.x, a0.z);
            a0.w = fma_rn(d.w, x.x, a0.w);
            a1.x = fma_rn(d.x, x.y, a1.x);
            a1.y = fma_rn(d.y, x.y, a1.y);
            a1.z = fma_rn(d.z, x.y, a1.z);
            a1.w = fma_rn(d.w, x.y, a1.w);
        }
        *reinterpret_cast<float4 *>(xs + rp * SB + row4) = a0;
        *reinterpret_cast<float4 *>(xs + (rp + 1) * SB + row4) = a1;
        __syncthreads();
    }
    else
    // the diagonal block: as in the per-block sweep
    {
        const int nsub = (sw + 31) / 32;
        for (int si = 0; si < nsub; ++si)
        {
            const int cb = 32 * (FORWARD ? si : nsub - 1 - si), cw = min(32, sw - cb);
            const int ra = warp, rb2 = warp + ST / 32;
            float *xa = xs + ra * SB + cb, *xc = xs + rb2 * SB + cb;
            const bool la = ra < nrhs, lb = rb2 < nrhs;
            float va = la && lane < cw ? xa[lane] : 0.0f;
            float vb = lb && lane < cw ? xc[lane] : 0.0f;
            if (!la && !lb)
            {
                // no right-hand side in this warp (and no dummy divisions: a zero dividend
                // takes the division's slow path)
            }
            else if (FORWARD)
            {
                for (int k = 0; k < cw; ++k)
                {
                    const float ka = __shfl_sync(0xffffffffu, va, k), kb = __shfl_sync(0xffffffffu, vb, k);
                    if (lane > k && lane < cw)
                    {
                        const float l = D[(cb + k) * SBP4 + cb + lane];
                        va = fma_rn(-l, ka, va);
                        vb = fma_rn(-l, kb, vb);
                    }
                }
            }
            else
            {
                // each lane's divisor is its own diagonal entry: reciprocal ahead of the chain
                const float dl = lane < cw ? D[(cb + lane) * SBP4 + cb + lane] : 1.0f;
                const float yl = div_prepare(dl);
                const bool okl = div_range(dl);
                for (int k = cw - 1; k >= 0; --k)
                {
                    if (lane == k)
                    {
                        va = div_by(va, dl, yl, okl);
                        if (lb) vb = div_by(vb, dl, yl, okl);
                    }
                    const float ka = __shfl_sync(0xffffffffu, va, k), kb = __shfl_sync(0xffffffffu, vb, k);
                    if (lane < k)
                    {
                        const float u = D[(cb + k) * SBP4 + cb + lane];
                        va = fma_rn(-u, ka, va);
                        vb = fma_rn(-u, kb, vb);
                    }
                }
            }
            if (la && lane < cw) xa[lane] = va;
            if (lb && lane < cw) xc[lane] = vb;
            __syncthreads();
            const int q0 = FORWARD ? cb + cw : 0, q1 = FORWARD ? sw : cb;
            const int nrow = q1 - q0;
            for (int e = t; e < nrow * nrhs; e += ST)
            {
                const int ii = q0 + e % nrow, r = e / nrow;
                float *x = xs + r * SB;
                float acc = x[ii];
                for (int kk = 0; kk < cw; ++kk)
                {
                    const int k = FORWARD ? kk : cw - 1 - kk;
                    acc = fma_rn(-D[(cb + k) * SBP4 + ii], x[cb + k], acc);
                }
                x[ii] = acc;
            }
            __syncthreads();
        }
    }
    // publish: the strip's solution, then its flag
    for (int e = t; e < nrhs * SB; e += ST)
    {
        const int r = e / SB, k = e % SB;
        if (k < sw) Y[(int64_t)r * n + s0 + k] = xs[r * SB + k];
    }
    __syncthreads();
    if (t == 0)
    {
        __threadfence();
        asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flags + s), "r"(epoch) : "memory");
    }
}

}  // namespace

size_t large_solve_scratch_bytes(int n, int nrhs)
{
    // Y (n x nrhs), the composed pivots (n), the sweeps' flags (one per 128-row block, two sweeps)
    return (size_t)n * nrhs * sizeof(float) + (size_t)n * sizeof(int) + 2 * ((size_t)(n + SB - 1) / SB) * sizeof(int) +
           64;
}

cudaError_t launch_large_perm(const int *ipiv, int n, int *perm, int *bad, cudaStream_t stream)
{
    if (n > LARGE_MAX_COLS) return cudaErrorInvalidValue;
    static std::atomic<unsigned long long> attr{0};
    cudaError_t e = once_per_device(attr, [] {
        return cudaFuncSetAttribute(large_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PERM_SMEM);
    });
    if (e != cudaSuccess) return e;
    large_perm_kernel<<<1, 1024, PERM_SMEM, stream>>>(ipiv, n, perm, bad);
    return cudaGetLastError();
}

cudaError_t launch_large_diag_inverses(const float *A, int lda, int n, float *inv, cudaStream_t stream)
{
    static std::atomic<unsigned long long> attr{0};
    const size_t smem = 2 * (size_t)SB * SBP4 * sizeof(float);
    cudaError_t e = once_per_device(attr, [smem] {
        return cudaFuncSetAttribute(large_diag_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    if (e != cudaSuccess) return e;
    large_diag_inverse<<<dim3((n + SB - 1) / SB, 2), SB, smem, stream>>>(A, lda, n, inv);
    return cudaGetLastError();
}

size_t large_diag_inverse_bytes(int n) { return (size_t)((n + SB - 1) / SB) * 2 * SB * SB * sizeof(float); }

cudaError_t launch_getrs_large(const float *A, const float *const *At, int lda, int n, const int *ipiv, float *X,
                               float *const *Xt, int ldx, int nrhs, void *scratch, int *bad, int *info,
                               cudaStream_t stream, const int *perm_in, const float *dinv)
{
    if (n > LARGE_MAX_COLS || nrhs > LARGE_SOLVE_MAX_RHS) return cudaErrorInvalidValue;
    float *Y = static_cast<float *>(scratch);
    int *perm = reinterpret_cast<int *>(Y + (size_t)n * nrhs);
    const size_t smem = (2 * SB * SBP4 + (size_t)LARGE_SOLVE_MAX_RHS * SB) * sizeof(float);
    static std::atomic<unsigned long long> attr{0};
    {
        cudaError_t e = once_per_device(attr, [smem] {
            cudaError_t r = cudaFuncSetAttribute(large_sweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (r == cudaSuccess)
                r = cudaFuncSetAttribute(large_sweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
            return r;
        });
        if (e != cudaSuccess) return e;
    }
    const int *use = perm_in;  // a permutation composed earlier (its *bad already set)
    if (!use && ipiv)
    {
        cudaError_t e = launch_large_perm(ipiv, n, perm, bad, stream);
        if (e != cudaSuccess) return e;
        use = perm;
    }
    else if (!use)
    {
        cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), stream);
        if (e != cudaSuccess) return e;
    }
    const int64_t total = (int64_t)n * nrhs;
    large_gather_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(X, Xt, ldx, n, nrhs, use, Y);
    const int nb = (n + SB - 1) / SB;
    // each sweep as one cooperative launch where all its blocks can be resident, else a launch
    // per 128-row block
    static std::atomic<int> coop_cache[ONCE_MAX_DEVICES];
    const size_t csmem = (3 * SB * SBP4 + 2 * (size_t)LARGE_SOLVE_MAX_RHS * SB) * sizeof(float);
    const int coop_ok = value_per_device(coop_cache, [csmem] {
        int dev = 0, attr_coop = 0, per_sm = 0, sms = 0, ok = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&attr_coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && attr_coop &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaFuncSetAttribute(large_sweep_coop<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem) ==
                cudaSuccess &&
            cudaFuncSetAttribute(large_sweep_coop<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, large_sweep_coop<true>, ST, csmem) == cudaSuccess)
            ok = per_sm * sms;  // blocks that can be resident at once
        cudaGetLastError();
        return ok;
    });
    if (coop_ok >= nb)
    {
        int *flags = perm + n;  // two sweeps' flags, cleared for this solve
        cudaError_t e0 = cudaMemsetAsync(flags, 0, 2 * (size_t)nb * sizeof(int), stream);
        if (e0 != cudaSuccess) return e0;
        static std::atomic<int> epoch{0};
        const int ep = (epoch.fetch_add(1) & 0x3fffffff) + 1;  // positive, differs from the cleared 0
        const float *a1 = A;
        const float *const *at = At;
        float *y = Y;
        int nn = n, nr = nrhs, ld = lda, epv = ep;
        int *fl = flags, *fb = flags + nb;
        const float *dv = dinv;
        void *fwd[] = {(void *)&a1, (void *)&at, (void *)&ld, (void *)&nn, (void *)&y, (void *)&nr, (void *)&fl,
                       (void *)&epv, (void *)&bad, (void *)&dv};
        cudaError_t e = cudaLaunchCooperativeKernel((const void *)large_sweep_coop<true>, dim3(nb), dim3(ST), fwd,
                                                    csmem, stream);
        if (e != cudaSuccess) return e;
        void *bwd[] = {(void *)&a1, (void *)&at, (void *)&ld, (void *)&nn, (void *)&y, (void *)&nr, (void *)&fb,
                       (void *)&epv, (void *)&bad, (void *)&dv};
        e = cudaLaunchCooperativeKernel((const void *)large_sweep_coop<false>, dim3(nb), dim3(ST), bwd, csmem, stream);
        if (e != cudaSuccess) return e;
    }
    else
    {
        for (int b = 0; b < nb; ++b)
            large_sweep_kernel<true><<<nb - b, ST, smem, stream>>>(A, At, lda, n, Y, nrhs, b, bad);
        for (int b = nb - 1; b >= 0; --b)
            large_sweep_kernel<false><<<b + 1, ST, smem, stream>>>(A, At, lda, n, Y, nrhs, b, bad);
    }
    large_scatter_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(X, Xt, ldx, n, nrhs, Y, bad, info);
    return cudaGetLastError();
}

}  // namespace ops_solver
