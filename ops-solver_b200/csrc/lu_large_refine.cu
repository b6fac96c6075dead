// lu_large_refine.cu -- FP64-residual iterative refinement for one large matrix (orders above
// the batched kernels, up to 8192, at most 16 right-hand sides) over the whole GPU.  The
// batched refinement (refine.cu) gives one block a whole system; here the residual
// r = b - A x (FP64 accumulation over the original FP32 A) is split over 128-row blocks and
// 1024-column chunks, and the chunks are summed in a fixed order (deterministic).  The
// decisions follow the batched refinement: converged when the normwise backward error
// ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol; a correction that does not halve it
// ends the iteration, and one that makes it worse is taken back.
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int RB = 128;    // rows per block
constexpr int CC = 1024;   // columns per chunk
constexpr int XS = 64;     // x rows staged at a time
constexpr int MAXR = LARGE_SOLVE_MAX_RHS;
static_assert(MAXR == 16 && RB % 2 == 0, "two rows and eight right-hand sides per thread");

__global__ void lir_copy_in(const float *const *B, int ldb, int n, int nrhs, float *r32)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * nrhs) return;
    const float *b = slot(B, 0);
    const int r = (int)(e / n), i = (int)(e % n);
    r32[e] = b[(int64_t)r * ldb + i];
}

// first: x64 = d; later, for running right-hand sides: xprev = x64, x64 += d
__global__ void lir_update(LargeIr s, int n, int nrhs, int first)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * nrhs) return;
    const int r = (int)(e / n);
    const double d = (double)s.r32[e];
    if (first)
        s.x64[e] = d;
    else if (s.state[r] == LIR_RUNNING)
    {
        s.xprev[e] = s.x64[e];
        s.x64[e] += d;
    }
}

// partial sums over one column chunk: part[chunk][r][i] = sum_j A(i, j) x(j, r), and the
// chunk's |A| row sums
__global__ void __launch_bounds__(RB) lir_partial(const float *const *Aarr, int lda, int n, int nrhs, LargeIr s)
{
    // register blocking: thread (p = t % 64, h = t / 64) owns rows 2p, 2p + 1 of the block and
    // right-hand sides 8h .. 8h + 7, so each staged x pair feeds four FMAs; per element the
    // products still accumulate in ascending column order
    __shared__ __align__(16) double xs[XS][MAXR];
    const float *A = slot(Aarr, 0);
    const int t = threadIdx.x;
    const int p = t % (RB / 2), h = t / (RB / 2);
    const int i0 = blockIdx.x * RB + 2 * p;
    const int j0 = blockIdx.y * CC, j1 = min(n, j0 + CC);
    double acc[2][MAXR / 2];
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int r = 0; r < MAXR / 2; ++r) acc[e][r] = 0.0;
    double asum[2] = {0.0, 0.0};
    const bool r0ok = i0 < n, r1ok = i0 + 1 < n;
    for (int jb = j0; jb < j1; jb += XS)
    {
        __syncthreads();
        for (int e = t; e < XS * MAXR; e += RB)
        {
            // consecutive threads: consecutive right-hand sides (conflict-free shared stores;
            // x is small and read from L2)
            const int r = e % MAXR, jj = e / MAXR;
            xs[jj][r] = (jb + jj < j1 && r < nrhs) ? s.x64[(int64_t)r * n + jb + jj] : 0.0;
        }
        __syncthreads();
        if (r0ok)
        {
            const int je = min(XS, j1 - jb);
            for (int jj = 0; jj < je; jj += 16)
            {
                float av[16][2];  // sixteen columns of the row pair in flight before their products
#pragma unroll
                for (int u = 0; u < 16; ++u)
                {
                    const float *col = A + (int64_t)(jb + jj + u) * lda + i0;
                    av[u][0] = jj + u < je ? col[0] : 0.0f;
                    av[u][1] = jj + u < je && r1ok ? col[1] : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < 16; ++u)
                {
                    const double a0 = (double)av[u][0], a1 = (double)av[u][1];
                    asum[0] += fabs(a0);
                    asum[1] += fabs(a1);
                    const double2 *xr = reinterpret_cast<const double2 *>(&xs[jj + u][h * (MAXR / 2)]);
#pragma unroll
                    for (int q = 0; q < MAXR / 4; ++q)
                    {
                        const double2 x = xr[q];
                        acc[0][2 * q] = fma(a0, x.x, acc[0][2 * q]);
                        acc[0][2 * q + 1] = fma(a0, x.y, acc[0][2 * q + 1]);
                        acc[1][2 * q] = fma(a1, x.x, acc[1][2 * q]);
                        acc[1][2 * q + 1] = fma(a1, x.y, acc[1][2 * q + 1]);
                    }
                }
            }
        }
    }
    if (!r0ok) return;
#pragma unroll
    for (int e = 0; e < 2; ++e)
    {
        if (e == 1 && !r1ok) break;
#pragma unroll
        for (int r = 0; r < MAXR / 2; ++r)  // static indices: acc stays in registers
            if (h * (MAXR / 2) + r < nrhs)
                s.part[((int64_t)blockIdx.y * MAXR + h * (MAXR / 2) + r) * n + i0 + e] = acc[e][r];
        if (h == 0) s.apart[(int64_t)blockIdx.y * n + i0 + e] = asum[e];
    }
}

// r = b - sum of the chunks (in chunk order) for every right-hand side; the FP32 copy for the
// next correction solve; per-block maxima of |r|, |x|, |b| and the |A| row sums
__global__ void __launch_bounds__(RB) lir_finish_rows(const float *const *B, int ldb, int n, int nrhs, int nch,
                                                      LargeIr s)
{
    __shared__ double red[4][RB];
    const int t = threadIdx.x;
    const int i = blockIdx.x * RB + t;
    const float *b = slot(B, 0);
    double arow = 0.0;
    if (i < n)
        for (int c = 0; c < nch; ++c) arow += s.apart[(int64_t)c * n + i];
    for (int r = 0; r < nrhs; ++r)
    {
        double rm = 0.0, xm = 0.0, bm = 0.0;
        if (i < n)
        {
            double ax = 0.0;
            for (int c = 0; c < nch; ++c) ax += s.part[((int64_t)c * MAXR + r) * n + i];
            const double bv = (double)b[(int64_t)r * ldb + i];
            const double res = bv - ax;
            s.r32[(int64_t)r * n + i] = (float)res;
            rm = fabs(res);
            xm = fabs(s.x64[(int64_t)r * n + i]);
            bm = fabs(bv);
        }
        red[0][t] = rm;
        red[1][t] = xm;
        red[2][t] = bm;
        __syncthreads();
        for (int h = RB / 2; h > 0; h >>= 1)
        {
            if (t < h)
                for (int q = 0; q < 3; ++q) red[q][t] = fmax(red[q][t], red[q][t + h]);
            __syncthreads();
        }
        if (t == 0)
            for (int q = 0; q < 3; ++q) s.bmax[((int64_t)blockIdx.x * MAXR + r) * 3 + q] = red[q][0];
        __syncthreads();
    }
    red[3][t] = arow;
    __syncthreads();
    for (int h = RB / 2; h > 0; h >>= 1)
    {
        if (t < h) red[3][t] = fmax(red[3][t], red[3][t + h]);
        __syncthreads();
    }
    if (t == 0) s.amax[blockIdx.x] = red[3][0];
}

// one thread per right-hand side: the backward error and the decision
__global__ void lir_decide(int n, int nrhs, int nblocks, double tol, LargeIr s, int first)
{
    const int r = threadIdx.x;
    double anorm = 0.0;
    for (int q = 0; q < nblocks; ++q) anorm = fmax(anorm, s.amax[q]);
    if (r < nrhs)
    {
        double rm = 0.0, xm = 0.0, bm = 0.0;
        for (int q = 0; q < nblocks; ++q)
        {
            rm = fmax(rm, s.bmax[((int64_t)q * MAXR + r) * 3 + 0]);
            xm = fmax(xm, s.bmax[((int64_t)q * MAXR + r) * 3 + 1]);
            bm = fmax(bm, s.bmax[((int64_t)q * MAXR + r) * 3 + 2]);
        }
        const double den = anorm * xm + bm;
        const double be = den > 0.0 ? rm / den : (rm > 0.0 ? INFINITY : 0.0);
        int st = s.state[r];
        if (first)
        {
            s.berr[r] = be;
            st = be <= tol ? LIR_CONVERGED : LIR_RUNNING;
        }
        else if (st == LIR_RUNNING)
        {
            if (be <= tol)
            {
                s.berr[r] = be;
                s.iters[r] += 1;
                st = LIR_CONVERGED;
            }
            else if (be <= 0.5 * s.berr[r])
            {
                s.berr[r] = be;
                s.iters[r] += 1;
            }
            else if (be <= s.berr[r])
            {
                s.berr[r] = be;  // still better, but no longer halving: keep it and stop
                s.iters[r] += 1;
                st = LIR_STALLED;
            }
            else
            {
                s.take[r] = 1;  // worse: the previous iterate is restored
                st = LIR_STALLED;
            }
        }
        s.state[r] = st;
    }
    __syncthreads();
    if (r == 0)
    {
        int any = 0;
        for (int q = 0; q < nrhs; ++q) any |= s.state[q] == LIR_RUNNING;
        *s.running = any;
    }
}

__global__ void lir_take_back(LargeIr s, int n, int nrhs)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * nrhs) return;
    const int r = (int)(e / n);
    if (s.take[r]) s.x64[e] = s.xprev[e];
}

__global__ void lir_clear_take(LargeIr s, int nrhs)
{
    if (threadIdx.x < (unsigned)nrhs) s.take[threadIdx.x] = 0;
}

__global__ void lir_write_x(float *const *X, int ldx, int n, int nrhs, LargeIr s)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * nrhs) return;
    float *x = slot(X, 0);
    const int r = (int)(e / n), i = (int)(e % n);
    x[(int64_t)r * ldx + i] = (float)s.x64[e];
}

__global__ void lir_report(int nrhs, LargeIr s, double *berr, int *iters, int failed)
{
    if (threadIdx.x != 0) return;
    double be = 0.0;
    int it = 0;
    for (int r = 0; r < nrhs; ++r)
    {
        be = fmax(be, s.berr[r]);
        it = max(it, s.iters[r]);
    }
    if (berr) *berr = failed ? NAN : be;
    if (iters) *iters = failed ? 0 : it;
}

}  // namespace

size_t large_ir_bytes(int n, int nrhs)
{
    const size_t v = (size_t)n * nrhs;
    const int nch = (n + CC - 1) / CC, nbl = (n + RB - 1) / RB;
    return v * sizeof(double) * 2 + v * sizeof(float) + (size_t)nch * MAXR * n * sizeof(double) +
           (size_t)nch * n * sizeof(double) + (size_t)nbl * MAXR * 3 * sizeof(double) + (size_t)nbl * sizeof(double) +
           MAXR * (sizeof(double) + 3 * sizeof(int)) + 64 + 16 * 256;
}

LargeIr large_ir_carve(void *base, int n, int nrhs)
{
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    char *p = static_cast<char *>(base);
    const size_t v = (size_t)n * nrhs;
    const int nch = (n + CC - 1) / CC, nbl = (n + RB - 1) / RB;
    LargeIr s;
    s.x64 = reinterpret_cast<double *>(p), p += up(v * sizeof(double));
    s.xprev = reinterpret_cast<double *>(p), p += up(v * sizeof(double));
    s.r32 = reinterpret_cast<float *>(p), p += up(v * sizeof(float));
    s.part = reinterpret_cast<double *>(p), p += up((size_t)nch * MAXR * n * sizeof(double));
    s.apart = reinterpret_cast<double *>(p), p += up((size_t)nch * n * sizeof(double));
    s.bmax = reinterpret_cast<double *>(p), p += up((size_t)nbl * MAXR * 3 * sizeof(double));
    s.amax = reinterpret_cast<double *>(p), p += up((size_t)nbl * sizeof(double));
    s.berr = reinterpret_cast<double *>(p), p += up(MAXR * sizeof(double));
    s.state = reinterpret_cast<int *>(p), p += up(MAXR * sizeof(int));
    s.iters = reinterpret_cast<int *>(p), p += up(MAXR * sizeof(int));
    s.take = reinterpret_cast<int *>(p), p += up(MAXR * sizeof(int));
    s.running = reinterpret_cast<int *>(p);
    return s;
}

cudaError_t launch_lir_init(const LargeIr &s, const float *const *B, int ldb, int n, int nrhs, cudaStream_t st)
{
    const int64_t v = (int64_t)n * nrhs;
    cudaError_t e = cudaMemsetAsync(s.iters, 0, MAXR * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.take, 0, MAXR * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.state, 0, MAXR * sizeof(int), st);
    if (e != cudaSuccess) return e;
    lir_copy_in<<<(unsigned)((v + 255) / 256), 256, 0, st>>>(B, ldb, n, nrhs, s.r32);
    return cudaGetLastError();
}

cudaError_t launch_lir_update(const LargeIr &s, int n, int nrhs, int first, cudaStream_t st)
{
    const int64_t v = (int64_t)n * nrhs;
    lir_update<<<(unsigned)((v + 255) / 256), 256, 0, st>>>(s, n, nrhs, first);
    return cudaGetLastError();
}

cudaError_t launch_lir_residual(const LargeIr &s, const float *const *A, int lda, const float *const *B, int ldb,
                                int n, int nrhs, double tol, int first, cudaStream_t st)
{
    const int nch = (n + CC - 1) / CC, nbl = (n + RB - 1) / RB;
    const int64_t v = (int64_t)n * nrhs;
    lir_partial<<<dim3(nbl, nch), RB, 0, st>>>(A, lda, n, nrhs, s);
    lir_finish_rows<<<nbl, RB, 0, st>>>(B, ldb, n, nrhs, nch, s);
    lir_decide<<<1, 32, 0, st>>>(n, nrhs, nbl, tol, s, first);
    lir_take_back<<<(unsigned)((v + 255) / 256), 256, 0, st>>>(s, n, nrhs);
    lir_clear_take<<<1, 32, 0, st>>>(s, nrhs);
    return cudaGetLastError();
}

cudaError_t launch_lir_finish(const LargeIr &s, float *const *X, int ldx, int n, int nrhs, double *berr, int *iters,
                              int failed, cudaStream_t st)
{
    const int64_t v = (int64_t)n * nrhs;
    if (!failed) lir_write_x<<<(unsigned)((v + 255) / 256), 256, 0, st>>>(X, ldx, n, nrhs, s);
    lir_report<<<1, 32, 0, st>>>(nrhs, s, berr, iters, failed);
    return cudaGetLastError();
}

}  // namespace ops_solver
