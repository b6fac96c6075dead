// api_refine.cpp -- aclsolverSgesvIrBatched: LU factorisation in a chosen precision plus
// FP64-residual iterative refinement.
//
// The reference's solve path is aclsolverSgetrf (src/sgetrf/sgetrf_host.cpp:96) followed by
// aclsolverSgetrs (src/sgetrs/sgetrs_host.cpp:131), FP32 throughout; this entry adds the
// refinement loop around the same factor/solve pair and lets the trailing update of the
// factorisation run on the tensor cores.
//
// Schedule (all on the handle stream, no host synchronisation):
//   LU <- A (copy);  getrf(LU, precision)
//   r32 <- B;  solve(LU, r32);  x64 <- r32
//   maxIter times: residual (FP64) -> state;  solve(LU, r32) for running systems;  x64 += r32
//   residual;  X <- x64
#include <stdio.h>

#include <algorithm>

#include "handle.h"
#include "launch.h"
#include "refine.h"

using namespace ops_solver;

namespace
{
constexpr int SMALL_N = 64;

size_t round_up(size_t v) { return (v + 255) & ~size_t(255); }

// One matrix above the batched orders: the whole-GPU factorisation and solves, the residual
// split over the GPU.  Unlike the batched schedule this one reads two flags back (info after
// the factorisation, and whether a system still refines after each residual), so the call
// returns after its work is done.
aclsolverStatus_t gesv_ir_large(Handle *h, int mode, int n, int nrhs, const float *const Aarray[], int lda,
                                const float *const Barray[], int ldb, float *const Xarray[], int ldx, int maxIter,
                                double tol, int *iterArray, double *berrArray, int *infoArray)
{
    cudaStream_t st = h->stream;
    const size_t sizes[9] = {(size_t)n * n * sizeof(float), (size_t)n * sizeof(int), sizeof(LargeStatus),
                             large_solve_scratch_bytes(n, nrhs), 256, large_ir_bytes(n, nrhs),
                             mode != 0 ? umma_scratch_bytes(n, n) : 0, (size_t)n * sizeof(int),
                             large_diag_inverse_bytes(n)};
    size_t total = 0;
    for (size_t v : sizes) total += round_up(v);
    ScratchBlock *blk = acquire_scratch(h, total);
    if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
    char *p = static_cast<char *>(blk->ptr);
    void *part[9];
    for (int i = 0; i < 9; ++i)
    {
        part[i] = p;
        p += round_up(sizes[i]);
    }
    float *lu = static_cast<float *>(part[0]);
    int *ipiv = static_cast<int *>(part[1]);
    LargeStatus *status = static_cast<LargeStatus *>(part[2]);
    void *solve_scratch = part[3];
    int *flags = static_cast<int *>(part[4]);  // [0] bad pivot (unused: pivots are ours)
    LargeIr s = large_ir_carve(part[5], n, nrhs);
    RealBatch src{nullptr, const_cast<float *const *>(Aarray), n, lda, 0, 1};
    RealBatch fac{lu, nullptr, n, n, 0, 1};
    int hinfo = 0, running = 0;
    cudaError_t e = launch_copy_matrices(src, fac, n, st);
    if (e == cudaSuccess)
        e = launch_getrf_large(lu, n, n, n, ipiv, infoArray, status, mode, st, mode != 0 ? part[6] : nullptr);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hinfo, infoArray, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    int *perm = static_cast<int *>(part[7]);  // the pivots composed once for every solve
    float *dinv = static_cast<float *>(part[8]);  // the factors' diagonal blocks, inverted once
    auto solve = [&]() {
        return launch_getrs_large(lu, nullptr, n, n, nullptr, s.r32, nullptr, n, nrhs, solve_scratch, flags, nullptr, st,
                                  perm, dinv);
    };
    if (e == cudaSuccess && hinfo == 0)
    {
        e = launch_large_perm(ipiv, n, perm, flags, st);
        if (e == cudaSuccess) e = launch_large_diag_inverses(lu, n, n, dinv, st);
        if (e == cudaSuccess) e = launch_lir_init(s, Barray, ldb, n, nrhs, st);
        if (e == cudaSuccess) e = solve();
        if (e == cudaSuccess) e = launch_lir_update(s, n, nrhs, 1, st);
        if (e == cudaSuccess) e = launch_lir_residual(s, Aarray, lda, Barray, ldb, n, nrhs, tol, 1, st);
        for (int it = 0; it < maxIter && e == cudaSuccess; ++it)
        {
            e = cudaMemcpyAsync(&running, s.running, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess || !running) break;
            e = solve();
            if (e == cudaSuccess) e = launch_lir_update(s, n, nrhs, 0, st);
            if (e == cudaSuccess) e = launch_lir_residual(s, Aarray, lda, Barray, ldb, n, nrhs, tol, 0, st);
        }
    }
    if (e == cudaSuccess) e = launch_lir_finish(s, Xarray, ldx, n, nrhs, berrArray, iterArray, hinfo != 0, st);
    aclsolverStatus_t launched = launch_status(e);
    aclsolverStatus_t fin = finish_scratch(h, blk);
    return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
}

aclsolverStatus_t fail_args(Handle *h, int *info, int count, int arg)
{
    if (info && count > 0 && is_device_pointer(info))
    {
        if (launch_fill_info(info, -arg, count, h->stream) != cudaSuccess) cudaGetLastError();
    }
    return ACLSOLVER_STATUS_INVALID_VALUE;
}
}  // namespace

extern "C" aclsolverStatus_t aclsolverSgesvIrBatched(aclsolverHandle_t handle, aclsolverFactorPrecision_t precision,
                                                     int n, int nrhs, const float *const Aarray[], int lda,
                                                     const float *const Barray[], int ldb, float *const Xarray[],
                                                     int ldx, int maxIter, double tol, int *iterArray,
                                                     double *berrArray, int *infoArray, int batchSize)
{
    if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
    Handle *h = to_handle(handle);
    const bool used = n > 0 && nrhs > 0 && batchSize > 0;
    int arg = 0;
    if (precision != ACLSOLVER_FACTOR_FP32 && precision != ACLSOLVER_FACTOR_BF16 &&
        precision != ACLSOLVER_FACTOR_BF16X3)
        arg = 1;
    else if (n < 0 || n > LARGE_MAX_COLS)
        arg = 2;
    else if (nrhs < 0)
        arg = 3;
    else if (used && !is_device_pointer(Aarray))
        arg = 4;
    else if (lda < std::max(1, n))
        arg = 5;
    else if (used && !is_device_pointer(Barray))
        arg = 6;
    else if (ldb < std::max(1, n))
        arg = 7;
    else if (used && !is_device_pointer(Xarray))
        arg = 8;
    else if (ldx < std::max(1, n))
        arg = 9;
    else if (maxIter < 0)
        arg = 10;
    else if (!(tol >= 0.0))
        arg = 11;
    else if (iterArray && batchSize > 0 && !is_device_pointer(iterArray))
        arg = 12;
    else if (berrArray && batchSize > 0 && !is_device_pointer(berrArray))
        arg = 13;
    else if (batchSize > 0 && !is_device_pointer(infoArray))
        arg = 14;
    else if (batchSize < 0)
        arg = 15;
    if (arg) return fail_args(h, infoArray, batchSize < 0 ? 1 : batchSize, arg);
    if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
    cudaStream_t st = h->stream;
    if (!used)
    {
        cudaError_t e = launch_fill_info(infoArray, 0, batchSize, st);
        if (e == cudaSuccess && iterArray) e = launch_fill_info(iterArray, 0, batchSize, st);
        if (e == cudaSuccess && berrArray) e = cudaMemsetAsync(berrArray, 0, sizeof(double) * batchSize, st);
        return launch_status(e);
    }

    const int mode = precision == ACLSOLVER_FACTOR_FP32 ? 0 : (precision == ACLSOLVER_FACTOR_BF16 ? 1 : 3);
    if (n > BLOCKED_MAX_N)
    {
        // one system at a time over the whole GPU, at most 16 right-hand sides
        if (nrhs > LARGE_SOLVE_MAX_RHS) return ACLSOLVER_STATUS_NOT_SUPPORTED;
        for (int q = 0; q < batchSize; ++q)
        {
            aclsolverStatus_t r = gesv_ir_large(h, mode, n, nrhs, Aarray + q, lda, Barray + q, ldb, Xarray + q, ldx,
                                                maxIter, tol, iterArray ? iterArray + q : nullptr,
                                                berrArray ? berrArray + q : nullptr, infoArray + q);
            if (r != ACLSOLVER_STATUS_SUCCESS) return r;
        }
        return ACLSOLVER_STATUS_SUCCESS;
    }

    // Workspace: LU copies, pivots and the panels' row changes, two pointer tables, FP64 solutions, FP32 staging,
    // per-job berr and state, per-matrix iterations.
    const size_t jobs = (size_t)batchSize * nrhs;
    const size_t vec = (size_t)n * jobs;
    const int nblk = (n + 31) / 32;
    const size_t sizes[10] = {(size_t)n * n * batchSize * sizeof(float),
                             (size_t)n * batchSize * sizeof(int),
                             (size_t)batchSize * BLOCKED_PANELS * PANEL_LIST_SHORTS * sizeof(short),
                             (size_t)batchSize * sizeof(float *),
                             (size_t)batchSize * sizeof(float *),
                             vec * sizeof(double),
                             vec * sizeof(float),
                             jobs * sizeof(double),
                             2 * jobs * sizeof(int),
                             (size_t)batchSize * nblk * 2 * 32 * 32 * sizeof(float)};
    size_t total = 0;
    for (size_t v : sizes) total += round_up(v);
    ScratchBlock *blk = acquire_scratch(h, total);
    if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
    char *p = static_cast<char *>(blk->ptr);
    void *part[10];
    for (int i = 0; i < 10; ++i)
    {
        part[i] = p;
        p += round_up(sizes[i]);
    }
    float *lu = static_cast<float *>(part[0]);
    int *ipiv = static_cast<int *>(part[1]);
    short *lists = static_cast<short *>(part[2]);  // the panels' row changes
    float **lu_table = static_cast<float **>(part[3]);
    float **r_table = static_cast<float **>(part[4]);
    IrState s;
    s.x64 = static_cast<double *>(part[5]);
    s.r32 = static_cast<float *>(part[6]);
    s.berr = static_cast<double *>(part[7]);
    s.state = static_cast<int *>(part[8]);
    s.iters = s.state + jobs;
    float *dinv = static_cast<float *>(part[9]);  // inverses of the factors' diagonal blocks

    RealBatch src{nullptr, const_cast<float *const *>(Aarray), n, lda, 0, batchSize};
    RealBatch fac{nullptr, lu_table, n, n, 0, batchSize};
    RealBatch rhs{nullptr, r_table, n, n, 0, batchSize};
    auto solve = [&](const int *skip)
    {
        return n <= SMALL_N ? launch_getrs_small(fac, ipiv, rhs, nrhs, 0, nullptr, st)
                            : launch_getrs_blocked(fac, nullptr, nullptr, rhs, nrhs, nullptr, skip, st, dinv,
                                                   lists);
    };
    cudaError_t e = launch_strided_table(lu_table, lu, (int64_t)n * n, batchSize, st);
    if (e == cudaSuccess) e = launch_strided_table(r_table, s.r32, (int64_t)n * nrhs, batchSize, st);
    if (e == cudaSuccess)
    {
        if (n <= SMALL_N)
        {
            e = launch_copy_matrices(src, fac, n, st);
            if (e == cudaSuccess) e = launch_getrf_small(fac, n, ipiv, infoArray, st);
        }
        else
        {
            // the factorisation copies A into the workspace itself; its L columns keep their
            // block's row order and the solves apply the panels' row changes as they go
            e = launch_getrf_blocked(fac, ipiv, infoArray, mode, st, src.table, lda, nullptr, lists);
            if (e == cudaSuccess) e = launch_diag_inverses(fac, dinv, st);
        }
    }
    if (e == cudaSuccess) e = launch_ir_init(s, Barray, ldb, infoArray, n, nrhs, batchSize, st);
    if (e == cudaSuccess) e = solve(s.state);
    if (e == cudaSuccess) e = launch_ir_update(s, 1, n, nrhs, batchSize, st);
    for (int it = 0; it < maxIter && e == cudaSuccess; ++it)
    {
        e = launch_ir_residual(s, Aarray, lda, Barray, ldb, n, nrhs, batchSize, tol, st);
        if (e == cudaSuccess) e = solve(s.state);
        if (e == cudaSuccess) e = launch_ir_update(s, 0, n, nrhs, batchSize, st);
    }
    if (e == cudaSuccess) e = launch_ir_residual(s, Aarray, lda, Barray, ldb, n, nrhs, batchSize, tol, st);
    if (e == cudaSuccess) e = launch_ir_finish(s, Xarray, ldx, n, nrhs, batchSize, berrArray, iterArray, st);
    aclsolverStatus_t launched = launch_status(e);
    aclsolverStatus_t fin = finish_scratch(h, blk);
    return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
}

extern "C" aclsolverStatus_t aclsolverSgetrfBatchedMixed(aclsolverHandle_t handle, aclsolverFactorPrecision_t precision,
                                                         int n, float *const Aarray[], int lda, int *PivotArray,
                                                         int *infoArray, int batchSize)
{
    if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
    Handle *h = to_handle(handle);
    int arg = 0;
    if (precision != ACLSOLVER_FACTOR_FP32 && precision != ACLSOLVER_FACTOR_BF16 &&
        precision != ACLSOLVER_FACTOR_BF16X3)
        arg = 1;
    else if (n < 0 || n > BLOCKED_MAX_N)
        arg = 2;
    else if (n > 0 && batchSize > 0 && !Aarray)
        arg = 3;
    else if (lda < std::max(1, n))
        arg = 4;
    else if (batchSize > 0 && !infoArray)
        arg = 6;
    else if (batchSize < 0)
        arg = 7;
    if (arg) return fail_args(h, infoArray, batchSize < 0 ? 1 : batchSize, arg);
    if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
    if (n == 0) return launch_status(launch_fill_info(infoArray, 0, batchSize, h->stream));
    RealBatch a{nullptr, Aarray, n, lda, 0, batchSize};
    const int mode = precision == ACLSOLVER_FACTOR_FP32 ? 0 : (precision == ACLSOLVER_FACTOR_BF16 ? 1 : 3);
    if (n <= SMALL_N) return launch_status(launch_getrf_small(a, n, PivotArray, infoArray, h->stream));
    return launch_status(launch_getrf_blocked(a, PivotArray, infoArray, mode, h->stream));
}
