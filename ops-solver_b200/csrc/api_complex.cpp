// api_complex.cpp -- complex64 Cholesky C entry points: Cpotrf(_bufferSize), Cpotrs,
// CpotrfBatched, CpotrsBatched and this build's multi-right-hand-side batched solve.
//
// Contracts follow the reference host code:
//   FactorArg / SolveArg           src/utils/cholesky/cholesky.h:24-66
//   Finish (info[0] pre-write)      src/cpotrf/arch35/cholesky_kernels.cpp:1585-1621
//   Cpotrf / RunInPlace             src/cpotrf/arch35/cpotrf.cpp:14-60
//   Cpotrs                          src/cpotrs/arch35/cpotrs.cpp:14-50
//   CpotrfBatched / CpotrsBatched   src/cpotrf_batched/arch35/cpotrf_batched.cpp:14-55,
//                                   src/cpotrs_batched/arch35/cpotrs_batched.cpp:14-61
// A null handle returns NOT_INITIALIZED (the complex family's convention); argument errors
// write -i to info[0] only and return INVALID_VALUE; info[0] is pre-written with 0 on the
// success path and the factor kernels then write every batch entry.
#include <stdio.h>

#include <vector>

#include "handle.h"
#include "launch.h"
#include "launch_complex.h"
#include "vbatched.h"

using namespace ops_solver;

namespace
{
constexpr int MAX_ORDER = 4096;
constexpr int MAX_RHS = 128;
constexpr int MAX_BATCH = 1000000;

bool valid_uplo(int u) { return u == 0 || u == 1; }

int factor_arg(int uplo, int n, const void *a, int lda, bool empty_batch)
{
    if (!valid_uplo(uplo)) return 1;
    if (n < 0 || n > MAX_ORDER) return 2;
    if (!a && n > 0 && !empty_batch) return 3;
    if (lda < (n > 0 ? n : 1)) return 4;
    return 0;
}

int solve_arg(int uplo, int n, int nrhs, const void *a, int lda, const void *b, int ldb, bool empty_batch)
{
    if (!valid_uplo(uplo)) return 1;
    if (n < 0 || n > MAX_ORDER) return 2;
    if (nrhs < 0 || nrhs > MAX_RHS) return 3;
    if (!a && n > 0 && nrhs > 0 && !empty_batch) return 4;
    if (lda < (n > 0 ? n : 1)) return 5;
    if (!b && n > 0 && nrhs > 0 && !empty_batch) return 6;
    if (ldb < (n > 0 ? n : 1)) return 7;
    return 0;
}

aclsolverStatus_t info_span(const int *info, int64_t count)
{
    if (reinterpret_cast<uintptr_t>(info) % alignof(int) != 0) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (!is_device_pointer(info)) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (!device_span(info, (size_t)count * sizeof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
    return ACLSOLVER_STATUS_SUCCESS;
}

// Orders above CPOTRF_PACKED_MAX: one matrix at a time over the whole GPU, the backup for
// the failure contract in handle scratch.  A batch's pointer table is read back first, so
// that call synchronises; a null slot sets its info to -3.
aclsolverStatus_t factor_large(Handle *h, float2 *single, float2 *const *table, int n, int lda, int upper, int count,
                               int *info)
{
    ScratchBlock *blk = acquire_scratch(h, cpotrf_large_scratch_bytes(n));
    if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
    cudaError_t e = cudaSuccess;
    if (!table)
        e = launch_cpotrf_large(single, lda, upper, n, info, blk->ptr, h->stream);
    else
    {
        std::vector<float2 *> ptrs((size_t)count);
        e = cudaMemcpyAsync(ptrs.data(), table, (size_t)count * sizeof(float2 *), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        for (int q = 0; q < count && e == cudaSuccess; ++q)
            e = ptrs[q] ? launch_cpotrf_large(ptrs[q], lda, upper, n, info + q, blk->ptr, h->stream)
                        : launch_fill_info(info + q, -3, 1, h->stream);
    }
    aclsolverStatus_t launched = launch_status(e);
    aclsolverStatus_t fin = finish_scratch(h, blk);
    return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
}

// Finish: pre-writes info[0] = -argument (0 when the arguments are valid).
aclsolverStatus_t finish(aclsolverHandle_t handle, int *info, int argument)
{
    if (!handle) return ACLSOLVER_STATUS_NOT_INITIALIZED;
    if (!info) return ACLSOLVER_STATUS_INVALID_VALUE;
    Handle *h = to_handle(handle);
    if (launch_fill_info(info, -argument, 1, h->stream) != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    return argument ? ACLSOLVER_STATUS_INVALID_VALUE : ACLSOLVER_STATUS_SUCCESS;
}

aclsolverStatus_t batched_solve(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                const aclsolverFloatComplex *const a[], int lda, aclsolverFloatComplex *b[], int ldb,
                                int *info, int batch, bool single_rhs)
{
    int arg = solve_arg(uplo, n, nrhs, a, lda, b, ldb, batch == 0);
    if (!arg && single_rhs && n > 0 && batch > 0 && nrhs != 1) arg = 3;
    if (!arg && !info) arg = 8;
    if (!arg && (batch < 0 || batch > MAX_BATCH)) arg = 9;
    if (info)
    {
        aclsolverStatus_t span = info_span(info, batch > 0 ? batch : 1);
        if (span != ACLSOLVER_STATUS_SUCCESS) return span;
    }
    aclsolverStatus_t st = finish(handle, info, arg);
    if (st != ACLSOLVER_STATUS_SUCCESS || n == 0 || batch == 0 || nrhs == 0) return st;
    Handle *h = to_handle(handle);
    return launch_status(launch_cpotrs(nullptr, reinterpret_cast<const float2 *const *>(a), nullptr,
                                       reinterpret_cast<float2 *const *>(b), n, lda, ldb, nrhs, uplo, batch, nullptr,
                                       h->stream));
}
}  // namespace

extern "C"
{
    aclsolverStatus_t aclsolverCpotrf_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                                 aclsolverFloatComplex *A, int lda, int *Lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_NOT_INITIALIZED;
        if (factor_arg(uplo, n, A, lda, false) || !Lwork) return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = 0;  // the factorisation runs in place
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCpotrf(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                      aclsolverFloatComplex *A, int lda, aclsolverFloatComplex *Workspace, int Lwork,
                                      int *devInfo)
    {
        int arg = factor_arg(uplo, n, A, lda, false);
        const int required = 0;
        const bool needs_work = Lwork > 0 || required > 0;
        if (!arg && !Workspace && needs_work) arg = 5;
        if (!arg && Lwork < required) arg = 6;
        if (!arg && !devInfo) arg = 7;
        if (devInfo)
        {
            aclsolverStatus_t span = info_span(devInfo, 1);
            if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        }
        aclsolverStatus_t st = finish(handle, devInfo, arg);
        if (st != ACLSOLVER_STATUS_SUCCESS || n == 0) return st;
        Handle *h = to_handle(handle);
        if (n > CPOTRF_PACKED_MAX) return factor_large(h, reinterpret_cast<float2 *>(A), nullptr, n, lda, uplo, 1, devInfo);
        return launch_status(launch_cpotrf(reinterpret_cast<float2 *>(A), nullptr, n, lda, uplo, 1, devInfo, h->stream));
    }

    aclsolverStatus_t aclsolverCpotri_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                                 aclsolverFloatComplex *A, int lda, int *Lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_NOT_INITIALIZED;
        if (factor_arg(uplo, n, A, lda, false) || !Lwork) return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = n * n;  // the identity the factor is solved against
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCpotri(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                      aclsolverFloatComplex *A, int lda, aclsolverFloatComplex *Workspace, int Lwork,
                                      int *devInfo)
    {
        int arg = factor_arg(uplo, n, A, lda, false);
        const int required = n * n;
        if (!arg && !Workspace && n > 0) arg = 5;
        if (!arg && Lwork < required) arg = 6;
        if (!arg && !devInfo) arg = 7;
        if (devInfo)
        {
            aclsolverStatus_t span = info_span(devInfo, 1);
            if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        }
        aclsolverStatus_t st = finish(handle, devInfo, arg);
        if (st != ACLSOLVER_STATUS_SUCCESS || n == 0) return st;
        Handle *h = to_handle(handle);
        float2 *a = reinterpret_cast<float2 *>(A);
        float2 *w = reinterpret_cast<float2 *>(Workspace);
        cudaError_t e = launch_cpotri_prepare(a, lda, n, w, devInfo, h->stream);
        if (e == cudaSuccess) e = launch_cpotrs(a, nullptr, w, nullptr, n, lda, n, n, uplo, 1, devInfo, h->stream);
        if (e == cudaSuccess) e = launch_cpotri_store(a, lda, uplo, n, w, devInfo, h->stream);
        return launch_status(e);
    }

    aclsolverStatus_t aclsolverCpotrs(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                      const aclsolverFloatComplex *A, int lda, aclsolverFloatComplex *B, int ldb,
                                      int *devInfo)
    {
        int arg = solve_arg(uplo, n, nrhs, A, lda, B, ldb, false);
        if (!arg && !devInfo) arg = 8;
        if (devInfo)
        {
            aclsolverStatus_t span = info_span(devInfo, 1);
            if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        }
        aclsolverStatus_t st = finish(handle, devInfo, arg);
        if (st != ACLSOLVER_STATUS_SUCCESS || n == 0 || nrhs == 0) return st;
        Handle *h = to_handle(handle);
        return launch_status(launch_cpotrs(reinterpret_cast<const float2 *>(A), nullptr, reinterpret_cast<float2 *>(B),
                                           nullptr, n, lda, ldb, nrhs, uplo, 1, nullptr, h->stream));
    }

    aclsolverStatus_t aclsolverCpotrfBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                             aclsolverFloatComplex *Aarray[], int lda, int *infoArray, int batchSize)
    {
        int arg = factor_arg(uplo, n, Aarray, lda, batchSize == 0);
        if (!arg && !infoArray) arg = 5;
        if (!arg && (batchSize < 0 || batchSize > MAX_BATCH)) arg = 6;
        if (infoArray)
        {
            aclsolverStatus_t span = info_span(infoArray, batchSize > 0 ? batchSize : 1);
            if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        }
        aclsolverStatus_t st = finish(handle, infoArray, arg);
        if (st != ACLSOLVER_STATUS_SUCCESS || batchSize == 0) return st;
        Handle *h = to_handle(handle);
        if (n == 0) return launch_status(launch_fill_info(infoArray, 0, batchSize, h->stream));
        if (n > CPOTRF_PACKED_MAX)
            return factor_large(h, nullptr, reinterpret_cast<float2 *const *>(Aarray), n, lda, uplo, batchSize,
                                infoArray);
        return launch_status(launch_cpotrf(nullptr, reinterpret_cast<float2 *const *>(Aarray), n, lda, uplo, batchSize,
                                           infoArray, h->stream));
    }

    aclsolverStatus_t aclsolverCpotrsBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                             const aclsolverFloatComplex *const Aarray[], int lda,
                                             aclsolverFloatComplex *Barray[], int ldb, int *info, int batchSize)
    {
        return batched_solve(handle, uplo, n, nrhs, Aarray, lda, Barray, ldb, info, batchSize, true);
    }

    aclsolverStatus_t aclsolverCpotrsBatchedMultiRhs(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                                     int nrhs, const aclsolverFloatComplex *const Aarray[], int lda,
                                                     aclsolverFloatComplex *Barray[], int ldb, int *info,
                                                     int batchSize)
    {
        return batched_solve(handle, uplo, n, nrhs, Aarray, lda, Barray, ldb, info, batchSize, false);
    }

    aclsolverStatus_t aclsolverCposvVbatchedPlanCreate(aclsolverHandle_t handle, aclsolverFillMode_t uplo,
                                                       const int *nArray, const int *ldaArray, const int *ldbArray,
                                                       int nrhs, int batchSize, int autotune,
                                                       aclsolverVbatchedPlan_t *plan)
    {
        if (!handle) return ACLSOLVER_STATUS_NOT_INITIALIZED;
        if (!plan || !valid_uplo(uplo) || nrhs < 0 || nrhs > MAX_RHS || batchSize < 0 || batchSize > MAX_BATCH ||
            (batchSize > 0 && (!nArray || !ldaArray || !ldbArray)) || (autotune != 0 && autotune != 1))
            return ACLSOLVER_STATUS_INVALID_VALUE;
        for (int q = 0; q < batchSize; ++q)
        {
            const int n = nArray[q];
            if (n < 0 || n > 160 || ldaArray[q] < (n > 0 ? n : 1) || ldbArray[q] < (n > 0 ? n : 1))
                return ACLSOLVER_STATUS_INVALID_VALUE;
        }
        VbPlan *p = nullptr;
        aclsolverStatus_t st =
            vb_plan_create(to_handle(handle), uplo, nArray, ldaArray, ldbArray, nrhs, batchSize, autotune, &p);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        *plan = reinterpret_cast<aclsolverVbatchedPlan_t>(p);
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCposvVbatched(aclsolverHandle_t handle, aclsolverVbatchedPlan_t plan,
                                             aclsolverFloatComplex *const Aarray[], aclsolverFloatComplex *const Barray[],
                                             int *infoArray)
    {
        if (!handle) return ACLSOLVER_STATUS_NOT_INITIALIZED;
        VbPlan *p = reinterpret_cast<VbPlan *>(plan);
        if (!p) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (p->count == 0) return ACLSOLVER_STATUS_SUCCESS;
        if (!Aarray || !infoArray || (p->nrhs > 0 && !Barray)) return ACLSOLVER_STATUS_INVALID_VALUE;
        aclsolverStatus_t span = info_span(infoArray, p->count);
        if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        return vb_plan_execute(p, reinterpret_cast<float2 *const *>(Aarray), reinterpret_cast<float2 *const *>(Barray),
                               infoArray, to_handle(handle)->stream);
    }

    aclsolverStatus_t aclsolverVbatchedPlanDestroy(aclsolverVbatchedPlan_t plan)
    {
        if (!plan) return ACLSOLVER_STATUS_INVALID_VALUE;
        vb_plan_destroy(reinterpret_cast<VbPlan *>(plan));
        return ACLSOLVER_STATUS_SUCCESS;
    }
}
