// api_cholesky.cpp -- real Cholesky C entry points (Spotrf, Spotrs, SpotrfBatched,
// SpotrsBatched and the workspace queries).
//
// Argument ladders, info conventions and empty-problem rules follow the reference host
// code src/cholesky/arch35/cholesky_host.cpp:
//   MatrixError :45-52 (1 uplo, 2 n in [0,4096], 3 null A when used, 4 lda < max(1,n))
//   Compute :226-250, SpotrfBatched :283-329, Spotrs :331-361, SpotrsBatched :363-396.
// Argument errors write -i through the info buffer (all batch entries for SpotrfBatched)
// and return INVALID_VALUE; numerical failures are reported in info with SUCCESS.
#include <algorithm>

#include <vector>

#include "handle.h"
#include "launch.h"

using namespace ops_solver;

namespace
{
bool valid_uplo(int u) { return u == 0 || u == 1; }

int matrix_error(int u, int n, const void *a, int ld, bool used)
{
    if (!valid_uplo(u)) return 1;
    if (n < 0 || n > 4096) return 2;
    if (used && !a) return 3;
    if (ld < std::max(1, n)) return 4;
    return 0;
}

aclsolverStatus_t arg_error(Handle *h, int *info, int index, int64_t count = 1)
{
    if (info && count > 0)
    {
        if (launch_fill_info(info, -index, count, h->stream) != cudaSuccess)
        {
            cudaGetLastError();
            return ACLSOLVER_STATUS_EXECUTION_FAILED;
        }
    }
    return ACLSOLVER_STATUS_INVALID_VALUE;
}

// Device-span check of an info array (the reference's DeviceSpan, complex_solver_host.h:94-117).
aclsolverStatus_t info_span(const int *info, int64_t count)
{
    if (count <= 0) return ACLSOLVER_STATUS_SUCCESS;
    if (reinterpret_cast<uintptr_t>(info) % alignof(int) != 0) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (!is_device_pointer(info)) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (!device_span(info, (size_t)count * sizeof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
    return ACLSOLVER_STATUS_SUCCESS;
}

// This build's factorisation needs no caller workspace at any order; the inverse needs the
// n x n right-hand side the identity is solved in.
int required_workspace(int n, bool inverse)
{
    return inverse ? n * n : 0;
}

// The single-matrix solve's dispatch (aclsolverSpotrs), info-gated: the kernels skip their
// work when info[0] != 0.
cudaError_t single_solve(const RealBatch &a, const RealBatch &b, int nrhs, int uplo, int *info, cudaStream_t s)
{
    if (a.n <= 8) return launch_potrs_small(a, b, nrhs, uplo, info, s);
    return launch_potrs_generic(a, b, nrhs, uplo, a.n <= 128 ? 1 : 0, info, s);
}

// Factor dispatch by order: up to 32 the register kernels, up to 256 a block per matrix
// with the packed triangle in shared memory, above that one matrix at a time over the whole
// GPU (a backup of the triangle in handle scratch; a batch's pointer table is read back, so
// that case synchronises with the host).
aclsolverStatus_t factor(Handle *h, const RealBatch &a, int upper, int *info)
{
    cudaStream_t s = h->stream;
    if (a.n <= 32) return launch_status(launch_potrf_small(a, upper, info, s));
    if (a.n <= POTRF_PACKED_MAX) return launch_status(launch_potrf_packed(a, upper, info, s));
    ScratchBlock *blk = acquire_scratch(h, potrf_large_scratch_bytes(a.n));
    if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
    cudaError_t e = cudaSuccess;
    if (!a.table)
        e = launch_potrf_large(a.single, a.ld, upper, a.n, info, blk->ptr, s);
    else
    {
        std::vector<float *> ptrs((size_t)a.count);
        e = cudaMemcpyAsync(ptrs.data(), a.table + a.first, (size_t)a.count * sizeof(float *), cudaMemcpyDeviceToHost,
                            s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        for (int64_t q = 0; q < a.count && e == cudaSuccess; ++q)
            e = ptrs[q] ? launch_potrf_large(ptrs[q], a.ld, upper, a.n, info + q, blk->ptr, s)
                        : launch_fill_info(info + q, -3, 1, s);
    }
    aclsolverStatus_t launched = launch_status(e);
    aclsolverStatus_t fin = finish_scratch(h, blk);
    return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
}

aclsolverStatus_t query(aclsolverHandle_t handle, int u, int n, float *a, int ld, int *lw, bool inverse)
{
    if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
    if (matrix_error(u, n, a, ld, false) || !lw) return ACLSOLVER_STATUS_INVALID_VALUE;
    *lw = required_workspace(n, inverse);
    return ACLSOLVER_STATUS_SUCCESS;
}
}  // namespace

extern "C"
{
    aclsolverStatus_t aclsolverSpotrf_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A,
                                                 int lda, int *Lwork)
    {
        return query(handle, uplo, n, A, lda, Lwork, false);
    }

    aclsolverStatus_t aclsolverSpotri_bufferSize(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A,
                                                 int lda, int *Lwork)
    {
        return query(handle, uplo, n, A, lda, Lwork, true);
    }

    aclsolverStatus_t aclsolverSpotrf(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A, int lda,
                                      float *Workspace, int Lwork, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const int need = required_workspace(n, false);
        int error = matrix_error(uplo, n, A, lda, n > 0);
        if (!error && n > 0 && n <= 4096 && (need || Lwork > 0) && !Workspace) error = 5;
        if (!error && (Lwork < 0 || Lwork < need)) error = 6;
        if (!error && !devInfo) error = 7;
        if (error) return arg_error(h, devInfo, error);
        if (!n) return launch_status(launch_fill_info(devInfo, 0, 1, h->stream));
        RealBatch a{A, nullptr, n, lda, 0, 1};
        return factor(h, a, uplo, devInfo);
    }

    aclsolverStatus_t aclsolverSpotri(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, float *A, int lda,
                                      float *Workspace, int Lwork, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const int need = required_workspace(n, true);
        int error = matrix_error(uplo, n, A, lda, n > 0);
        if (!error && n > 0 && !Workspace) error = 5;
        if (!error && (Lwork < 0 || Lwork < need)) error = 6;
        if (!error && !devInfo) error = 7;
        if (error) return arg_error(h, devInfo, error);
        if (!n) return launch_status(launch_fill_info(devInfo, 0, 1, h->stream));
        RealBatch a{A, nullptr, n, lda, 0, 1};
        RealBatch w{Workspace, nullptr, n, n, 0, 1};
        cudaError_t e = launch_potri_prepare(A, lda, n, Workspace, devInfo, h->stream);
        if (e == cudaSuccess) e = single_solve(a, w, n, uplo, devInfo, h->stream);
        if (e == cudaSuccess) e = launch_potri_store(A, lda, uplo, n, Workspace, devInfo, h->stream);
        return launch_status(e);
    }

    aclsolverStatus_t aclsolverSpotrfBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n,
                                             float *Aarray[], int lda, int *infoArray, int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const int count = batchSize;
        int error = matrix_error(uplo, n, Aarray, lda, n > 0 && count > 0);
        if (!error && count > 0 && !infoArray) error = 5;
        if (!error && count < 0) error = 6;
        if (infoArray && count > 0)
        {
            aclsolverStatus_t span = info_span(infoArray, count);
            if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        }
        if (error) return arg_error(h, infoArray, error, count > 0 ? count : (count < 0 ? 1 : 0));
        if (!n || !count)
        {
            if (count) return launch_status(launch_fill_info(infoArray, 0, count, h->stream));
            return ACLSOLVER_STATUS_SUCCESS;
        }
        RealBatch a{nullptr, Aarray, n, lda, 0, count};
        return factor(h, a, uplo, infoArray);
    }

    aclsolverStatus_t aclsolverSpotrs(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                      const float *A, int lda, float *B, int ldb, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int error = !valid_uplo(uplo)            ? 1
                    : n < 0 || n > 4096          ? 2
                    : nrhs < 0 || nrhs > 128     ? 3
                    : n && nrhs && !A            ? 4
                    : lda < std::max(1, n)       ? 5
                    : n && nrhs && !B            ? 6
                    : ldb < std::max(1, n)       ? 7
                    : !devInfo                   ? 8
                                                 : 0;
        if (error) return arg_error(h, devInfo, error);
        cudaError_t e = launch_fill_info(devInfo, 0, 1, h->stream);
        if (e == cudaSuccess && n && nrhs)
        {
            RealBatch a{const_cast<float *>(A), nullptr, n, lda, 0, 1};
            RealBatch b{B, nullptr, n, ldb, 0, 1};
            e = single_solve(a, b, nrhs, uplo, devInfo, h->stream);
        }
        return launch_status(e);
    }

    aclsolverStatus_t aclsolverSpotrsBatched(aclsolverHandle_t handle, aclsolverFillMode_t uplo, int n, int nrhs,
                                             float *Aarray[], int lda, float *Barray[], int ldb, int *info,
                                             int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const int count = batchSize;
        const bool used = n > 0 && count > 0;
        int error = !valid_uplo(uplo)                  ? 1
                    : n < 0 || n > 4096                ? 2
                    : nrhs < 0 || (used && nrhs != 1)  ? 3
                    : used && !Aarray                  ? 4
                    : lda < std::max(1, n)             ? 5
                    : used && !Barray                  ? 6
                    : ldb < std::max(1, n)             ? 7
                    : !info                            ? 8
                    : count < 0                        ? 9
                                                       : 0;
        if (error) return arg_error(h, info, error);
        if (!used) return launch_status(launch_fill_info(info, 0, 1, h->stream));
        aclsolverStatus_t span = info_span(info, count);
        if (span != ACLSOLVER_STATUS_SUCCESS) return span;
        int *flags = device_flags(h);
        if (!flags) return ACLSOLVER_STATUS_ALLOC_FAILED;
        cudaError_t e = launch_solve_slot_check(info, Aarray, Barray, count, flags + SLOT_CHECK_FLAGS, h->stream);
        if (e == cudaSuccess)
        {
            RealBatch a{nullptr, Aarray, n, lda, 0, count};
            RealBatch b{nullptr, Barray, n, ldb, 0, count};
            if (n <= 32)
                e = launch_potrs_small(a, b, 1, uplo, info, h->stream);
            else
                e = launch_potrs_generic(a, b, 1, uplo, n <= 128 ? 1 : 0, info, h->stream);
        }
        return launch_status(e);
    }
}
