// api_complex_lu.cpp -- complex64 LU C entry points: Cgetrf(_bufferSize), Cgetri(_bufferSize),
// CgetriBatched, CmatinvBatched and the host-buffer Cgetrs.
//
// Argument ladders follow the reference host code (paths relative to the reference root):
//   Cgetrf / _bufferSize     src/cgetrf/cgetrf_host.cpp:22-82 (InvalidShape :25-31)
//   Cgetri / _bufferSize     src/cgetri/cgetri_host.cpp:21-115 (ValidateBuffers :31-76)
//   CgetriBatched            src/cgetri_batched/cgetri_batched_host.cpp:21-79
//   CmatinvBatched           src/cmatinv_batched/cmatinv_batched_host.cpp:21-74
//   Reject / CompleteGetri   src/utils/complex_solver_host.h:117-192 (info = -argument when
//                            the info buffer is usable; a pivot out of range, seen on the
//                            device, turns the synchronous status into INVALID_VALUE)
//   Cgetrs                   src/cgetrs/cgetrs_host.cpp:96-231 (CheckCgetrsArgs :96-116)
// A null handle returns HANDLE_IS_NULLPTR.
#include <stdio.h>

#include <algorithm>
#include <vector>

#include "handle.h"
#include "launch.h"
#include "launch_complex.h"

using namespace ops_solver;

namespace
{
constexpr int MAX_ORDER = 4096;          // complex_solver_host.h:30
constexpr int MAX_COLS = 8192;           // cgetrf_host.cpp:28
constexpr int MAX_BATCH = 1000000;       // complex_solver_host.h:31
constexpr int MAX_BATCH_MATINV = 10000000;  // complex_solver_host.h:34

bool overlap(const void *a, size_t abytes, const void *b, size_t bbytes)
{
    uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x <= y ? y - x < abytes : x - y < bbytes;
}

bool span_ok(const void *p, size_t bytes, size_t align)
{
    return p && reinterpret_cast<uintptr_t>(p) % align == 0 && is_device_pointer(p) && device_span(p, bytes);
}

int error_count(int batch, int limit) { return batch < 0 || batch > limit ? 1 : batch; }

// Reject: -argument into info[0..count) when that buffer is usable, INVALID_VALUE either way.
aclsolverStatus_t reject(Handle *h, int argument, int *info, int count)
{
    if (info && count > 0 && span_ok(info, (size_t)count * sizeof(int), alignof(int)))
        if (launch_fill_info(info, -argument, count, h->stream) != cudaSuccess)
        {
            cudaGetLastError();
            return ACLSOLVER_STATUS_EXECUTION_FAILED;
        }
    return ACLSOLVER_STATUS_INVALID_VALUE;
}

aclsolverStatus_t fill(Handle *h, int *info, int count, int value)
{
    return launch_status(launch_fill_info(info, value, count, h->stream));
}

// CompleteGetri: with pivots supplied, read the per-matrix info back and report a device
// pivot error through the status.
aclsolverStatus_t complete_getri(Handle *h, const int *pivots, const int *info, int count)
{
    if (cudaPeekAtLastError() != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    if (!pivots) return ACLSOLVER_STATUS_SUCCESS;
    int *host = static_cast<int *>(host_stage(h, (size_t)count * sizeof(int)));
    if (!host) return ACLSOLVER_STATUS_ALLOC_FAILED;
    cudaError_t e = cudaMemcpyAsync(host, info, (size_t)count * sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    cudaError_t s = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess || s != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    return std::find(host, host + count, -4) != host + count ? ACLSOLVER_STATUS_INVALID_VALUE
                                                             : ACLSOLVER_STATUS_SUCCESS;
}

struct Span
{
    uintptr_t begin, end;
    int role;  // 0 input matrix, 1 output matrix, otherwise the argument index of a view
};

// ValidateMatrices (complex_solver_host.h:254-418): both pointer tables read back, every
// slot a device span of its matrix, no output overlapping an input, another output or an
// extra view (pivots, info).  On failure *bad is the argument to report.
aclsolverStatus_t check_matrices(Handle *h, const void *a_table, const void *c_table, int n, int lda, int ldc,
                                 int batch, int in_arg, int out_arg, const void *const *extra, const size_t *extra_bytes,
                                 const int *extra_arg, int n_extra, int *bad)
{
    const size_t ptr_bytes = (size_t)batch * sizeof(uintptr_t);
    uint8_t *host = static_cast<uint8_t *>(host_stage(h, 2 * ptr_bytes));
    if (!host) return ACLSOLVER_STATUS_ALLOC_FAILED;
    cudaError_t e = cudaMemcpyAsync(host, a_table, ptr_bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host + ptr_bytes, c_table, ptr_bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    const uintptr_t *in = reinterpret_cast<const uintptr_t *>(host);
    const uintptr_t *out = reinterpret_cast<const uintptr_t *>(host + ptr_bytes);
    const size_t a_bytes = (size_t)lda * n * sizeof(float2), c_bytes = (size_t)ldc * n * sizeof(float2);
    std::vector<Span> ins, outs, spans;
    try
    {
        ins.reserve((size_t)batch);
        outs.reserve((size_t)batch);
        spans.resize((size_t)batch * 2);
    }
    catch (...)
    {
        return ACLSOLVER_STATUS_ALLOC_FAILED;
    }
    SpanCache in_cache, out_cache;
    for (int q = 0; q < batch; ++q)
    {
        const void *ib = reinterpret_cast<const void *>(in[q]);
        const void *ob = reinterpret_cast<const void *>(out[q]);
        if (!in_cache.ok(ib, a_bytes, alignof(float2)))
        {
            *bad = in_arg;
            return ACLSOLVER_STATUS_INVALID_VALUE;
        }
        if (!out_cache.ok(ob, c_bytes, alignof(float2)))
        {
            *bad = out_arg;
            return ACLSOLVER_STATUS_INVALID_VALUE;
        }
        for (int x = 0; x < n_extra; ++x)
            if (extra_bytes[x] &&
                (overlap(ib, a_bytes, extra[x], extra_bytes[x]) || overlap(ob, c_bytes, extra[x], extra_bytes[x])))
            {
                *bad = extra_arg[x];
                return ACLSOLVER_STATUS_INVALID_VALUE;
            }
        ins.push_back({in[q], in[q] + a_bytes, 0});
        outs.push_back({out[q], out[q] + c_bytes, 1});
    }
    for (int x = 0; x < n_extra; ++x)
        for (int y = x + 1; y < n_extra; ++y)
            if (extra_bytes[x] && extra_bytes[y] && overlap(extra[x], extra_bytes[x], extra[y], extra_bytes[y]))
            {
                *bad = extra_arg[y];
                return ACLSOLVER_STATUS_INVALID_VALUE;
            }
    // tables over a slab arrive in ascending order: sort only when they do not, then merge
    auto before = [](const Span &x, const Span &y) { return x.begin < y.begin || (x.begin == y.begin && x.role < y.role); };
    if (!std::is_sorted(ins.begin(), ins.end(), before)) std::sort(ins.begin(), ins.end(), before);
    if (!std::is_sorted(outs.begin(), outs.end(), before)) std::sort(outs.begin(), outs.end(), before);
    std::merge(ins.begin(), ins.end(), outs.begin(), outs.end(), spans.begin(), before);
    uintptr_t read_end = 0, write_end = 0;
    for (const Span &s : spans)
    {
        if (s.role == 0)
        {
            if (s.begin < write_end)
            {
                *bad = out_arg;
                return ACLSOLVER_STATUS_INVALID_VALUE;
            }
            read_end = std::max(read_end, s.end);
        }
        else
        {
            if (s.begin < read_end || s.begin < write_end)
            {
                *bad = out_arg;
                return ACLSOLVER_STATUS_INVALID_VALUE;
            }
            write_end = s.end;
        }
    }
    return ACLSOLVER_STATUS_SUCCESS;
}

int getrf_shape(int m, int n, int lda)
{
    if (m < 0 || m > MAX_ORDER) return 1;
    if (n < 0 || n > MAX_COLS) return 2;
    if (lda < std::max(1, m)) return 4;
    return 0;
}

// The inverse of `count` LU factors into C (tables or one strided buffer), with handle
// scratch for orders above the register-resident kernel.
aclsolverStatus_t run_getri(Handle *h, const float2 *a_single, const float2 *const *a_table, int lda,
                            const int *pivots, float2 *c_single, float2 *const *c_table, int ldc, int n, int count,
                            int *info)
{
    const size_t bytes = cgetri_scratch_bytes(n);
    ScratchBlock *blk = nullptr;
    if (bytes)
    {
        blk = acquire_scratch(h, bytes);
        if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
    }
    aclsolverStatus_t st = launch_status(launch_cgetri(a_single, a_table, lda, 0, pivots, c_single, c_table, ldc, 0,
                                                       n, count, info, blk ? blk->ptr : nullptr, h->stream));
    if (blk)
    {
        aclsolverStatus_t fin = finish_scratch(h, blk);
        if (st == ACLSOLVER_STATUS_SUCCESS) st = fin;
    }
    return st;
}
}  // namespace

extern "C"
{
    aclsolverStatus_t aclsolverCgetrf_bufferSize(aclsolverHandle_t handle, int m, int n, aclFloatComplex *A, int lda,
                                                 int *Lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (getrf_shape(m, n, lda)) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!Lwork) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (m > 0 && n > 0 && !span_ok(A, (size_t)lda * n * sizeof(float2), alignof(float2)))
            return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = 0;  // panels factor in shared memory: no caller workspace
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCgetrf(aclsolverHandle_t handle, int m, int n, aclFloatComplex *A, int lda,
                                      aclFloatComplex *Workspace, int *devIpiv, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        if (int bad = getrf_shape(m, n, lda)) return reject(h, bad, devInfo, 1);
        if (!span_ok(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (m > 0 && n > 0)
        {
            if (!span_ok(A, (size_t)lda * n * sizeof(float2), alignof(float2))) return reject(h, 3, devInfo, 1);
            if (devIpiv && !span_ok(devIpiv, (size_t)std::min(m, n) * sizeof(int), alignof(int)))
                return reject(h, 6, devInfo, 1);
            if (Workspace && !span_ok(Workspace, 0, alignof(float2))) return reject(h, 5, devInfo, 1);
        }
        aclsolverStatus_t st = fill(h, devInfo, 1, 0);
        if (st != ACLSOLVER_STATUS_SUCCESS || m == 0 || n == 0) return st;
        cudaError_t e = launch_cgetrf(reinterpret_cast<float2 *>(A), lda, m, n, devIpiv, devInfo, h->stream);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            return ACLSOLVER_STATUS_EXECUTION_FAILED;
        }
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCgetri_bufferSize(aclsolverHandle_t handle, int n, aclFloatComplex *A, int lda,
                                                 int *Lwork)
    {
        (void)A;  // the size follows from n alone; A may still be unallocated
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (n < 0 || n > MAX_ORDER || lda < std::max(1, n)) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!Lwork) return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = n * n;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverCgetri(aclsolverHandle_t handle, int n, aclFloatComplex *A, int lda, int *devIpiv,
                                      aclFloatComplex *Workspace, int Lwork, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        if (n < 0 || n > MAX_ORDER) return reject(h, 1, devInfo, 1);
        if (lda < std::max(1, n)) return reject(h, 3, devInfo, 1);
        if (Lwork < n * n) return reject(h, 6, devInfo, 1);
        if (!span_ok(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (n == 0) return fill(h, devInfo, 1, 0);
        const size_t a_bytes = (size_t)lda * n * sizeof(float2), p_bytes = (size_t)n * sizeof(int),
                     w_bytes = (size_t)n * n * sizeof(float2);
        if (!span_ok(A, a_bytes, alignof(float2))) return reject(h, 2, devInfo, 1);
        if (devIpiv && !span_ok(devIpiv, p_bytes, alignof(int))) return reject(h, 4, devInfo, 1);
        if (!span_ok(Workspace, w_bytes, alignof(float2))) return reject(h, 5, devInfo, 1);
        const struct
        {
            const void *p;
            size_t bytes;
            int arg;
        } views[4] = {{A, a_bytes, 2}, {devIpiv, devIpiv ? p_bytes : 0, 4}, {Workspace, w_bytes, 5},
                      {devInfo, sizeof(int), 7}};
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j)
                if (views[i].bytes && views[j].bytes && overlap(views[i].p, views[i].bytes, views[j].p, views[j].bytes))
                    return views[j].arg == 7 ? ACLSOLVER_STATUS_INVALID_VALUE : reject(h, views[j].arg, devInfo, 1);
        float2 *w = reinterpret_cast<float2 *>(Workspace);
        aclsolverStatus_t st =
            run_getri(h, reinterpret_cast<const float2 *>(A), nullptr, lda, devIpiv, w, nullptr, n, n, 1, devInfo);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        if (launch_ccopy_ok(w, n, reinterpret_cast<float2 *>(A), lda, devInfo, h->stream) != cudaSuccess)
        {
            cudaGetLastError();
            return ACLSOLVER_STATUS_EXECUTION_FAILED;
        }
        return complete_getri(h, devIpiv, devInfo, 1);
    }

    aclsolverStatus_t aclsolverCgetriBatched(aclsolverHandle_t handle, int n, const aclFloatComplex *const Aarray[],
                                             int lda, const int *PivotArray, aclFloatComplex *const Carray[], int ldc,
                                             int *infoArray, int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int bad = 0;
        if (n < 0 || n > MAX_ORDER)
            bad = 1;
        else if (lda < std::max(1, n))
            bad = 3;
        else if (ldc < std::max(1, n))
            bad = 6;
        else if (batchSize < 0 || batchSize > MAX_BATCH)
            bad = 8;
        if (bad) return reject(h, bad, infoArray, error_count(batchSize, MAX_BATCH));
        if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
        const size_t info_bytes = (size_t)batchSize * sizeof(int);
        if (!span_ok(infoArray, info_bytes, alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (n == 0) return fill(h, infoArray, batchSize, 0);
        const size_t table_bytes = (size_t)batchSize * sizeof(uintptr_t);
        if (!span_ok(Aarray, table_bytes, alignof(uintptr_t))) return reject(h, 2, infoArray, batchSize);
        if (!span_ok(Carray, table_bytes, alignof(uintptr_t))) return reject(h, 5, infoArray, batchSize);
        const size_t piv_bytes = PivotArray ? (size_t)n * batchSize * sizeof(int) : 0;
        if (PivotArray && !span_ok(PivotArray, piv_bytes, alignof(int))) return reject(h, 4, infoArray, batchSize);
        const void *extra[2] = {PivotArray, infoArray};
        const size_t extra_bytes[2] = {piv_bytes, info_bytes};
        const int extra_arg[2] = {4, 7};
        aclsolverStatus_t st =
            check_matrices(h, Aarray, Carray, n, lda, ldc, batchSize, 2, 5, extra, extra_bytes, extra_arg, 2, &bad);
        if (st == ACLSOLVER_STATUS_INVALID_VALUE) return bad == 7 ? st : reject(h, bad, infoArray, batchSize);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        st = run_getri(h, nullptr, reinterpret_cast<const float2 *const *>(Aarray), lda, PivotArray, nullptr,
                       reinterpret_cast<float2 *const *>(Carray), ldc, n, batchSize, infoArray);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return complete_getri(h, PivotArray, infoArray, batchSize);
    }

    aclsolverStatus_t aclsolverCmatinvBatched(aclsolverHandle_t handle, int n, const aclFloatComplex *const A[],
                                              int lda, aclFloatComplex *const Ainv[], int lda_inv, int *info,
                                              int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int bad = 0;
        if (n < 0 || n > 32)
            bad = 1;
        else if (lda < std::max(1, n))
            bad = 3;
        else if (lda_inv < std::max(1, n))
            bad = 5;
        else if (batchSize < 0 || batchSize > MAX_BATCH_MATINV)
            bad = 7;
        if (bad) return reject(h, bad, info, error_count(batchSize, MAX_BATCH_MATINV));
        if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
        const size_t info_bytes = (size_t)batchSize * sizeof(int);
        if (!span_ok(info, info_bytes, alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (n == 0) return fill(h, info, batchSize, 0);
        const size_t table_bytes = (size_t)batchSize * sizeof(uintptr_t);
        if (!span_ok(A, table_bytes, alignof(uintptr_t))) return reject(h, 2, info, batchSize);
        if (!span_ok(Ainv, table_bytes, alignof(uintptr_t))) return reject(h, 4, info, batchSize);
        const void *extra[1] = {info};
        const size_t extra_bytes[1] = {info_bytes};
        const int extra_arg[1] = {6};
        aclsolverStatus_t st =
            check_matrices(h, A, Ainv, n, lda, lda_inv, batchSize, 2, 4, extra, extra_bytes, extra_arg, 1, &bad);
        if (st == ACLSOLVER_STATUS_INVALID_VALUE) return bad == 6 ? st : reject(h, bad, info, batchSize);
        if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        return launch_status(launch_cmatinv(reinterpret_cast<const float2 *const *>(A),
                                            reinterpret_cast<float2 *const *>(Ainv), n, lda, lda_inv, info, batchSize,
                                            h->stream));
    }

    aclError aclsolverCgetrs(aclsolverHandle_t handle, const uint64_t trans, const int64_t n, const int64_t nrhs,
                             aclFloatComplex *A, const int64_t lda, int32_t *ipiv, aclFloatComplex *B,
                             const int64_t ldb, int32_t *info)
    {
        if (!(n > 0 && n <= 8192 && nrhs > 0 && nrhs <= 8192 && lda >= n && ldb >= nrhs && A && B && ipiv && info &&
              lda - n <= 8191 && ldb - nrhs <= 8191 && (nrhs <= 4096 || ldb - nrhs <= 4095)))
        {
            fprintf(stderr, "[aclsolver] aclsolverCgetrs invalid param\n");
            return ACL_ERROR_INVALID_PARAM;
        }
        if (trans > 2)
        {
            fprintf(stderr, "[aclsolver] aclsolverCgetrs invalid param: trans must be 0, 1 or 2\n");
            return ACL_ERROR_INVALID_PARAM;
        }
        for (int64_t k = 0; k < n; ++k)
            if (ipiv[k] < 1 || ipiv[k] > n)
            {
                *info = -4;
                return ACL_ERROR_INVALID_PARAM;
            }
        cudaStream_t stream = handle ? to_handle(handle)->stream : nullptr;
        // Row-major host A (lda) and B (ldb) -> device.  Viewed column-major the raw A is A^T,
        // which is the working matrix of trans 1 as it stands (conjugated in place for
        // trans 2); trans 0 converts it to column-major A.  B becomes column-major n x nrhs.
        const size_t a_raw = (size_t)n * lda * sizeof(float2), b_raw = (size_t)n * ldb * sizeof(float2);
        const size_t a_cm = trans == 0 ? (size_t)n * n * sizeof(float2) : 0;
        const size_t x_cm = (size_t)n * nrhs * sizeof(float2), p_bytes = (size_t)n * sizeof(int);
        char *base = nullptr;
        const size_t total = a_raw + b_raw + a_cm + x_cm + p_bytes + 5 * 256;
        if (cudaMallocAsync(reinterpret_cast<void **>(&base), total, stream) != cudaSuccess)
        {
            cudaGetLastError();
            return (aclError)cudaErrorMemoryAllocation;
        }
        char *start = base;
        auto carve = [&](size_t bytes)
        {
            char *p = base;
            base += (bytes + 255) & ~size_t(255);
            return p;
        };
        float2 *d_araw = reinterpret_cast<float2 *>(carve(a_raw));
        float2 *d_braw = reinterpret_cast<float2 *>(carve(b_raw));
        float2 *d_a = trans == 0 ? reinterpret_cast<float2 *>(carve(a_cm)) : d_araw;
        float2 *d_x = reinterpret_cast<float2 *>(carve(x_cm));
        int *d_p = reinterpret_cast<int *>(carve(p_bytes));
        const int ldm = trans == 0 ? (int)n : (int)lda;
        cudaError_t e = cudaMemcpyAsync(d_araw, A, a_raw, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_braw, B, b_raw, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_p, ipiv, p_bytes, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess && trans == 0) e = launch_ctranspose(d_araw, lda, d_a, n, (int)n, (int)n, false, stream);
        if (e == cudaSuccess && trans == 2) e = launch_cconj(d_araw, (int64_t)n * lda, stream);
        if (e == cudaSuccess) e = launch_ctranspose(d_braw, ldb, d_x, n, (int)n, (int)nrhs, false, stream);
        if (e == cudaSuccess) e = launch_cgetrs(d_a, ldm, d_p, d_x, (int)n, (int)n, (int)nrhs, (int)trans, stream);
        if (e == cudaSuccess) e = launch_ctranspose(d_x, n, d_braw, ldb, (int)nrhs, (int)n, false, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(B, d_braw, b_raw, cudaMemcpyDeviceToHost, stream);
        cudaError_t fe = cudaFreeAsync(start, stream);
        cudaError_t se = cudaStreamSynchronize(stream);
        if (e != cudaSuccess || fe != cudaSuccess || se != cudaSuccess)
        {
            cudaError_t err = e != cudaSuccess ? e : (fe != cudaSuccess ? fe : se);
            cudaGetLastError();
            return (aclError)err;
        }
        *info = 0;
        return ACL_SUCCESS;
    }
}
