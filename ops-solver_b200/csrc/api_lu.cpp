// api_lu.cpp -- real LU C entry points: Sgetrf, Sgetri, SgetriBatched, SmatinvBatched,
// the host-buffer Sgetrs, and this build's SgetrfBatched / SgetrsBatched.
//
// Argument ladders and validation follow the reference host code:
//   Sgetrf          src/sgetrf/sgetrf_host.cpp:24-124   (FactorArgument :46-73)
//   Sgetri          src/sgetri/sgetri_host.cpp:14-118   (InverseArgument :31-58)
//   SgetriBatched   src/sgetri_batched/sgetri_batched_host.cpp:41-113
//   SmatinvBatched  src/smatinv_batched/smatinv_batched_host.cpp:11-61
//   shared checks   src/utils/real_lu_common.h (BatchedArgument :20-60, CheckSingle :61-89,
//                   CheckFinite :90-132, CheckPivots :134-182, ArrayValidation :196-421)
//   Sgetrs          src/sgetrs/sgetrs_host.cpp:131-195
// The device-data checks (finite values, pivot ranges, pointer tables) copy metadata to
// the host and synchronise the handle stream, exactly where the reference does; the
// SgetrfBatched / SgetrsBatched additions never synchronise.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "handle.h"
#include "launch.h"

using namespace ops_solver;

namespace
{
constexpr int MAX_BATCH = 10000000;  // real_lu_common.h:18
constexpr int SMALL_N = 64;          // largest order of the register-resident kernels

bool device_fits(const void *p, size_t bytes, size_t align)
{
    return p && reinterpret_cast<uintptr_t>(p) % align == 0 && is_device_pointer(p) && device_span(p, bytes);
}

bool overlap(const void *a, size_t abytes, const void *b, size_t bbytes)
{
    uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x <= y ? y - x < abytes : x - y < bbytes;
}

// Writes -argument to info[0..count) when info is a usable device buffer; INVALID_VALUE.
aclsolverStatus_t invalid(Handle *h, int *info, int64_t count, int argument)
{
    if (count > 0 && device_fits(info, (size_t)count * sizeof(int), alignof(int)))
    {
        if (launch_fill_info(info, -argument, count, h->stream) != cudaSuccess) cudaGetLastError();
    }
    return ACLSOLVER_STATUS_INVALID_VALUE;
}

aclsolverStatus_t empty_info(Handle *h, int *info, int64_t count)
{
    if (!device_fits(info, (size_t)count * sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
    return launch_status(launch_fill_info(info, 0, count, h->stream));
}

// Copies `bytes` of device metadata to pinned host staging and waits for the stream.
aclsolverStatus_t fetch(Handle *h, void *host, const void *dev, size_t bytes)
{
    if (bytes == 0) return ACLSOLVER_STATUS_SUCCESS;
    if (cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    {
        cudaGetLastError();
        cudaStreamSynchronize(h->stream);
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    return ACLSOLVER_STATUS_SUCCESS;
}

aclsolverStatus_t sync(Handle *h)
{
    if (cudaStreamSynchronize(h->stream) != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    return ACLSOLVER_STATUS_SUCCESS;
}

// CheckFinite: scan, read the flag back, reject non-finite input with info = -argument.
aclsolverStatus_t check_finite(Handle *h, const RealBatch &a, int m, int *info, int64_t info_count, int argument)
{
    int *flag = device_flags(h);
    int *host = static_cast<int *>(host_stage(h, 64));
    if (!flag || !host) return ACLSOLVER_STATUS_ALLOC_FAILED;
    if (cudaMemsetAsync(flag, 0, sizeof(int), h->stream) != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    if (launch_finite_scan(a, m, flag, h->stream) != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    aclsolverStatus_t st = fetch(h, host, flag, sizeof(int));
    if (st == ACLSOLVER_STATUS_SUCCESS) st = sync(h);
    if (st != ACLSOLVER_STATUS_SUCCESS) return st;
    if (host[0] != 0) return invalid(h, info, info_count, argument);
    return ACLSOLVER_STATUS_SUCCESS;
}

// CheckPivots: every pivot k (1-based) must lie in [k+1, n].
aclsolverStatus_t check_pivots(Handle *h, const int *piv, int n, int *info, int batch, bool *identity)
{
    *identity = true;
    if (!piv) return ACLSOLVER_STATUS_SUCCESS;
    size_t bytes = (size_t)n * batch * sizeof(int);
    if (!device_fits(piv, bytes, alignof(int))) return invalid(h, info, batch, 4);
    int *host = static_cast<int *>(host_stage(h, bytes));
    if (!host) return ACLSOLVER_STATUS_ALLOC_FAILED;
    aclsolverStatus_t st = fetch(h, host, piv, bytes);
    if (st == ACLSOLVER_STATUS_SUCCESS) st = sync(h);
    if (st != ACLSOLVER_STATUS_SUCCESS) return st;
    for (int64_t b = 0; b < batch; ++b)
        for (int k = 0; k < n; ++k)
        {
            int v = host[b * n + k];
            if (v < k + 1 || v > n) return invalid(h, info, batch, 4);
            if (v != k + 1) *identity = false;
        }
    return ACLSOLVER_STATUS_SUCCESS;
}

struct Layout
{
    bool contiguous = true;
    bool identity = true;
    const float *input = nullptr;
    float *output = nullptr;
};

struct Span
{
    uintptr_t begin, end;
    int role;  // 0 read-only input, 1 output, otherwise the argument index of metadata
};

// ArrayValidation (real_lu_common.h:196-421): pointer tables, per-slot capacity, pivot
// ranges, and no output overlapping any other buffer (inputs may alias each other).
aclsolverStatus_t check_arrays(Handle *h, int n, const float *const *a, int lda, const int *piv, float *const *c,
                               int ldc, int *info, int batch, bool factor, Layout &layout)
{
    const int out_arg = factor ? 4 : 5;
    const size_t ptr_bytes = (size_t)batch * sizeof(uintptr_t);
    const size_t piv_bytes = piv ? (size_t)batch * n * sizeof(int) : 0;
    const size_t a_bytes = (size_t)lda * n * sizeof(float);
    const size_t c_bytes = (size_t)ldc * n * sizeof(float);
    const size_t info_bytes = (size_t)batch * sizeof(int);
    if (!device_fits(a, ptr_bytes, alignof(uintptr_t))) return invalid(h, info, batch, 2);
    if (!device_fits(c, ptr_bytes, alignof(uintptr_t))) return invalid(h, info, batch, out_arg);
    if (!device_fits(info, info_bytes, alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (piv && !device_fits(piv, piv_bytes, alignof(int))) return invalid(h, info, batch, 4);
    struct View
    {
        const void *p;
        size_t bytes;
        int arg;
    } views[4] = {{a, ptr_bytes, 2}, {c, ptr_bytes, out_arg}, {piv, piv_bytes, 4}, {info, info_bytes, factor ? 6 : 7}};
    for (int i = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j)
            if (views[i].bytes && views[j].bytes && overlap(views[i].p, views[i].bytes, views[j].p, views[j].bytes))
                return j == 3 ? ACLSOLVER_STATUS_INVALID_VALUE : invalid(h, info, batch, views[j].arg);

    uint8_t *host = static_cast<uint8_t *>(host_stage(h, 2 * ptr_bytes + piv_bytes));
    if (!host) return ACLSOLVER_STATUS_ALLOC_FAILED;
    aclsolverStatus_t st = fetch(h, host, a, ptr_bytes);
    if (st == ACLSOLVER_STATUS_SUCCESS) st = fetch(h, host + ptr_bytes, c, ptr_bytes);
    if (st == ACLSOLVER_STATUS_SUCCESS && piv) st = fetch(h, host + 2 * ptr_bytes, piv, piv_bytes);
    if (st == ACLSOLVER_STATUS_SUCCESS) st = sync(h);
    if (st != ACLSOLVER_STATUS_SUCCESS) return st;
    const uintptr_t *in = reinterpret_cast<const uintptr_t *>(host);
    const uintptr_t *out = reinterpret_cast<const uintptr_t *>(host + ptr_bytes);
    const int *pv = reinterpret_cast<const int *>(host + 2 * ptr_bytes);
    layout.input = reinterpret_cast<const float *>(in[0]);
    layout.output = reinterpret_cast<float *>(out[0]);
    std::vector<Span> spans;
    try
    {
        spans.reserve((size_t)batch * 2 + 4);
    }
    catch (...)
    {
        return ACLSOLVER_STATUS_ALLOC_FAILED;
    }
    SpanCache in_cache, out_cache;
    for (int b = 0; b < batch; ++b)
    {
        if (in[b] != in[0] + (size_t)b * a_bytes || out[b] != out[0] + (size_t)b * c_bytes) layout.contiguous = false;
        const void *ib = reinterpret_cast<const void *>(in[b]);
        const void *ob = reinterpret_cast<const void *>(out[b]);
        if (!in_cache.ok(ib, a_bytes, alignof(float))) return invalid(h, info, batch, 2);
        if (!out_cache.ok(ob, c_bytes, alignof(float))) return invalid(h, info, batch, out_arg);
        if (overlap(ib, a_bytes, info, info_bytes) || overlap(ob, c_bytes, info, info_bytes))
            return ACLSOLVER_STATUS_INVALID_VALUE;
        for (int i = 0; i < 3; ++i)
            if (views[i].bytes && (overlap(ib, a_bytes, views[i].p, views[i].bytes) ||
                                   overlap(ob, c_bytes, views[i].p, views[i].bytes)))
                return invalid(h, info, batch, views[i].arg);
        spans.push_back({in[b], in[b] + a_bytes, 0});
        spans.push_back({out[b], out[b] + c_bytes, 1});
        if (piv)
            for (int k = 0; k < n; ++k)
            {
                int v = pv[(size_t)b * n + k];
                if (v < k + 1 || v > n) return invalid(h, info, batch, 4);
                if (v != k + 1) layout.identity = false;
            }
    }
    for (int i = 0; i < 4; ++i)
        if (views[i].bytes && (i != 2 || piv))
            spans.push_back({reinterpret_cast<uintptr_t>(views[i].p),
                             reinterpret_cast<uintptr_t>(views[i].p) + views[i].bytes, views[i].arg});
    std::sort(spans.begin(), spans.end(), [](const Span &x, const Span &y)
              { return x.begin < y.begin || (x.begin == y.begin && x.role < y.role); });
    uintptr_t read_end = 0, write_end = 0;
    int previous = out_arg;
    for (const Span &s : spans)
    {
        if (s.role == 0)
        {
            if (s.begin < write_end) return invalid(h, info, batch, previous);
            read_end = std::max(read_end, s.end);
        }
        else
        {
            if (s.begin < read_end || s.begin < write_end) return invalid(h, info, batch, s.role == 1 ? out_arg : s.role);
            write_end = s.end;
            previous = s.role == 1 ? out_arg : s.role;
        }
    }
    return ACLSOLVER_STATUS_SUCCESS;
}

// The small and batched-blocked factorisations run in place (a token buffer keeps the
// reference contract); the whole-GPU path above them keeps its per-panel pivot lists and
// zero-pivot bits there.
bool large_path(int m, int n) { return !(m <= SMALL_N && n <= SMALL_N) && !(m == n && n <= BLOCKED_MAX_N) && m >= n; }

int factor_workspace(int m, int n)
{
    return large_path(m, n) ? (int)((sizeof(LargeStatus) + sizeof(float) - 1) / sizeof(float)) : 8;
}

int inverse_workspace(int n)
{
    int64_t size = (int64_t)n * n;
    return size > 0x7fffffff ? -1 : (int)size;
}

int batched_argument(int n, const void *a, int lda, const void *piv, const void *c, int ldc, int *info, int batch,
                     bool factor)
{
    if (n < 0 || n > (factor ? 32 : 4096)) return 1;
    if (n > 0 && batch > 0 && !is_device_pointer(a)) return 2;
    if (lda < std::max(1, n)) return 3;
    if (!factor && piv != nullptr && !is_device_pointer(piv)) return 4;
    if (n > 0 && batch > 0 && !is_device_pointer(c)) return factor ? 4 : 5;
    if (ldc < std::max(1, n)) return factor ? 5 : 6;
    if (batch > 0 && !is_device_pointer(info)) return factor ? 6 : 7;
    if (batch < 0) return factor ? 7 : 8;
    return 0;
}
}  // namespace

extern "C"
{
    aclsolverStatus_t aclsolverSgetrf_bufferSize(aclsolverHandle_t handle, int m, int n, float *A, int lda, int *Lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (m < 0 || m > 8192 || n < 0 || lda < std::max(1, m) || !Lwork || is_device_pointer(Lwork) ||
            (A && !is_device_pointer(A)))
            return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = m == 0 || n == 0 ? 0 : factor_workspace(m, n);
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSgetrf(aclsolverHandle_t handle, int m, int n, float *A, int lda, float *Workspace,
                                      int *devIpiv, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int arg = 0;
        if (m < 0 || m > 8192)
            arg = 1;
        else if (n < 0 || (int64_t)((m + 7) / 8 * 8) * n > 0x7fffffff)
            arg = 2;
        else if (m > 0 && n > 0 && !is_device_pointer(A))
            arg = 3;
        else if (lda < std::max(1, m))
            arg = 4;
        else if (m > 0 && n > 0 && !is_device_pointer(Workspace))
            arg = 5;
        else if (devIpiv && !is_device_pointer(devIpiv))
            arg = 6;
        else if (!is_device_pointer(devInfo))
            arg = 7;
        if (arg) return invalid(h, devInfo, 1, arg);
        if (m == 0 || n == 0) return empty_info(h, devInfo, 1);
        // CheckSingle: capacity and overlap of A, pivots, workspace and info.
        if (!device_fits(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        const size_t a_bytes = (size_t)lda * n * sizeof(float);
        const size_t w_bytes = (size_t)factor_workspace(m, n) * sizeof(float);
        const size_t p_bytes = (size_t)std::min(m, n) * sizeof(int);
        if (!device_fits(A, a_bytes, alignof(float))) return invalid(h, devInfo, 1, 3);
        if (!device_fits(Workspace, w_bytes, alignof(float))) return invalid(h, devInfo, 1, 5);
        if (devIpiv && !device_fits(devIpiv, p_bytes, alignof(int))) return invalid(h, devInfo, 1, 6);
        struct
        {
            const void *p;
            size_t b;
            int arg;
        } v[4] = {{A, a_bytes, 3}, {Workspace, w_bytes, 5}, {devIpiv, devIpiv ? p_bytes : 0, 6}, {devInfo, 4, 7}};
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j)
                if (v[i].b && v[j].b && overlap(v[i].p, v[i].b, v[j].p, v[j].b))
                    return j == 3 ? ACLSOLVER_STATUS_INVALID_VALUE : invalid(h, devInfo, 1, v[j].arg);
        RealBatch a{A, nullptr, n, lda, 0, 1};
        if (h->device_checks)
        {
            aclsolverStatus_t st = check_finite(h, a, m, devInfo, 1, 3);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        }
        if (m <= SMALL_N && n <= SMALL_N) return launch_status(launch_getrf_small(a, m, devIpiv, devInfo, h->stream));
        if (m == n && n <= BLOCKED_MAX_N) return launch_status(launch_getrf_blocked(a, devIpiv, devInfo, 0, h->stream));
        if (large_path(m, n))
        {
            if (reinterpret_cast<uintptr_t>(Workspace) % alignof(LargeStatus)) return invalid(h, devInfo, 1, 5);
            return launch_status(launch_getrf_large(A, m, n, lda, devIpiv, devInfo,
                                                    reinterpret_cast<LargeStatus *>(Workspace), 0, h->stream));
        }
        return ACLSOLVER_STATUS_NOT_SUPPORTED;
    }

    aclsolverStatus_t aclsolverSgetri_bufferSize(aclsolverHandle_t handle, int n, float *A, int lda, int *Lwork)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (n < 0 || n > 4096 || lda < std::max(1, n) || !Lwork || is_device_pointer(Lwork) ||
            (A && !is_device_pointer(A)))
            return ACLSOLVER_STATUS_INVALID_VALUE;
        *Lwork = inverse_workspace(n);
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSgetri(aclsolverHandle_t handle, int n, float *A, int lda, int *devIpiv,
                                      float *Workspace, int Lwork, int *devInfo)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int arg = 0;
        if (n < 0 || n > 4096)
            arg = 1;
        else if (n > 0 && !is_device_pointer(A))
            arg = 2;
        else if (lda < std::max(1, n))
            arg = 3;
        else if (devIpiv && !is_device_pointer(devIpiv))
            arg = 4;
        else if (n > 0 && (!is_device_pointer(Workspace) ||
                           overlap(A, (size_t)lda * n * sizeof(float), Workspace, (size_t)n * n * sizeof(float))))
            arg = 5;
        else if (Lwork < inverse_workspace(n))
            arg = 6;
        else if (!is_device_pointer(devInfo))
            arg = 7;
        if (arg) return invalid(h, devInfo, 1, arg);
        if (n == 0) return empty_info(h, devInfo, 1);
        if (!device_fits(devInfo, sizeof(int), alignof(int))) return ACLSOLVER_STATUS_INVALID_VALUE;
        if (!device_fits(A, (size_t)lda * n * sizeof(float), alignof(float))) return invalid(h, devInfo, 1, 2);
        bool identity = devIpiv == nullptr;
        RealBatch a{A, nullptr, n, lda, 0, 1};
        if (h->device_checks)
        {
            aclsolverStatus_t st = check_pivots(h, devIpiv, n, devInfo, 1, &identity);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
            st = check_finite(h, a, n, devInfo, 1, 2);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        }
        if (n > SMALL_N)
        {
            // above the register-resident orders: the factors copied to the workspace, A set to
            // the identity and solved in place by the blocked solve (the batched entry's path)
            ScratchBlock *blk = acquire_scratch(h, getri_blocked_scratch_bytes(n, 1));
            if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
            RealBatch w{Workspace, nullptr, n, n, 0, 1};
            cudaError_t e = launch_copy_matrices(a, w, n, h->stream);
            if (e == cudaSuccess)
                e = launch_getri_blocked(w, identity ? nullptr : devIpiv, a, devInfo, blk->ptr, h->stream);
            aclsolverStatus_t launched = launch_status(e);
            aclsolverStatus_t fin = finish_scratch(h, blk);
            return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
        }
        return launch_status(launch_getri_small(a, identity ? nullptr : devIpiv, a, devInfo, h->stream));
    }

    aclsolverStatus_t aclsolverSgetriBatched(aclsolverHandle_t handle, int n, const float *const Aarray[], int lda,
                                             const int *PivotArray, float *const Carray[], int ldc, int *infoArray,
                                             int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int arg = batched_argument(n, Aarray, lda, PivotArray, Carray, ldc, infoArray, batchSize, false);
        if (arg) return invalid(h, infoArray, batchSize < 0 ? 1 : batchSize, arg);
        if (batchSize > MAX_BATCH) return invalid(h, infoArray, batchSize, 8);
        if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
        if (n == 0) return empty_info(h, infoArray, batchSize);
        Layout layout;
        layout.identity = PivotArray == nullptr;
        RealBatch a{nullptr, const_cast<float *const *>(Aarray), n, lda, 0, batchSize};
        if (h->device_checks)
        {
            aclsolverStatus_t st =
                check_arrays(h, n, Aarray, lda, PivotArray, Carray, ldc, infoArray, batchSize, false, layout);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
            st = check_finite(h, a, n, infoArray, batchSize, 2);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        }
        RealBatch c{nullptr, Carray, n, ldc, 0, batchSize};
        if (n > SMALL_N)
        {
            // above the register-resident orders: the blocked solve against the identity
            // (within tolerance of the reference's inverse order, not bit for bit)
            if (n > BLOCKED_SOLVE_MAX_N) return ACLSOLVER_STATUS_NOT_SUPPORTED;
            ScratchBlock *blk = acquire_scratch(h, getri_blocked_scratch_bytes(n, batchSize));
            if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
            aclsolverStatus_t launched = launch_status(launch_getri_blocked(
                a, layout.identity ? nullptr : PivotArray, c, infoArray, blk->ptr, h->stream));
            aclsolverStatus_t fin = finish_scratch(h, blk);
            return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
        }
        return launch_status(
            launch_getri_small(a, layout.identity ? nullptr : PivotArray, c, infoArray, h->stream));
    }

    aclsolverStatus_t aclsolverSmatinvBatched(aclsolverHandle_t handle, int n, const float *const A[], int lda,
                                              float *const Ainv[], int lda_inv, int *info, int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int arg = batched_argument(n, A, lda, nullptr, Ainv, lda_inv, info, batchSize, true);
        if (arg) return invalid(h, info, batchSize < 0 ? 1 : batchSize, arg);
        if (batchSize > MAX_BATCH) return invalid(h, info, batchSize, 7);
        if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
        if (n == 0) return empty_info(h, info, batchSize);
        Layout layout;
        RealBatch a{nullptr, const_cast<float *const *>(A), n, lda, 0, batchSize};
        if (h->device_checks)
        {
            aclsolverStatus_t st = check_arrays(h, n, A, lda, nullptr, Ainv, lda_inv, info, batchSize, true, layout);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
            st = check_finite(h, a, n, info, batchSize, 2);
            if (st != ACLSOLVER_STATUS_SUCCESS) return st;
        }
        // LU of a copy in Ainv (pivots in handle scratch), then the inverse in place.
        ScratchBlock *piv = acquire_scratch(h, (size_t)batchSize * n * sizeof(int));
        if (!piv) return ACLSOLVER_STATUS_ALLOC_FAILED;
        RealBatch c{nullptr, Ainv, n, lda_inv, 0, batchSize};
        cudaError_t e = launch_copy_matrices(a, c, n, h->stream);
        if (e == cudaSuccess) e = launch_getrf_small(c, n, static_cast<int *>(piv->ptr), info, h->stream);
        if (e == cudaSuccess) e = launch_getri_small(c, static_cast<int *>(piv->ptr), c, info, h->stream);
        aclsolverStatus_t launched = launch_status(e);
        aclsolverStatus_t fin = finish_scratch(h, piv);
        return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
    }

    aclsolverStatus_t aclsolverSgetrfBatched(aclsolverHandle_t handle, int n, float *const Aarray[], int lda,
                                             int *PivotArray, int *infoArray, int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        int arg = 0;
        if (n < 0 || n > 4096)
            arg = 1;
        else if (n > 0 && batchSize > 0 && !Aarray)
            arg = 2;
        else if (lda < std::max(1, n))
            arg = 3;
        else if (batchSize > 0 && !infoArray)
            arg = 5;
        else if (batchSize < 0)
            arg = 6;
        if (arg) return invalid(h, infoArray, batchSize < 0 ? 1 : batchSize, arg);
        if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
        if (n == 0) return launch_status(launch_fill_info(infoArray, 0, batchSize, h->stream));
        RealBatch a{nullptr, Aarray, n, lda, 0, batchSize};
        if (n <= SMALL_N) return launch_status(launch_getrf_small(a, n, PivotArray, infoArray, h->stream));
        if (n <= BLOCKED_MAX_N)
            return launch_status(launch_getrf_blocked(a, PivotArray, infoArray, 0, h->stream));
        // above the batched orders: one matrix at a time over the whole GPU; the pointer table
        // is read back first (this call synchronises once)
        std::vector<float *> ptrs((size_t)batchSize);
        cudaError_t e = cudaMemcpyAsync(ptrs.data(), Aarray, sizeof(float *) * (size_t)batchSize,
                                        cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return launch_status(e);
        ScratchBlock *blk = acquire_scratch(h, sizeof(LargeStatus) + 256);
        if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
        LargeStatus *status = static_cast<LargeStatus *>(blk->ptr);
        for (int q = 0; q < batchSize && e == cudaSuccess; ++q)
        {
            if (!ptrs[q])
                e = launch_fill_info(infoArray + q, -2, 1, h->stream);
            else
                e = launch_getrf_large(ptrs[q], n, n, lda, PivotArray ? PivotArray + (size_t)q * n : nullptr,
                                       infoArray + q, status, 0, h->stream);
        }
        aclsolverStatus_t launched = launch_status(e);
        aclsolverStatus_t fin = finish_scratch(h, blk);
        return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
    }

    aclsolverStatus_t aclsolverSgetrsBatched(aclsolverHandle_t handle, aclsolverOperation_t trans, int n, int nrhs,
                                             const float *const Aarray[], int lda, const int *PivotArray,
                                             float *const Barray[], int ldb, int *infoArray, int batchSize)
    {
        if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        const bool used = n > 0 && nrhs > 0 && batchSize > 0;
        int arg = 0;
        if (trans != ACLSOLVER_OP_N && trans != ACLSOLVER_OP_T)
            arg = 1;
        else if (n < 0 || n > LARGE_MAX_COLS)
            arg = 2;
        else if (nrhs < 0)
            arg = 3;
        else if (used && !Aarray)
            arg = 4;
        else if (lda < std::max(1, n))
            arg = 5;
        else if (used && !Barray)
            arg = 7;
        else if (ldb < std::max(1, n))
            arg = 8;
        else if (batchSize > 0 && !infoArray)
            arg = 9;
        else if (batchSize < 0)
            arg = 10;
        if (arg) return invalid(h, infoArray, batchSize < 0 ? 1 : batchSize, arg);
        if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
        if (!used) return launch_status(launch_fill_info(infoArray, 0, batchSize, h->stream));
        RealBatch a{nullptr, const_cast<float *const *>(Aarray), n, lda, 0, batchSize};
        RealBatch b{nullptr, Barray, n, ldb, 0, batchSize};
        if (n <= SMALL_N)
            return launch_status(launch_getrs_small(a, PivotArray, b, nrhs, trans == ACLSOLVER_OP_T ? 1 : 0,
                                                    infoArray, h->stream));
        if (trans == ACLSOLVER_OP_N && batchSize == 1 && n > BLOCKED_MAX_N && nrhs <= LARGE_SOLVE_MAX_RHS)
        {
            // one large system: the whole GPU sweeps it (same order, same bad-pivot contract)
            const size_t bytes = large_solve_scratch_bytes(n, nrhs) + 256;
            ScratchBlock *blk = acquire_scratch(h, bytes);
            if (!blk) return ACLSOLVER_STATUS_ALLOC_FAILED;
            int *bad = reinterpret_cast<int *>(static_cast<char *>(blk->ptr) + ((bytes - 256 + 15) & ~size_t(15)));
            aclsolverStatus_t launched = launch_status(launch_getrs_large(nullptr, Aarray, lda, n, PivotArray, nullptr,
                                                                          Barray, ldb, nrhs, blk->ptr, bad, infoArray,
                                                                          h->stream));
            aclsolverStatus_t fin = finish_scratch(h, blk);
            return launched != ACLSOLVER_STATUS_SUCCESS ? launched : fin;
        }
        return launch_status(launch_getrs_blocked(a, PivotArray, nullptr, b, nrhs, infoArray, nullptr, h->stream,
                                                  nullptr, nullptr, trans == ACLSOLVER_OP_T ? 1 : 0));
    }

    aclError aclsolverSgetrs(aclsolverHandle_t handle, const uint64_t trans, const int64_t n, const int64_t nrhs,
                             float *A, const int64_t lda, int32_t *ipiv, float *B, const int64_t ldb, int32_t *info)
    {
        if (!(n > 0 && n <= 8192 && nrhs > 0 && nrhs <= 8192 && lda >= n && ldb >= nrhs && A && B && ipiv && info &&
              lda - n <= 16383 && ldb - nrhs <= 16383))
        {
            fprintf(stderr, "[aclsolver] aclsolverSgetrs invalid param\n");
            return ACL_ERROR_INVALID_PARAM;
        }
        if (trans > 1)
        {
            fprintf(stderr, "[aclsolver] aclsolverSgetrs invalid param: trans must be 0 or 1\n");
            return ACL_ERROR_INVALID_PARAM;
        }
        for (int64_t k = 0; k < n; ++k)
            if (ipiv[k] < 1 || ipiv[k] > n)
            {
                *info = -4;
                return ACL_ERROR_INVALID_PARAM;
            }
        cudaStream_t stream = handle ? to_handle(handle)->stream : nullptr;
        // Stage: row-major host A (lda) -> device raw -> column-major LU (n x n, ld n);
        // row-major host B (ldb) -> device raw -> column-major (n x nrhs, ld n).
        const size_t a_raw = (size_t)n * lda * sizeof(float), b_raw = (size_t)n * ldb * sizeof(float);
        const size_t a_cm = (size_t)n * n * sizeof(float), b_cm = (size_t)n * nrhs * sizeof(float);
        const size_t p_bytes = (size_t)n * sizeof(int);
        char *base = nullptr;
        size_t total = a_raw + b_raw + a_cm + b_cm + p_bytes + 5 * 256;
        if (cudaMallocAsync(reinterpret_cast<void **>(&base), total, stream) != cudaSuccess)
        {
            cudaGetLastError();
            return (aclError)cudaErrorMemoryAllocation;
        }
        auto carve = [&](size_t bytes)
        {
            char *p = base;
            base += (bytes + 255) & ~size_t(255);
            return p;
        };
        char *start = base;
        float *d_araw = reinterpret_cast<float *>(carve(a_raw));
        float *d_braw = reinterpret_cast<float *>(carve(b_raw));
        float *d_a = reinterpret_cast<float *>(carve(a_cm));
        float *d_b = reinterpret_cast<float *>(carve(b_cm));
        int *d_p = reinterpret_cast<int *>(carve(p_bytes));
        cudaError_t e = cudaMemcpyAsync(d_araw, A, a_raw, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_braw, B, b_raw, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_p, ipiv, p_bytes, cudaMemcpyHostToDevice, stream);
        // Row-major (n rows, stride lda) viewed column-major is the n x n transpose.
        if (e == cudaSuccess) e = launch_transpose(d_araw, (int)lda, d_a, (int)n, (int)n, (int)n, stream);
        if (e == cudaSuccess) e = launch_transpose(d_braw, (int)ldb, d_b, (int)n, (int)nrhs, (int)n, stream);
        if (e == cudaSuccess)
        {
            RealBatch a{d_a, nullptr, (int)n, (int)n, 0, 1};
            RealBatch b{d_b, nullptr, (int)n, (int)n, 0, 1};
            e = n <= SMALL_N ? launch_getrs_small(a, d_p, b, (int)nrhs, (int)trans, nullptr, stream)
                             : launch_getrs_blocked(a, d_p, nullptr, b, (int)nrhs, nullptr, nullptr, stream, nullptr,
                                                    nullptr, (int)trans);
        }
        if (e == cudaSuccess) e = launch_transpose(d_b, (int)n, d_braw, (int)ldb, (int)n, (int)nrhs, stream);
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
