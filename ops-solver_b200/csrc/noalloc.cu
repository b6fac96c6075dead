// noalloc.cu -- aclsolverSmatinvBatchedNoAlloc: the batched small-matrix inverse for
// callers that must not allocate device memory.
//
// aclsolverSmatinvBatched keeps the row-interchange pivots of the LU step in handle-owned
// scratch, which the handle allocates with cudaMalloc the first time (and again whenever a
// larger batch needs more).  Some callers cannot let a library allocate: hosts that hand
// all device memory out from their own pool and forbid allocations after start-up, and
// latency-critical loops where an allocation's implicit device synchronisation is not
// acceptable.  This entry keeps the pivots in a fixed array compiled into the library
// instead, so a call allocates nothing.  Its first call on a device (and the first call
// after that device's context was reset) resolves the array's device address
// (cudaGetSymbolAddress) and should come before any stream capture.
//
// The array (PIVOT_CAPACITY ints, 4 MiB) lives in every GPU that loads the library until the
// process exits.  All calls share it and it keeps the last call's contents; the LU step
// writes every pivot of every matrix before the inverse step reads it, so nothing needs
// clearing.  Calls whose executions overlap on the GPU (different streams or handles, or
// different host threads) race on the array: serialise them.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>

#include "handle.h"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int PIVOT_CAPACITY = 1 << 20;  // ints: n * batchSize must not exceed this
constexpr int MAX_BATCH = 10000000;      // the batched inverse's limit (real_lu_common.h:18)
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) int pivot_scratch[PIVOT_CAPACITY];

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Process-unique id of the current context (cuCtxGetId never reuses an id, unlike the
// CUcontext handle, which a context created after a reset may share with its predecessor).
// 0 when the driver does not offer the query.
unsigned long long current_context_id()
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, []
    {
        void *p = nullptr, *q = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1) == cudaSuccess &&
            r1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2) == cudaSuccess &&
            r2 == cudaDriverEntryPointSuccess)
        {
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
            get_id = reinterpret_cast<CtxGetIdFn>(q);
        }
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of pivot_scratch for the current device and context.  In host code the
// symbol names a host-side stand-in, never the device array, so the address must come from
// cudaGetSymbolAddress with the device current.  It is resolved once per device and
// context: a reset device gets a new context (new id), whose module holds the array at a
// new address.  Without the context query the address is resolved on every call.
int *pivot_address(int device)
{
    static std::mutex lock;
    static int *address[MAX_DEVICES] = {nullptr};
    static unsigned long long context[MAX_DEVICES] = {0};
    if (device < 0 || device >= MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> guard(lock);
    const unsigned long long id = current_context_id();
    if (id != 0 && address[device] && context[device] == id) return address[device];
    int *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), pivot_scratch);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        fprintf(stderr, "[aclsolver] aclsolverSmatinvBatchedNoAlloc: cudaGetSymbolAddress failed: %s\n",
                cudaGetErrorString(e));
        return nullptr;
    }
    // The runtime has set the context up by now; its id keys the cached address (0, no
    // query available: nothing is cached and the next call resolves the address again).
    address[device] = ptr;
    context[device] = current_context_id();
    return ptr;
}

// True when info[0..count) is an aligned span inside one device allocation (the rule the
// batched LU entries apply before they write argument errors to info).
bool info_fits(const int *info, int64_t count)
{
    return info && reinterpret_cast<uintptr_t>(info) % alignof(int) == 0 && is_device_pointer(info) &&
           device_span(info, (size_t)count * sizeof(int));
}

aclsolverStatus_t invalid(Handle *h, int *info, int64_t count, int argument)
{
    if (count > 0 && info_fits(info, count))
    {
        if (launch_fill_info(info, -argument, count, h->stream) != cudaSuccess) cudaGetLastError();
    }
    return ACLSOLVER_STATUS_INVALID_VALUE;
}
}  // namespace
}  // namespace ops_solver

using namespace ops_solver;

extern "C" __attribute__((visibility("default"))) aclsolverStatus_t aclsolverSmatinvBatchedNoAlloc(
    aclsolverHandle_t handle, int n, const float *const A[], int lda, float *const Ainv[], int lda_inv, int *info,
    int batchSize)
{
    if (!handle) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
    Handle *h = to_handle(handle);
    // Argument ladder of aclsolverSmatinvBatched (real_lu_common.h:20-60 with factor = true).
    int arg = 0;
    if (n < 0 || n > 32)
        arg = 1;
    else if (n > 0 && batchSize > 0 && !is_device_pointer(A))
        arg = 2;
    else if (lda < (n > 1 ? n : 1))
        arg = 3;
    else if (n > 0 && batchSize > 0 && !is_device_pointer(Ainv))
        arg = 4;
    else if (lda_inv < (n > 1 ? n : 1))
        arg = 5;
    else if (batchSize > 0 && !is_device_pointer(info))
        arg = 6;
    else if (batchSize < 0)
        arg = 7;
    if (arg) return invalid(h, info, batchSize < 0 ? 1 : batchSize, arg);
    if (batchSize > MAX_BATCH) return invalid(h, info, batchSize, 7);
    if ((int64_t)n * batchSize > PIVOT_CAPACITY)
    {
        fprintf(stderr,
                "[aclsolver] aclsolverSmatinvBatchedNoAlloc: n * batchSize = %lld exceeds the fixed pivot array "
                "(%d entries); split the batch\n",
                (long long)n * batchSize, PIVOT_CAPACITY);
        return invalid(h, info, batchSize, 7);
    }
    if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
    if (!info_fits(info, batchSize)) return ACLSOLVER_STATUS_INVALID_VALUE;
    if (n == 0) return launch_status(launch_fill_info(info, 0, batchSize, h->stream));
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    if (device != h->device)
    {
        fprintf(stderr,
                "[aclsolver] aclsolverSmatinvBatchedNoAlloc: the current device (%d) is not the handle's (%d)\n",
                device, h->device);
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    int *pivots = pivot_address(device);
    if (!pivots) return ACLSOLVER_STATUS_EXECUTION_FAILED;
    RealBatch a{nullptr, const_cast<float *const *>(A), n, lda, 0, batchSize};
    RealBatch c{nullptr, Ainv, n, lda_inv, 0, batchSize};
    cudaError_t e = launch_copy_matrices(a, c, n, h->stream);
    if (e == cudaSuccess) e = launch_getrf_small(c, n, pivots, info, h->stream);
    if (e == cudaSuccess) e = launch_getri_small(c, pivots, c, info, h->stream);
    return launch_status(e);
}
