// noalloc.cu -- aclsolverSmatinvBatchedNoAlloc: the batched small-matrix inverse for
// callers that must not allocate device memory.
//
// aclsolverSmatinvBatched keeps the row-interchange pivots of the LU step in handle-owned
// scratch, which the handle allocates with cudaMalloc the first time (and again whenever a
// larger batch needs more).  Some callers cannot let a library allocate: hosts that hand
// all device memory out from their own pool and forbid allocations after start-up, and
// latency-critical loops where an allocation's implicit device synchronisation is not
// acceptable.  This entry keeps the pivots in a fixed array compiled into the library
// instead, so a call allocates nothing.  Its first call on a device resolves the array's
// device address (cudaGetSymbolAddress) and should come before any stream capture.
//
// The array (PIVOT_CAPACITY ints, 4 MiB) lives in every GPU that loads the library until the
// process exits.  All calls share it and it keeps the last call's contents; the LU step
// writes every pivot of every matrix before the inverse step reads it, so nothing needs
// clearing.  Calls whose executions overlap on the GPU (different streams or handles, or
// different host threads) race on the array: serialise them.
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
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) int pivot_scratch[PIVOT_CAPACITY];

// Device address of pivot_scratch, resolved once per device.  In host code the symbol
// names a host-side stand-in, never the device array, so the address must come from
// cudaGetSymbolAddress with the device current.
int *pivot_address(int device)
{
    static std::mutex lock;
    static int *address[MAX_DEVICES] = {nullptr};
    if (device < 0 || device >= MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> guard(lock);
    if (!address[device])
    {
        int *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), pivot_scratch);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            fprintf(stderr, "[aclsolver] aclsolverSmatinvBatchedNoAlloc: cudaGetSymbolAddress failed: %s\n",
                    cudaGetErrorString(e));
            return nullptr;
        }
        address[device] = ptr;
    }
    return address[device];
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
    else if ((int64_t)n * batchSize > PIVOT_CAPACITY)
    {
        fprintf(stderr,
                "[aclsolver] aclsolverSmatinvBatchedNoAlloc: n * batchSize = %lld exceeds the fixed pivot array "
                "(%d entries); split the batch\n",
                (long long)n * batchSize, PIVOT_CAPACITY);
        arg = 7;
    }
    if (arg)
    {
        const int64_t count = batchSize < 0 ? 1 : batchSize;
        if (info && count > 0 && is_device_pointer(info)) launch_fill_info(info, -arg, count, h->stream);
        cudaGetLastError();
        return ACLSOLVER_STATUS_INVALID_VALUE;
    }
    if (batchSize == 0) return ACLSOLVER_STATUS_SUCCESS;
    if (n == 0) return launch_status(launch_fill_info(info, 0, batchSize, h->stream));
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess)
    {
        cudaGetLastError();
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
