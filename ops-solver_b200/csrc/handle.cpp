// handle.cpp -- aclsolverCreate / Destroy / SetStream / GetStream and scratch management.
//
// Contracts follow src/utils/aclsolver_auxiliary.cpp:167-256 of the reference:
//   Create: NULL output -> HANDLE_IS_NULLPTR; *handle != NULL -> INVALID_VALUE;
//           no usable CUDA device/context -> NOT_INITIALIZED; allocation -> ALLOC_FAILED.
//   Destroy: NULL -> HANDLE_IS_NULLPTR; waits for every scratch block's last user.
//   SetStream: NULL handle -> HANDLE_IS_NULLPTR (NULL stream = legacy default stream).
//   GetStream: NULL handle -> HANDLE_IS_NULLPTR; NULL output -> INVALID_VALUE.
#include "handle.h"

#include <cuda.h>
#include <stdio.h>

#include <new>

namespace ops_solver
{
namespace
{
typedef CUresult (*MemGetAddressRangeFn)(CUdeviceptr *, size_t *, CUdeviceptr);

MemGetAddressRangeFn address_range_fn()
{
    static MemGetAddressRangeFn fn = []() -> MemGetAddressRangeFn
    {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
        {
            cudaGetLastError();
            return nullptr;
        }
        return reinterpret_cast<MemGetAddressRangeFn>(p);
    }();
    return fn;
}

void report(const char *what) { fprintf(stderr, "[aclsolver] %s\n", what); }

bool block_completed(const ScratchBlock &b)
{
    if (!b.recorded) return true;
    cudaError_t e = cudaEventQuery(b.done);
    if (e == cudaErrorNotReady)
    {
        return false;
    }
    if (e != cudaSuccess) cudaGetLastError();
    return e == cudaSuccess;
}
}  // namespace

bool is_device_pointer(const void *p)
{
    if (p == nullptr) return false;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

bool device_span(const void *p, size_t bytes)
{
    if (p == nullptr) return false;
    MemGetAddressRangeFn fn = address_range_fn();
    if (!fn) return true;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (fn(&base, &size, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) return false;
    uintptr_t a = (uintptr_t)p, b0 = (uintptr_t)base;
    return a >= b0 && bytes <= size - (a - b0);
}

bool SpanCache::ok(const void *p, size_t bytes, size_t align)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    if (!p || a % align != 0) return false;
    if (a >= begin && a < end && bytes <= end - a) return true;
    if (!is_device_pointer(p)) return false;
    MemGetAddressRangeFn fn = address_range_fn();
    if (!fn) return true;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (fn(&base, &size, (CUdeviceptr)a) != CUDA_SUCCESS) return false;
    begin = (uintptr_t)base;
    end = begin + size;
    return a >= begin && bytes <= end - a;
}

aclsolverStatus_t launch_status(cudaError_t launch)
{
    cudaError_t last = cudaGetLastError();
    return launch == cudaSuccess && last == cudaSuccess ? ACLSOLVER_STATUS_SUCCESS : ACLSOLVER_STATUS_EXECUTION_FAILED;
}

ScratchBlock *acquire_scratch(Handle *h, size_t bytes)
{
    if (bytes == 0) bytes = 256;
    for (ScratchBlock *b : h->scratch)
    {
        if (b->leased || b->bytes < bytes) continue;
        // Pending work on the same stream is ordered before the next use; another stream
        // must have finished with the block.
        if (b->stream != h->stream && !block_completed(*b)) continue;
        b->leased = true;
        return b;
    }
    ScratchBlock *b = new (std::nothrow) ScratchBlock;
    if (!b) return nullptr;
    if (cudaMalloc(&b->ptr, bytes) != cudaSuccess)
    {
        cudaGetLastError();
        delete b;
        return nullptr;
    }
    if (cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
    {
        cudaGetLastError();
        cudaFree(b->ptr);
        delete b;
        return nullptr;
    }
    b->bytes = bytes;
    b->leased = true;
    try
    {
        h->scratch.push_back(b);
    }
    catch (const std::bad_alloc &)
    {
        cudaEventDestroy(b->done);
        cudaFree(b->ptr);
        delete b;
        return nullptr;
    }
    return b;
}

aclsolverStatus_t finish_scratch(Handle *h, ScratchBlock *b)
{
    b->stream = h->stream;
    b->leased = false;
    if (cudaEventRecord(b->done, h->stream) != cudaSuccess)
    {
        cudaGetLastError();
        // Unknown completion: drain the stream so the block can be reused safely.
        b->recorded = false;
        if (cudaStreamSynchronize(h->stream) != cudaSuccess)
        {
            cudaGetLastError();
            b->leased = true;  // quarantined: never reused, leaked at Destroy
        }
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    b->recorded = true;
    return ACLSOLVER_STATUS_SUCCESS;
}

void *host_stage(Handle *h, size_t bytes)
{
    if (h->host_stage_bytes >= bytes && h->host_stage) return h->host_stage;
    if (h->host_stage) cudaFreeHost(h->host_stage);
    h->host_stage = nullptr;
    h->host_stage_bytes = 0;
    size_t want = bytes < 4096 ? 4096 : bytes;
    if (cudaMallocHost(&h->host_stage, want) != cudaSuccess)
    {
        cudaGetLastError();
        h->host_stage = nullptr;
        return nullptr;
    }
    h->host_stage_bytes = want;
    return h->host_stage;
}

int *device_flags(Handle *h)
{
    if (!h->dev_flags)
    {
        if (cudaMalloc(&h->dev_flags, 64 * sizeof(int)) != cudaSuccess ||
            cudaMemset(h->dev_flags, 0, 64 * sizeof(int)) != cudaSuccess)
        {
            cudaGetLastError();
            cudaFree(h->dev_flags);
            h->dev_flags = nullptr;
        }
    }
    return h->dev_flags;
}

}  // namespace ops_solver

using namespace ops_solver;

extern "C"
{
    aclsolverStatus_t aclsolverCreate(aclsolverHandle_t *handle)
    {
        if (handle == nullptr)
        {
            report("solver handle output is null");
            return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        }
        if (*handle != nullptr)
        {
            report("handle already initialized (*handle is not NULL)");
            return ACLSOLVER_STATUS_INVALID_VALUE;
        }
        int device = -1;
        if (cudaGetDevice(&device) != cudaSuccess || device < 0 || cudaFree(nullptr) != cudaSuccess)
        {
            cudaGetLastError();
            report("solver requires an initialized CUDA device context");
            return ACLSOLVER_STATUS_NOT_INITIALIZED;
        }
        Handle *h = new (std::nothrow) Handle;
        if (!h)
        {
            report("solver handle allocation failed");
            return ACLSOLVER_STATUS_ALLOC_FAILED;
        }
        h->device = device;
        *handle = h;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverDestroy(aclsolverHandle_t handle)
    {
        if (handle == nullptr) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        Handle *h = to_handle(handle);
        for (ScratchBlock *b : h->scratch)
        {
            bool safe = true;
            if (b->recorded && cudaEventSynchronize(b->done) != cudaSuccess)
            {
                cudaGetLastError();
                safe = b->stream && cudaStreamSynchronize(b->stream) == cudaSuccess;
                if (!safe) cudaGetLastError();
            }
            if (b->leased) safe = false;  // quarantined: completion unknown, leak it
            if (safe)
            {
                cudaEventDestroy(b->done);
                cudaFree(b->ptr);
            }
            delete b;
        }
        h->scratch.clear();
        if (h->dev_flags)
        {
            cudaStreamSynchronize(h->stream);
            cudaFree(h->dev_flags);
        }
        if (h->host_stage) cudaFreeHost(h->host_stage);
        cudaGetLastError();
        h->magic = 0;
        delete h;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSetStream(aclsolverHandle_t handle, aclrtStream stream)
    {
        if (handle == nullptr) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        to_handle(handle)->stream = reinterpret_cast<cudaStream_t>(stream);
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverSetDeviceChecks(aclsolverHandle_t handle, int enabled)
    {
        if (handle == nullptr) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (enabled != 0 && enabled != 1) return ACLSOLVER_STATUS_INVALID_VALUE;
        to_handle(handle)->device_checks = enabled != 0;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverGetDeviceChecks(aclsolverHandle_t handle, int *enabled)
    {
        if (handle == nullptr) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (enabled == nullptr) return ACLSOLVER_STATUS_INVALID_VALUE;
        *enabled = to_handle(handle)->device_checks ? 1 : 0;
        return ACLSOLVER_STATUS_SUCCESS;
    }

    aclsolverStatus_t aclsolverGetStream(aclsolverHandle_t handle, aclrtStream *stream)
    {
        if (handle == nullptr) return ACLSOLVER_STATUS_HANDLE_IS_NULLPTR;
        if (stream == nullptr) return ACLSOLVER_STATUS_INVALID_VALUE;
        *stream = reinterpret_cast<aclrtStream>(to_handle(handle)->stream);
        return ACLSOLVER_STATUS_SUCCESS;
    }
}
