// handle.h -- the solver handle and the host helpers shared by the C entry points.
//
// Mirrors the reference handle (src/utils/aclsolver_handle_internal.h:81-100): a stream
// binding plus handle-owned scratch that is reused across calls and released at
// Destroy only once its last user on the GPU has provably finished (event or stream
// synchronisation; a block whose completion cannot be proven is leaked rather than freed,
// as cholesky_host.cpp:80-99 does).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "cann_ops_solver.h"

namespace ops_solver
{

struct ScratchBlock
{
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;
    cudaStream_t stream = nullptr;
    bool leased = false;
    bool recorded = false;
};

struct Handle
{
    static constexpr uint32_t MAGIC = 0x42323030u;  // "B200"
    uint32_t magic = MAGIC;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool device_checks = true;  // synchronous device-data checks of the real LU family
    std::vector<ScratchBlock *> scratch;
    // Validation staging: a device flag word array and its pinned host mirror.
    int *dev_flags = nullptr;
    int *host_flags = nullptr;
    void *host_stage = nullptr;
    size_t host_stage_bytes = 0;
};

inline Handle *to_handle(aclsolverHandle_t h) { return static_cast<Handle *>(h); }

// Scratch lease: a block of at least `bytes` usable on the handle stream.  Returns nullptr
// on allocation failure.  finish_scratch records the completion event.
ScratchBlock *acquire_scratch(Handle *h, size_t bytes);
aclsolverStatus_t finish_scratch(Handle *h, ScratchBlock *b);

// Pinned host staging of at least `bytes` (grown on demand, freed at Destroy).
void *host_stage(Handle *h, size_t bytes);
// Device flag words (64 ints, zeroed when first allocated).  Words 0..31 are zeroed by their
// users before each use; words 60..63 belong to the batched solves' slot check, which leaves
// them zero after every launch.
int *device_flags(Handle *h);
constexpr int SLOT_CHECK_FLAGS = 60;

// Pointer classification: true for device (or managed) memory of the current context.
bool is_device_pointer(const void *p);
// True when [p, p+bytes) lies inside one device allocation (cuMemGetAddressRange).  When
// the driver query is unavailable the span is accepted.
bool device_span(const void *p, size_t bytes);

// Per-call memo of verified device allocations for pointer tables: a slot that lies inside
// an allocation already queried needs no driver call (tables of 10^6 slots over one slab
// cost one query instead of two per slot).
struct SpanCache
{
    uintptr_t begin = 0, end = 0;
    bool ok(const void *p, size_t bytes, size_t align);
};

// Status of the launches just enqueued (consumes this library's last CUDA error).
aclsolverStatus_t launch_status(cudaError_t launch);

}  // namespace ops_solver
