// vbatched.h -- the uneven-order batched complex Cholesky plan (see vbatched.cu).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <utility>
#include <vector>

#include "cann_ops_solver.h"

namespace ops_solver
{
struct Handle;

struct VbTask
{
    int first;  // position in the order-sorted index list
    int count;  // matrices in this task
};

// Kernel-side view of one execution: the caller's tables plus the plan's metadata.
struct VbDesc
{
    float2 *const *a = nullptr;
    float2 *const *b = nullptr;
    int *info = nullptr;
    const int *n = nullptr;
    const int *lda = nullptr;
    const int *ldb = nullptr;
    const int *order = nullptr;
    int nrhs = 0;
    int upper = 0;
};

struct VbPlan
{
    Handle *handle = nullptr;
    int count = 0, nrhs = 0;
    std::vector<int> host_n, host_lda, host_ldb;
    int *d_n = nullptr, *d_lda = nullptr, *d_ldb = nullptr, *d_order = nullptr, *d_counters = nullptr;
    VbTask *d_tasks = nullptr;
    // per warp-path cutoff (8, 16, 32): (offset, count) into d_tasks, and the block path's
    // largest order
    std::map<int, std::pair<int, int>> warp_tasks, block_tasks;
    std::map<int, int> block_nmax;
    // the block tasks of each cutoff split by order: above 128 (generic block kernel), 65..128
    // and up to 64 (packed-triangle kernels of 128 and 64 threads): (offset, count) and the
    // largest order of each part
    std::map<int, std::pair<int, int>> big_tasks, mid_tasks, small_tasks;
    std::map<int, int> mid_nmax, small_nmax;
    VbDesc desc;
    int cutoff = 32, threads = 128, warp_blocks = 8;  // the tuned launch shape
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    float2 *const *graph_a = nullptr;
    float2 *const *graph_b = nullptr;
    int *graph_info = nullptr;
    cudaStream_t graph_stream = nullptr;
};

aclsolverStatus_t vb_plan_create(Handle *h, int uplo, const int *n, const int *lda, const int *ldb, int nrhs,
                                 int count, int autotune, VbPlan **out);
aclsolverStatus_t vb_plan_execute(VbPlan *p, float2 *const *a, float2 *const *b, int *info, cudaStream_t stream);
void vb_plan_destroy(VbPlan *p);
}  // namespace ops_solver
