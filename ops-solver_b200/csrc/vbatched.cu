// vbatched.cu -- uneven-order batched complex64 Cholesky factor + solve in one persistent,
// size-bucketed launch, captured in a CUDA graph, with an autotuned launch shape.
//
// The reference factors one uniform order per call (src/cpotrf_batched/arch35/
// cpotrf_batched.cpp:14, Cholesky::Factor takes a single n), so an uneven batch costs it one
// factor call and one solve call per distinct order, and its batched solve takes one
// right-hand side per call (cpotrs_batched.cpp:19-21).  Here the plan sorts the matrices by
// order (largest first) into two task queues:
//   warp tasks  (n <= cutoff): one matrix per warp (or per 8/16-lane sub-warp), the factor
//               rows in registers, then the solve of every right-hand side in place;
//   block tasks (n >  cutoff): one matrix per block, the lower triangle in shared memory,
//               factor and solve without leaving shared memory -- orders up to 128 through
//               the packed-triangle routine of complex_block.cuh (a thread per row, in two
//               launches sized for 65..128 and for up to 64, so small matrices pack more
//               blocks per SM), larger ones through a generic block kernel.
// Two persistent kernels drain the queues through atomic task counters (no waiting: a
// block that finds the queue empty exits) and run as parallel branches of one graph.
// The arithmetic is that of complex_chol.cu (same per-element order), so results are
// bit-identical to aclsolverCpotrfBatched + aclsolverCpotrsBatchedMultiRhs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "complex_block.cuh"
#include "handle.h"
#include "vbatched.h"

namespace ops_solver
{
namespace
{
constexpr float FLT_MAX_VALUE = 3.402823466e38F;
constexpr int WT = 128;  // warp-kernel block size

__device__ __forceinline__ void sub_lconj(float &re, float &im, float ar, float ai, float cr, float ci)
{
    re = fma_rn(-ar, cr, re);
    re = fma_rn(-ai, ci, re);
    im = fma_rn(-ai, cr, im);
    im = fma_rn(ar, ci, im);
}
__device__ __forceinline__ void sub_prod(float &re, float &im, float ar, float ai, float yr, float yi)
{
    re = fma_rn(-ar, yr, re);
    re = fma_rn(ai, yi, re);
    im = fma_rn(-ar, yi, im);
    im = fma_rn(-ai, yr, im);
}
__device__ __forceinline__ float2 load_tri(const float2 *p, int lda, int upper, int i, int j)
{
    if (upper)
    {
        float2 v = p[(int64_t)i * lda + j];
        return make_float2(v.x, -v.y);
    }
    return p[(int64_t)j * lda + i];
}
__device__ __forceinline__ void store_tri(float2 *p, int lda, int upper, int i, int j, float re, float im)
{
    if (upper)
        p[(int64_t)i * lda + j] = make_float2(re, -im);
    else
        p[(int64_t)j * lda + i] = make_float2(re, im);
}

// Factor column K (orders differ between the sub-warps of a warp: every step up to the
// warp-wide order `nl` runs on all lanes; a failure is recorded only below the sub-warp's
// own order `n`, and steps beyond it touch only padding).  Recursion keeps indices static.
template <int N, int K>
__device__ __forceinline__ void vfactor_step(float (&re)[N], float (&im)[N], int n, int nl, int row, float2 *col,
                                             int &failure)
{
    if constexpr (K < N)
    {
        if (K < nl)
        {
            const float d = __shfl_sync(0xffffffffu, re[K], K, N);
            if (K < n && !(d > 0.0f && d <= FLT_MAX_VALUE) && failure == 0) failure = K + 1;
            const float s = sqrt_rn(d);
            if (row == K)
            {
                re[K] = s;
                im[K] = 0.0f;
            }
            else
            {
                re[K] = div_rn(re[K], s);
                im[K] = div_rn(im[K], s);
            }
            __syncwarp();
            col[row] = make_float2(re[K], im[K]);
            __syncwarp();
#pragma unroll
            for (int j = K + 1; j < N; ++j)
            {
                if (j < nl)
                {
                    const float2 c = col[j];
                    sub_lconj(re[j], im[j], re[K], im[K], c.x, c.y);
                }
            }
            vfactor_step<N, K + 1>(re, im, n, nl, row, col, failure);
        }
    }
}

// Forward sweep step K: y_K = z_K / l_KK broadcast, rows below subtract l_iK y_K.
template <int N, int K>
__device__ __forceinline__ void vforward_step(const float (&re)[N], const float (&im)[N], float &zr, float &zi, int n,
                                              int nl, int row)
{
    if constexpr (K < N)
    {
        if (K < nl)
        {
            const float dk = __shfl_sync(0xffffffffu, re[K], K, N);
            const float yr = div_rn(__shfl_sync(0xffffffffu, zr, K, N), dk);
            const float yi = div_rn(__shfl_sync(0xffffffffu, zi, K, N), dk);
            if (K < n && row > K) sub_prod(zr, zi, re[K], im[K], yr, yi);
            if (row == K)
            {
                zr = yr;
                zi = yi;
            }
            vforward_step<N, K + 1>(re, im, zr, zi, n, nl, row);
        }
    }
}

// Backward sweep step K (descending): x_K = z_K / l_KK broadcast, rows above subtract
// conj(l_Ki) x_K with l_Ki read from the shared-memory copy of the factor rows.
template <int N, int K>
__device__ __forceinline__ void vbackward_step(const float (&re)[N], float &zr, float &zi, int n, int nl, int row,
                                               const float2 *tile)
{
    if constexpr (K >= 0)
    {
        if (K < nl)
        {
            const float dk = __shfl_sync(0xffffffffu, re[K], K, N);
            const float yr = div_rn(__shfl_sync(0xffffffffu, zr, K, N), dk);
            const float yi = div_rn(__shfl_sync(0xffffffffu, zi, K, N), dk);
            if (K < n && row < K)
            {
                const float2 l = tile[K * (N + 1) + row];  // L(K, row)
                sub_prod(zr, zi, l.x, -l.y, yr, yi);
            }
            if (row == K)
            {
                zr = yr;
                zi = yi;
            }
        }
        vbackward_step<N, K - 1>(re, zr, zi, n, nl, row, tile);
    }
}

// One matrix per width-N sub-warp: factor (rows in registers), then nrhs solves.
template <int N>
__device__ void warp_posv(float2 *pa, float2 *pb, int n, int nl, int lda, int ldb, int nrhs, int upper, int row,
                          float2 *col, float2 *tile, int *info_out)
{
    float re[N], im[N];
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
        float2 v = make_float2(0.0f, 0.0f);
        if (pa && j < n && row < n && j <= row) v = load_tri(pa, lda, upper, row, j);
        re[j] = v.x;
        im[j] = v.y;
    }
    int failure = 0;
    vfactor_step<N, 0>(re, im, n, nl, row, col, failure);
    if (pa)
    {
        const int done = failure ? failure - 1 : n;
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (j < done && row < n && j <= row) store_tri(pa, lda, upper, row, j, re[j], im[j]);
    }
    if (row == 0 && info_out) *info_out = pa ? failure : -3;
    const bool solve = !failure && pa && pb;  // uniform within the sub-warp
    __syncwarp();
#pragma unroll
    for (int j = 0; j < N; ++j) tile[row * (N + 1) + j] = make_float2(re[j], im[j]);
    __syncwarp();
    for (int r = 0; r < nrhs; ++r)
    {
        float2 *xb = solve ? pb + (int64_t)r * ldb : nullptr;
        float zr = 0.0f, zi = 0.0f;
        if (solve && row < n)
        {
            const float2 v = xb[row];
            zr = v.x;
            zi = v.y;
        }
        vforward_step<N, 0>(re, im, zr, zi, n, nl, row);
        vbackward_step<N, N - 1>(re, zr, zi, n, nl, row, tile);
        if (solve && row < n) xb[row] = make_float2(zr, zi);
    }
}

template <int N>
__global__ void __launch_bounds__(WT) vb_warp_kernel(VbDesc d, const VbTask *tasks, int ntasks, int *counter)
{
    constexpr int MPW = 32 / N;
    __shared__ float2 cols[WT];
    __shared__ float2 tiles[(WT / 32) * MPW * N * (N + 1)];
    __shared__ int task_id;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row = lane % N, sub = lane / N;
    float2 *col = cols + warp * 32 + sub * N;
    float2 *tile = tiles + (warp * MPW + sub) * N * (N + 1);
    for (;;)
    {
        if (threadIdx.x == 0) task_id = atomicAdd(counter, 1);
        __syncthreads();
        const int t = task_id;
        __syncthreads();
        if (t >= ntasks) return;
        const VbTask task = tasks[t];
        const int slotq = warp * MPW + sub;  // matrix index within the task
        const bool mine = slotq < task.count;
        const int q = mine ? d.order[task.first + slotq] : 0;
        const int n = mine ? d.n[q] : 0;
        float2 *pa = mine ? slot(d.a, q) : nullptr;
        float2 *pb = mine ? slot(d.b, q) : nullptr;
        const int nl = (int)__reduce_max_sync(0xffffffffu, (unsigned)n);
        warp_posv<N>(pa, pb, n, nl, mine ? d.lda[q] : 1, mine ? d.ldb[q] : 1, d.nrhs, d.upper, row, col, tile,
                     mine ? d.info + q : nullptr);
    }
}

// One matrix per block: factor and solve in shared memory.
template <int T>
__global__ void __launch_bounds__(T) vb_block_kernel(VbDesc d, const VbTask *tasks, int ntasks, int *counter, int nmax)
{
    extern __shared__ float2 sa[];
    __shared__ int task_id;
    const int t = threadIdx.x;
    for (;;)
    {
        if (t == 0) task_id = atomicAdd(counter, 1);
        __syncthreads();
        const int id = task_id;
        __syncthreads();
        if (id >= ntasks) return;
        const int q = d.order[tasks[id].first];
        const int n = d.n[q], lda = d.lda[q], ldb = d.ldb[q], ps = n + 1;
        float2 *pa = slot(d.a, q);
        float2 *pb = slot(d.b, q);
        float2 *x = sa + (size_t)nmax * (nmax + 1);
        if (!pa)
        {
            if (t == 0) d.info[q] = -3;
            continue;
        }
        for (int j = 0; j < n; ++j)
            for (int i = j + t; i < n; i += T) sa[j * ps + i] = load_tri(pa, lda, d.upper, i, j);
        __syncthreads();
        int failure = 0;
        for (int k = 0; k < n; ++k)
        {
            const float dk = sa[k * ps + k].x;
            if (!(dk > 0.0f && dk <= FLT_MAX_VALUE))
            {
                failure = k + 1;
                break;
            }
            const float s = sqrt_rn(dk);
            __syncthreads();
            for (int i = k + t; i < n; i += T)
            {
                const float2 v = sa[k * ps + i];
                sa[k * ps + i] = i == k ? make_float2(s, 0.0f) : make_float2(div_rn(v.x, s), div_rn(v.y, s));
            }
            __syncthreads();
            for (int i = k + 1 + t; i < n; i += T)
            {
                const float2 l = sa[k * ps + i];
                for (int j = k + 1; j <= i; ++j)
                {
                    const float2 c = sa[k * ps + j];
                    float2 z = sa[j * ps + i];
                    sub_lconj(z.x, z.y, l.x, l.y, c.x, c.y);
                    sa[j * ps + i] = z;
                }
            }
            __syncthreads();
        }
        const int done = failure ? failure - 1 : n;
        for (int j = 0; j < done; ++j)
            for (int i = j + t; i < n; i += T)
            {
                const float2 v = sa[j * ps + i];
                store_tri(pa, lda, d.upper, i, j, v.x, v.y);
            }
        if (t == 0) d.info[q] = failure;
        if (!failure && pb)
        {
            for (int r = 0; r < d.nrhs; ++r)
            {
                float2 *xb = pb + (int64_t)r * ldb;
                for (int i = t; i < n; i += T) x[i] = xb[i];
                __syncthreads();
                for (int k = 0; k < n; ++k)
                {
                    const float dk = sa[k * ps + k].x;
                    const float2 zk = x[k];
                    const float yr = div_rn(zk.x, dk), yi = div_rn(zk.y, dk);
                    for (int i = k + 1 + t; i < n; i += T)
                    {
                        const float2 l = sa[k * ps + i];
                        float2 z = x[i];
                        sub_prod(z.x, z.y, l.x, l.y, yr, yi);
                        x[i] = z;
                    }
                    __syncthreads();
                    if (t == 0) x[k] = make_float2(yr, yi);
                    __syncthreads();
                }
                for (int k = n - 1; k >= 0; --k)
                {
                    const float dk = sa[k * ps + k].x;
                    const float2 zk = x[k];
                    const float yr = div_rn(zk.x, dk), yi = div_rn(zk.y, dk);
                    for (int i = t; i < k; i += T)
                    {
                        const float2 l = sa[i * ps + k];  // L(k, i)
                        float2 z = x[i];
                        sub_prod(z.x, z.y, l.x, -l.y, yr, yi);
                        x[i] = z;
                    }
                    __syncthreads();
                    if (t == 0) x[k] = make_float2(yr, yi);
                    __syncthreads();
                }
                for (int i = t; i < n; i += T) xb[i] = x[i];
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

// Orders up to T: one matrix per block through the packed-triangle routine.
template <int T>
__global__ void __launch_bounds__(T) vb_cb_kernel(VbDesc d, const VbTask *tasks, int ntasks, int *counter)
{
    extern __shared__ __align__(16) float cb_mem[];
    __shared__ int task_id;
    for (;;)
    {
        if (threadIdx.x == 0) task_id = atomicAdd(counter, 1);
        __syncthreads();
        const int id = task_id;
        __syncthreads();
        if (id >= ntasks) return;
        const int q = d.order[tasks[id].first];
        const int n = d.n[q];
        float2 *pa = slot(d.a, q);
        float2 *pb = slot(d.b, q);
        if (!pa)
        {
            if (threadIdx.x == 0) d.info[q] = -3;
            continue;
        }
        const CbShared s = cb_carve(cb_mem, n);
        cb_load<T>(s, pa, d.lda[q], d.upper, n);
        __syncthreads();
        const int failure = cb_factor<T>(s, n);
        cb_store<T>(s, pa, d.lda[q], d.upper, n, failure ? failure - 1 : n);
        if (threadIdx.x == 0) d.info[q] = failure;
        if (!failure && pb) cb_solve<T>(s, n, pb, d.ldb[q], d.nrhs);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// host side: buckets, tasks, launch shapes, autotuning and the graph
// ---------------------------------------------------------------------------------------
struct Shape
{
    int cutoff;       // largest order on the warp path: 8, 16 or 32
    int threads;      // block-path threads: 64, 128 or 256
    int warp_blocks;  // persistent warp-kernel blocks per SM
};

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

size_t block_smem(int nmax) { return ((size_t)nmax * (nmax + 1) + nmax) * sizeof(float2); }

cudaError_t launch_shape(const VbPlan *p, const Shape &s, const VbDesc &d, cudaStream_t main, cudaStream_t side)
{
    cudaError_t e = cudaSuccess;
    const int sms = sm_count();
    if (p->warp_tasks.at(s.cutoff).second > 0)
    {
        const VbTask *tasks = p->d_tasks + p->warp_tasks.at(s.cutoff).first;
        const int nt = p->warp_tasks.at(s.cutoff).second;
        int blocks = std::min(nt, sms * s.warp_blocks);
        if (s.cutoff == 8)
            vb_warp_kernel<8><<<blocks, WT, 0, side>>>(d, tasks, nt, p->d_counters + 0);
        else if (s.cutoff == 16)
            vb_warp_kernel<16><<<blocks, WT, 0, side>>>(d, tasks, nt, p->d_counters + 0);
        else
            vb_warp_kernel<32><<<blocks, WT, 0, side>>>(d, tasks, nt, p->d_counters + 0);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    // packed-triangle launches: 65..128 (128 threads), then up to 64 (64 threads)
    for (int part = 0; part < 2 && e == cudaSuccess; ++part)
    {
        const auto &range = part == 0 ? p->mid_tasks.at(s.cutoff) : p->small_tasks.at(s.cutoff);
        if (range.second == 0) continue;
        const int nmax = part == 0 ? p->mid_nmax.at(s.cutoff) : p->small_nmax.at(s.cutoff);
        const size_t smem = cb_smem_bytes(nmax);
        const VbTask *tasks = p->d_tasks + range.first;
        int per_sm = 1;
        if (part == 0)
        {
            cudaFuncSetAttribute(vb_cb_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vb_cb_kernel<128>, 128, smem);
            const int blocks = std::min(range.second, sms * std::max(1, per_sm));
            vb_cb_kernel<128><<<blocks, 128, smem, main>>>(d, tasks, range.second, p->d_counters + 2);
        }
        else
        {
            cudaFuncSetAttribute(vb_cb_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vb_cb_kernel<64>, 64, smem);
            const int blocks = std::min(range.second, sms * std::max(1, per_sm));
            vb_cb_kernel<64><<<blocks, 64, smem, main>>>(d, tasks, range.second, p->d_counters + 3);
        }
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    const auto &bt = p->big_tasks.at(s.cutoff);
    if (bt.second > 0)
    {
        const int nmax = p->block_nmax.at(s.cutoff);
        const size_t smem = block_smem(nmax);
        int per_sm = (int)std::max<size_t>(1, (200 * 1024) / std::max<size_t>(smem, 1));
        per_sm = std::min(per_sm, 2048 / s.threads);
        const int blocks = std::min(bt.second, sms * per_sm);
        const VbTask *tasks = p->d_tasks + bt.first;
        if (s.threads == 64)
        {
            cudaFuncSetAttribute(vb_block_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            vb_block_kernel<64><<<blocks, 64, smem, main>>>(d, tasks, bt.second, p->d_counters + 1, nmax);
        }
        else if (s.threads == 128)
        {
            cudaFuncSetAttribute(vb_block_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            vb_block_kernel<128><<<blocks, 128, smem, main>>>(d, tasks, bt.second, p->d_counters + 1, nmax);
        }
        else
        {
            cudaFuncSetAttribute(vb_block_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            vb_block_kernel<256><<<blocks, 256, smem, main>>>(d, tasks, bt.second, p->d_counters + 1, nmax);
        }
        e = cudaGetLastError();
    }
    return e;
}

// Enqueue one full execution: reset counters, fork the warp branch, block branch, join.
cudaError_t enqueue(VbPlan *p, const Shape &s, const VbDesc &d, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(p->d_counters, 0, 4 * sizeof(int), stream);
    if (e == cudaSuccess) e = cudaEventRecord(p->fork, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->side, p->fork, 0);
    if (e == cudaSuccess) e = launch_shape(p, s, d, stream, p->side);
    if (e == cudaSuccess) e = cudaEventRecord(p->join, p->side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, p->join, 0);
    return e;
}

std::string tune_key(const VbPlan *p)
{
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    // bucket histogram of orders (by 8) + nrhs + count
    std::vector<int> hist(513, 0);
    for (int n : p->host_n) hist[std::min(512, n / 8)]++;
    std::ostringstream k;
    k << prop.name << "|r" << p->nrhs << "|c" << p->count;
    unsigned long long h = 1469598103934665603ull;
    for (int v : hist) h = (h ^ (unsigned)v) * 1099511628211ull;
    k << "|h" << std::hex << h;
    return k.str();
}

std::string cache_path()
{
    const char *env = getenv("OPS_SOLVER_TUNE_CACHE");
    if (env && *env) return env;
    const char *home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/ops_solver_b200_vbatched_tune.txt";
}

bool load_cached(const std::string &key, Shape &s)
{
    std::ifstream in(cache_path());
    std::string line;
    while (std::getline(in, line))
    {
        size_t bar = line.rfind('\t');
        if (bar == std::string::npos || line.substr(0, bar) != key) continue;
        if (sscanf(line.c_str() + bar + 1, "%d %d %d", &s.cutoff, &s.threads, &s.warp_blocks) == 3) return true;
    }
    return false;
}

void store_cached(const std::string &key, const Shape &s)
{
    std::string path = cache_path();
    size_t slash = path.rfind('/');
    if (slash != std::string::npos)
    {
        std::string dir = path.substr(0, slash);
        std::string cmd = "mkdir -p '" + dir + "' 2>/dev/null";
        if (system(cmd.c_str()) != 0) return;
    }
    std::ofstream out(path, std::ios::app);
    out << key << '\t' << s.cutoff << ' ' << s.threads << ' ' << s.warp_blocks << '\n';
}

// Fills a scratch copy of the plan's matrices with n*I (positive definite, the timing of
// the kernels does not depend on the values) and B with ones.
__global__ void tune_fill(float2 *const *a, float2 *const *b, const int *n, const int *lda, const int *ldb, int nrhs,
                          int count)
{
    for (int q = blockIdx.x; q < count; q += gridDim.x)
    {
        const int nn = n[q];
        for (int e = threadIdx.x; e < nn * lda[q]; e += blockDim.x)
        {
            const int j = e / lda[q], i = e % lda[q];
            a[q][e] = make_float2(i == j ? (float)nn : 0.0f, 0.0f);
        }
        for (int e = threadIdx.x; e < nrhs * ldb[q]; e += blockDim.x) b[q][e] = make_float2(1.0f, 0.0f);
    }
}

Shape autotune(VbPlan *p, cudaStream_t stream)
{
    Shape best{32, 128, 8};
    std::string key = tune_key(p);
    if (load_cached(key, best)) return best;
    // scratch matrices of the plan's shapes
    size_t a_elems = 0, b_elems = 0;
    std::vector<size_t> a_off(p->count), b_off(p->count);
    for (int q = 0; q < p->count; ++q)
    {
        a_off[q] = a_elems;
        b_off[q] = b_elems;
        a_elems += (size_t)p->host_lda[q] * std::max(1, p->host_n[q]);
        b_elems += (size_t)p->host_ldb[q] * std::max(1, p->nrhs);
    }
    float2 *a = nullptr, *b = nullptr;
    float2 **ta = nullptr, **tb = nullptr;
    int *info = nullptr;
    if (cudaMalloc(&a, a_elems * sizeof(float2)) != cudaSuccess || cudaMalloc(&b, b_elems * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&ta, p->count * sizeof(void *)) != cudaSuccess ||
        cudaMalloc(&tb, p->count * sizeof(void *)) != cudaSuccess ||
        cudaMalloc(&info, p->count * sizeof(int)) != cudaSuccess)
    {
        cudaGetLastError();
        cudaFree(a);
        cudaFree(b);
        cudaFree(ta);
        cudaFree(tb);
        cudaFree(info);
        return best;
    }
    std::vector<float2 *> ha(p->count), hb(p->count);
    for (int q = 0; q < p->count; ++q)
    {
        ha[q] = a + a_off[q];
        hb[q] = b + b_off[q];
    }
    cudaMemcpy(ta, ha.data(), p->count * sizeof(void *), cudaMemcpyHostToDevice);
    cudaMemcpy(tb, hb.data(), p->count * sizeof(void *), cudaMemcpyHostToDevice);
    VbDesc d = p->desc;
    d.a = ta;
    d.b = tb;
    d.info = info;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_ms = 1e30f;
    const int cutoffs[3] = {8, 16, 32};
    const int threads[3] = {64, 128, 256};
    const int wblocks[2] = {4, 8};
    for (int c : cutoffs)
        for (int t : threads)
            for (int w : wblocks)
            {
                if (p->block_nmax[c] > 0 && block_smem(p->block_nmax[c]) > 220 * 1024) continue;
                Shape s{c, t, w};
                float ms = 0.0f;
                for (int rep = 0; rep < 3; ++rep)
                {
                    tune_fill<<<sm_count() * 4, 256, 0, stream>>>(ta, tb, p->d_n, p->d_lda, p->d_ldb, p->nrhs, p->count);
                    cudaEventRecord(e0, stream);
                    cudaError_t err = enqueue(p, s, d, stream);
                    cudaEventRecord(e1, stream);
                    if (err != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
                    {
                        cudaGetLastError();
                        ms = 1e30f;
                        break;
                    }
                    float one = 0.0f;
                    cudaEventElapsedTime(&one, e0, e1);
                    if (rep > 0) ms += one;
                }
                if (ms < best_ms)
                {
                    best_ms = ms;
                    best = s;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(a);
    cudaFree(b);
    cudaFree(ta);
    cudaFree(tb);
    cudaFree(info);
    cudaGetLastError();
    store_cached(key, best);
    return best;
}
}  // namespace

aclsolverStatus_t vb_plan_create(Handle *h, int uplo, const int *n, const int *lda, const int *ldb, int nrhs,
                                 int count, int autotune_flag, VbPlan **out)
{
    VbPlan *p = new (std::nothrow) VbPlan;
    if (!p) return ACLSOLVER_STATUS_ALLOC_FAILED;
    p->handle = h;
    p->count = count;
    p->nrhs = nrhs;
    p->host_n.assign(n, n + count);
    p->host_lda.assign(lda, lda + count);
    p->host_ldb.assign(ldb, ldb + count);
    // sort by order, largest first
    std::vector<int> order(count);
    for (int q = 0; q < count; ++q) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return n[x] > n[y]; });
    // task lists for every cutoff: [warp tasks][block tasks], contiguous per cutoff
    std::vector<VbTask> tasks;
    for (int cutoff : {8, 16, 32})
    {
        const int per_task = (WT / 32) * (32 / cutoff);
        std::vector<VbTask> warp, block;
        int nmax = 0;
        int i = 0;
        while (i < count && n[order[i]] > cutoff)
        {
            block.push_back({i, 1});
            nmax = std::max(nmax, n[order[i]]);
            ++i;
        }
        for (; i < count; i += per_task) warp.push_back({i, std::min(per_task, count - i)});
        p->warp_tasks[cutoff] = {(int)tasks.size(), (int)warp.size()};
        tasks.insert(tasks.end(), warp.begin(), warp.end());
        p->block_tasks[cutoff] = {(int)tasks.size(), (int)block.size()};
        p->block_nmax[cutoff] = nmax;
        // the block tasks are in descending order: split them at 128 and 64
        int big = 0, mid = 0;
        while (big < (int)block.size() && n[order[block[big].first]] > 128) ++big;
        while (big + mid < (int)block.size() && n[order[block[big + mid].first]] > 64) ++mid;
        const int base = (int)tasks.size();
        p->big_tasks[cutoff] = {base, big};
        p->mid_tasks[cutoff] = {base + big, mid};
        p->small_tasks[cutoff] = {base + big + mid, (int)block.size() - big - mid};
        p->mid_nmax[cutoff] = mid ? n[order[block[big].first]] : 0;
        p->small_nmax[cutoff] = big + mid < (int)block.size() ? n[order[block[big + mid].first]] : 0;
        tasks.insert(tasks.end(), block.begin(), block.end());
    }
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **ptr, size_t bytes)
    {
        if (e == cudaSuccess) e = cudaMalloc(ptr, bytes ? bytes : 4);
    };
    alloc((void **)&p->d_n, count * sizeof(int));
    alloc((void **)&p->d_lda, count * sizeof(int));
    alloc((void **)&p->d_ldb, count * sizeof(int));
    alloc((void **)&p->d_order, count * sizeof(int));
    alloc((void **)&p->d_tasks, tasks.size() * sizeof(VbTask));
    alloc((void **)&p->d_counters, 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(p->d_n, n, count * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_lda, lda, count * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_ldb, ldb, count * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_order, order.data(), count * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !tasks.empty())
        e = cudaMemcpy(p->d_tasks, tasks.data(), tasks.size() * sizeof(VbTask), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        vb_plan_destroy(p);
        return ACLSOLVER_STATUS_ALLOC_FAILED;
    }
    p->desc.n = p->d_n;
    p->desc.lda = p->d_lda;
    p->desc.ldb = p->d_ldb;
    p->desc.order = p->d_order;
    p->desc.nrhs = nrhs;
    p->desc.upper = uplo;
    Shape s = autotune_flag ? autotune(p, h->stream) : Shape{32, 128, 8};
    p->cutoff = s.cutoff;
    p->threads = s.threads;
    p->warp_blocks = s.warp_blocks;
    *out = p;
    return ACLSOLVER_STATUS_SUCCESS;
}

aclsolverStatus_t vb_plan_execute(VbPlan *p, float2 *const *a, float2 *const *b, int *info, cudaStream_t stream)
{
    VbDesc d = p->desc;
    d.a = a;
    d.b = b;
    d.info = info;
    Shape s{p->cutoff, p->threads, p->warp_blocks};
    // The graph is rebuilt when the caller's tables change; replays are a single launch.
    if (!p->graph_exec || p->graph_a != a || p->graph_b != b || p->graph_info != info || p->graph_stream != stream)
    {
        if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
        p->graph_exec = nullptr;
        cudaStream_t cap = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
        {
            cudaGetLastError();
            return ACLSOLVER_STATUS_EXECUTION_FAILED;
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) e = enqueue(p, s, d, cap);
        cudaError_t end = cudaStreamEndCapture(cap, &graph);
        if (e == cudaSuccess) e = end;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&p->graph_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            p->graph_exec = nullptr;
            return ACLSOLVER_STATUS_EXECUTION_FAILED;
        }
        p->graph_a = a;
        p->graph_b = b;
        p->graph_info = info;
        p->graph_stream = stream;
    }
    if (cudaGraphLaunch(p->graph_exec, stream) != cudaSuccess)
    {
        cudaGetLastError();
        return ACLSOLVER_STATUS_EXECUTION_FAILED;
    }
    return ACLSOLVER_STATUS_SUCCESS;
}

void vb_plan_destroy(VbPlan *p)
{
    if (!p) return;
    if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
    if (p->side) cudaStreamSynchronize(p->side);
    cudaFree(p->d_n);
    cudaFree(p->d_lda);
    cudaFree(p->d_ldb);
    cudaFree(p->d_order);
    cudaFree(p->d_tasks);
    cudaFree(p->d_counters);
    if (p->fork) cudaEventDestroy(p->fork);
    if (p->join) cudaEventDestroy(p->join);
    if (p->side) cudaStreamDestroy(p->side);
    cudaGetLastError();
    delete p;
}

}  // namespace ops_solver
