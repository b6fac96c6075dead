// potrf_small.cu -- batched real Cholesky factor and solve for n <= 32 on sm_100a.
//
// Layout: a sub-warp of N lanes (N = 8, 16 or 32) owns one matrix; lane i holds row i of
// the factor triangle in registers (r[j] = A(i, j) for j <= i).  32/N matrices share a
// warp, so an 8x8 batch keeps every lane busy.  Column broadcasts use width-N shuffles;
// the rank-4 trailing update reads the four finished columns of a row from a per-warp
// shared-memory stage (one broadcast 16-byte load per target column instead of four
// shuffles).  Failed matrices keep computing with the rest of the warp (no divergence
// around the shuffles) and store only their completed columns.
//
// Orders (the parity contract, restated in oracle/oracle.c):
//   ORDER_SIMT  (n <= 8)   cholesky_simt.cpp:52-92  left-looking fmaf, sqrt refined once
//   ORDER_GROUP (9..32)    cholesky_vector.cpp:588-794  groups of four, separate rounding
// Solve: cholesky_simt.cpp:93-117 (SolveKernel): forward fmaf chain then IEEE division,
// backward fmaf chain over ascending j then IEEE division.
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int ORDER_SIMT = 0;
constexpr int ORDER_GROUP = 1;
constexpr int THREADS = 128;
constexpr float FLT_MAX_VALUE = 3.402823466e38F;

// Row i of the lower factor: lower reads A[i + j*lda], upper reads the mirror A[j + i*lda].
__device__ __forceinline__ int64_t tri_index(int lda, int upper, int i, int j)
{
    return upper ? (int64_t)i * lda + j : (int64_t)j * lda + i;
}

// One group of four columns (cholesky_vector.cpp:745-794), then the next group; the
// recursion keeps every register index a compile-time constant.
template <int N, int BASE>
__device__ __forceinline__ void group_factor(float (&r)[N], int n, int row, int sub, int lane, float4 *my_stage,
                                             int &failure)
{
    if constexpr (BASE < N)
    {
        if (BASE < n)
        {
#pragma unroll
            for (int t = 0; t < 4; ++t)
            {
                const int k = BASE + t;
                if (k < n)
                {
                    float d = __shfl_sync(0xffffffffu, r[k], k, N);
                    if (!(d > 0.0f && d <= FLT_MAX_VALUE) && failure == 0) failure = k + 1;
                    float s = sqrt_rn(d);
                    r[k] = row == k ? s : div_rn(r[k], s);
#pragma unroll
                    for (int j = k + 1; j < BASE + 4; ++j)
                    {
                        if (j < n)
                        {
                            float alpha = __shfl_sync(0xffffffffu, r[k], j, N);
                            r[j] = sub_rn(r[j], mul_rn(r[k], alpha));
                        }
                    }
                }
            }
            if (BASE + 4 < n)
            {
                __syncwarp();
                my_stage[lane] = make_float4(r[BASE], r[BASE + 1], r[BASE + 2], r[BASE + 3]);
                __syncwarp();
#pragma unroll
                for (int j = BASE + 4; j < N; ++j)
                {
                    if (j < n)
                    {
                        float4 al = my_stage[sub * N + j];
                        float sum = mul_rn(r[BASE], al.x);
                        sum = add_rn(sum, mul_rn(r[BASE + 1], al.y));
                        sum = add_rn(sum, mul_rn(r[BASE + 2], al.z));
                        sum = add_rn(sum, mul_rn(r[BASE + 3], al.w));
                        r[j] = sub_rn(r[j], sum);
                    }
                }
            }
            group_factor<N, BASE + 4>(r, n, row, sub, lane, my_stage, failure);
        }
    }
}

template <int N, int ORDER>
__global__ void __launch_bounds__(THREADS) potrf_small_kernel(float *single, float *const *table, int first, int n,
                                                               int lda, int upper, int count, int *info)
{
    constexpr int MPW = 32 / N;  // matrices per warp
    __shared__ float4 stage[THREADS];
    const int lane = threadIdx.x & 31;
    const int row = lane % N;
    const int sub = lane / N;
    const int warp_global = (blockIdx.x * THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * THREADS) >> 5;
    float4 *my_stage = stage + (threadIdx.x & ~31);

    for (int64_t group = warp_global; group * MPW < count; group += warps_total)
    {
        const int64_t q = group * MPW + sub;
        const bool in_batch = q < count;
        float *p = nullptr;
        if (in_batch) p = table ? slot(table, first + q) : single;
        const bool live = p != nullptr;

        float r[N];
#pragma unroll
        for (int j = 0; j < N; ++j)
        {
            r[j] = 0.0f;
            if (live && j < n && row < n && j <= row) r[j] = p[tri_index(lda, upper, row, j)];
        }

        int failure = 0;
        if (ORDER == ORDER_SIMT)
        {
#pragma unroll
            for (int k = 0; k < N; ++k)
            {
                if (k < n)
                {
                    // acc = A(i,k) - sum_t A(i,t) A(k,t), fmaf in ascending t; on lane k this
                    // is the diagonal chain d = fmaf(-f, f, d).
                    float acc = r[k];
#pragma unroll
                    for (int t = 0; t < k; ++t)
                    {
                        float lk = __shfl_sync(0xffffffffu, r[t], k, N);
                        acc = fma_rn(-r[t], lk, acc);
                    }
                    float d = __shfl_sync(0xffffffffu, acc, k, N);
                    if (!(d > 0.0f) && failure == 0) failure = k + 1;
                    float root = sqrt_rn(d);
                    float correction = fma_rn(-root, root, d);
                    d = fma_rn(correction, div_rn(0.5f, root), root);
                    r[k] = row == k ? d : div_rn(acc, d);
                }
            }
        }
        else
        {
            group_factor<N, 0>(r, n, row, sub, lane, my_stage, failure);
        }

        if (live)
        {
            const int done = failure ? failure - 1 : n;
#pragma unroll
            for (int j = 0; j < N; ++j)
                if (j < done && row < n && j <= row) p[tri_index(lda, upper, row, j)] = r[j];
        }
        if (in_batch && row == 0) info[q] = live ? failure : -3;
    }
}

// SolveKernel order.  Forward: lane j divides its accumulated value at step j and
// broadcasts it; rows below take fmaf(-L(i,j), x_j, x).  Backward: x_i accumulates
// fmaf(-L(j,i), x_j, x) over ascending j > i, so each x_i waits for x_{i+1}; lane i holds
// column i of L (read back transposed from shared memory) and all lanes keep the
// broadcast solution values xs[] in registers.
template <int N>
__global__ void __launch_bounds__(THREADS) potrs_small_kernel(float *a_single, float *const *a_table, int a_first,
                                                               float *b_single, float *const *b_table, int b_first,
                                                               int n, int lda, int ldb, int nrhs, int upper, int count,
                                                               const int *info)
{
    constexpr int MPW = 32 / N;
    constexpr int P = N + 1;
    __shared__ float stage[(THREADS / 32) * MPW * N * P];
    if (info[0] != 0) return;
    const int lane = threadIdx.x & 31;
    const int row = lane % N;
    const int sub = lane / N;
    const int warp = threadIdx.x >> 5;
    const int warp_global = (blockIdx.x * THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * THREADS) >> 5;
    float *tile = stage + (warp * MPW + sub) * N * P;

    for (int64_t group = warp_global; group * MPW < count; group += warps_total)
    {
        const int64_t q = group * MPW + sub;
        const bool in_batch = q < count;
        float *pa = nullptr, *pb = nullptr;
        if (in_batch)
        {
            pa = a_table ? slot(a_table, a_first + q) : a_single;
            pb = b_table ? slot(b_table, b_first + q) : b_single;
        }
        const bool live = pa != nullptr && pb != nullptr;

        float r[N];  // row `row` of L
        float diag = 1.0f;
#pragma unroll
        for (int j = 0; j < N; ++j)
        {
            r[j] = 0.0f;
            if (live && j < n && row < n && j <= row) r[j] = pa[tri_index(lda, upper, row, j)];
            if (j == row) diag = r[j];
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < N; ++j) tile[j * P + row] = r[j];  // tile[j*P + i] = L(i, j)
        __syncwarp();
        float c[N];  // column `row` of L: c[j] = L(j, row)
#pragma unroll
        for (int j = 0; j < N; ++j) c[j] = tile[row * P + j];

        for (int rhs = 0; rhs < nrhs; ++rhs)
        {
            float *x_ptr = live ? pb + (int64_t)rhs * ldb : nullptr;
            float x = (live && row < n) ? x_ptr[row] : 0.0f;
            // forward
#pragma unroll
            for (int j = 0; j < N; ++j)
            {
                if (j < n)
                {
                    if (row == j) x = div_rn(x, diag);
                    float xj = __shfl_sync(0xffffffffu, x, j, N);
                    if (row > j) x = fma_rn(-r[j], xj, x);
                }
            }
            // backward
            float xs[N];
#pragma unroll
            for (int i = N - 1; i >= 0; --i)
            {
                xs[i] = 0.0f;
                if (i < n)
                {
                    float acc = x;
#pragma unroll
                    for (int j = i + 1; j < N; ++j)
                        if (j < n) acc = fma_rn(-c[j], xs[j], acc);
                    acc = div_rn(acc, diag);
                    if (row == i) x = acc;
                    xs[i] = __shfl_sync(0xffffffffu, x, i, N);
                }
            }
            if (live && row < n) x_ptr[row] = x;
        }
    }
}

template <int N, int ORDER>
cudaError_t potrf_small_n(const RealBatch &a, int upper, int *info, cudaStream_t stream)
{
    constexpr int MPW = 32 / N;
    int64_t warps = (a.count + MPW - 1) / MPW;
    int64_t blocks = (warps * 32 + THREADS - 1) / THREADS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    potrf_small_kernel<N, ORDER><<<(unsigned)blocks, THREADS, 0, stream>>>(a.single, a.table, a.first, a.n, a.ld,
                                                                           upper, a.count, info);
    return cudaGetLastError();
}

template <int N>
cudaError_t potrs_small_n(const RealBatch &a, const RealBatch &b, int nrhs, int upper, const int *info,
                          cudaStream_t stream)
{
    constexpr int MPW = 32 / N;
    int64_t warps = (a.count + MPW - 1) / MPW;
    int64_t blocks = (warps * 32 + THREADS - 1) / THREADS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    potrs_small_kernel<N><<<(unsigned)blocks, THREADS, 0, stream>>>(a.single, a.table, a.first, b.single, b.table,
                                                                    b.first, a.n, a.ld, b.ld, nrhs, upper, a.count,
                                                                    info);
    return cudaGetLastError();
}

__global__ void fill_info_kernel(int *info, int value, int64_t count)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        info[i] = value;
}

// One block scans both pointer tables; a single thread writes the outcome.
__global__ void __launch_bounds__(1024) solve_slot_check_kernel(int *info, float *const *a, float *const *b,
                                                                int count)
{
    __shared__ int flags;
    if (threadIdx.x == 0) flags = 0;
    __syncthreads();
    int mask = 0;
    for (int q = threadIdx.x; q < count; q += blockDim.x)
    {
        if (!slot(a, q)) mask |= 1;
        if (!slot(b, q)) mask |= 2;
    }
    if (mask) atomicOr(&flags, mask);
    __syncthreads();
    if (threadIdx.x == 0) info[0] = (flags & 1) ? -4 : (flags & 2) ? -6 : 0;
}
}  // namespace

cudaError_t launch_fill_info(int *info, int value, int64_t count, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    int64_t blocks = (count + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    fill_info_kernel<<<(unsigned)blocks, 256, 0, stream>>>(info, value, count);
    return cudaGetLastError();
}

cudaError_t launch_solve_slot_check(int *info, float *const *a, float *const *b, int count, cudaStream_t stream)
{
    int threads = 128;
    while (threads < count && threads < 1024) threads *= 2;
    solve_slot_check_kernel<<<1, threads, 0, stream>>>(info, a, b, count);
    return cudaGetLastError();
}

cudaError_t launch_potrf_small(const RealBatch &a, int upper, int *info, cudaStream_t stream)
{
    if (a.n <= 8) return potrf_small_n<8, ORDER_SIMT>(a, upper, info, stream);
    if (a.n <= 16) return potrf_small_n<16, ORDER_GROUP>(a, upper, info, stream);
    return potrf_small_n<32, ORDER_GROUP>(a, upper, info, stream);
}

cudaError_t launch_potrs_small(const RealBatch &a, const RealBatch &b, int nrhs, int upper, const int *info,
                               cudaStream_t stream)
{
    if (a.n <= 8) return potrs_small_n<8>(a, b, nrhs, upper, info, stream);
    if (a.n <= 16) return potrs_small_n<16>(a, b, nrhs, upper, info, stream);
    return potrs_small_n<32>(a, b, nrhs, upper, info, stream);
}

}  // namespace ops_solver
