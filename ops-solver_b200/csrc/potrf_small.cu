// potrf_small.cu -- batched real Cholesky factor and solve for n <= 32 on sm_100a.
//
// Factor, n <= 8: a sub-warp of 8 lanes per matrix, lane i holds row i of the factor in
// registers (r[j] = A(i, j), j <= i); column broadcasts are width-8 shuffles.
// Factor, 9..32 (the grouped order): L = 8 or 16 lanes per matrix, each lane holding
// N / L rows paired so that every lane holds the same number of elements (lane l takes rows
// l and 2L - 1 - l of each 2L-row band: 0 and 31, 1 and 30, ... for L = 16); the square root
// and divisions of a column run on all rows at once, column values are broadcast by width-L
// shuffles, and the rank-4 trailing update reads the four finished columns of a row from a
// per-matrix shared stage (one broadcast 16-byte load per target row).  Failed matrices keep
// computing with the rest of the warp (no divergence around the shuffles) and store only
// their completed columns.
// Solve (the reference's SolveKernel shape): one lane per matrix; a warp stages its 32
// matrices' lower triangles in shared memory (coalesced column copies) and lane m runs the
// forward and backward sweeps of matrix m there, so no lane idles and no value is broadcast.
//
// Orders (the parity contract, restated in oracle/oracle.c):
//   ORDER_SIMT  (n <= 8)   cholesky_simt.cpp:52-92  left-looking fmaf, sqrt refined once
//   ORDER_GROUP (9..32)    cholesky_vector.cpp:588-794  groups of four, separate rounding
// Solve: cholesky_simt.cpp:93-117 (SolveKernel): forward fmaf chain then IEEE division,
// backward fmaf chain over ascending j then IEEE division.
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
constexpr int ORDER_SIMT = 0;
constexpr int THREADS = 128;
constexpr float FLT_MAX_VALUE = 3.402823466e38F;

// Row i of the lower factor: lower reads A[i + j*lda], upper reads the mirror A[j + i*lda].
__device__ __forceinline__ int64_t tri_index(int lda, int upper, int i, int j)
{
    return upper ? (int64_t)i * lda + j : (int64_t)j * lda + i;
}

template <int N, int ORDER>
__global__ void __launch_bounds__(THREADS) potrf_small_kernel(float *single, float *const *table, int first, int n,
                                                               int lda, int upper, int count, int *info)
{
    constexpr int MPW = 32 / N;  // matrices per warp
    const int lane = threadIdx.x & 31;
    const int row = lane % N;
    const int sub = lane / N;
    const int warp_global = (blockIdx.x * THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * THREADS) >> 5;

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

// Row held in slot s by lane l of an L-lane group: even slots run up a 2L-row band, odd
// slots run down it, so each lane's rows sum to the same length.
__device__ __forceinline__ int group_row(int s, int l, int L) { return (s & 1) ? (s + 1) * L - 1 - l : s * L + l; }

// In-group update of column J by the finished column K: a_ij -= l_iK * l_JK (separate
// roundings), for every row (rows above J take junk).
template <int N, int L, int K, int J, int END>
__device__ __forceinline__ void lgroup_inner(float (&r)[N / L][N], int n)
{
    constexpr int R = N / L;
    constexpr int SJ = J / L;
    constexpr int LJ = (SJ & 1) ? (SJ + 1) * L - 1 - J : J - SJ * L;
    if constexpr (J < END)
    {
        if (J < n)
        {
            const float alpha = __shfl_sync(0xffffffffu, r[SJ][K], LJ, L);
#pragma unroll
            for (int s = 0; s < R; ++s)
                if ((s + 1) * L - 1 >= J) r[s][J] = sub_rn(r[s][J], mul_rn(r[s][K], alpha));
            lgroup_inner<N, L, K, J + 1, END>(r, n);
        }
    }
}

// Column K of the grouped order with L lanes per matrix and R = N / L rows per lane
// (r[s][j] = A(row_s, j); entries right of a row's diagonal and rows at or past n are junk
// that is never stored): the pivot check, the square root, the column's IEEE divisions and the
// in-group updates of the group's later columns.  Template indices keep every register
// index static.
template <int N, int L, int K, int END>
__device__ __forceinline__ void lgroup_column(float (&r)[N / L][N], const int (&row)[N / L], int n, int &failure)
{
    constexpr int R = N / L;
    constexpr int SK = K / L;
    constexpr int LK = (SK & 1) ? (SK + 1) * L - 1 - K : K - SK * L;
    if constexpr (K < END)
    {
        if (K < n)
        {
            const float d = __shfl_sync(0xffffffffu, r[SK][K], LK, L);
            if (!(d > 0.0f && d <= FLT_MAX_VALUE) && failure == 0) failure = K + 1;
            const float sq = sqrt_rn(d);
            const float y = div_prepare(sq);
            const bool ok = div_range(sq);
#pragma unroll
            for (int s = 0; s < R; ++s)
            {
                if ((s + 1) * L - 1 >= K)
                {
                    if (row[s] == K)
                        r[s][K] = sq;
                    else if (row[s] > K)
                        r[s][K] = div_by(r[s][K], sq, y, ok);
                }
            }
            lgroup_inner<N, L, K, K + 1, END>(r, n);
            lgroup_column<N, L, K + 1, END>(r, row, n, failure);
        }
    }
}

// Rank-4 trailing update of column J (J >= BASE + 4) from the stage of the group's columns.
template <int N, int L, int BASE, int J>
__device__ __forceinline__ void lgroup_trail(float (&r)[N / L][N], int n, const float4 *stage)
{
    constexpr int R = N / L;
    if constexpr (J < N)
    {
        if (J < n)
        {
            const float4 al = stage[J];
#pragma unroll
            for (int s = 0; s < R; ++s)
            {
                if ((s + 1) * L - 1 >= J)
                {
                    float sum = mul_rn(r[s][BASE], al.x);
                    sum = add_rn(sum, mul_rn(r[s][BASE + 1], al.y));
                    sum = add_rn(sum, mul_rn(r[s][BASE + 2], al.z));
                    sum = add_rn(sum, mul_rn(r[s][BASE + 3], al.w));
                    r[s][J] = sub_rn(r[s][J], sum);
                }
            }
            lgroup_trail<N, L, BASE, J + 1>(r, n, stage);
        }
    }
}

// One group of four columns, then the next.
template <int N, int L, int BASE>
__device__ __forceinline__ void lgroup_factor(float (&r)[N / L][N], const int (&row)[N / L], int n, float4 *stage,
                                              int &failure)
{
    constexpr int R = N / L;
    if constexpr (BASE < N)
    {
        if (BASE < n)
        {
            lgroup_column<N, L, BASE, BASE + 4>(r, row, n, failure);
            if (BASE + 4 < n)
            {
                __syncwarp();
#pragma unroll
                for (int s = 0; s < R; ++s)
                    stage[row[s]] = make_float4(r[s][BASE], r[s][BASE + 1], r[s][BASE + 2], r[s][BASE + 3]);
                __syncwarp();
                lgroup_trail<N, L, BASE, BASE + 4>(r, n, stage);
            }
            lgroup_factor<N, L, BASE + 4>(r, row, n, stage, failure);
        }
    }
}

template <int N, int L>
__global__ void __launch_bounds__(THREADS, 5) potrf_group_kernel(float *single, float *const *table, int first, int n,
                                                               int lda, int upper, int count, int *info)
{
    constexpr int R = N / L;     // rows per lane
    constexpr int MPW = 32 / L;  // matrices per warp
    __shared__ float4 stage[THREADS / 32][MPW][N + 1];
    const int lane = threadIdx.x & 31;
    const int l = lane % L;
    const int sub = lane / L;
    const int warp_global = (blockIdx.x * THREADS + threadIdx.x) >> 5;
    const int warps_total = (gridDim.x * THREADS) >> 5;
    float4 *my_stage = stage[threadIdx.x >> 5][sub];
    int row[R];
#pragma unroll
    for (int s = 0; s < R; ++s) row[s] = group_row(s, l, L);

    for (int64_t group = warp_global; group * MPW < count; group += warps_total)
    {
        const int64_t q = group * MPW + sub;
        const bool in_batch = q < count;
        float *p = nullptr;
        if (in_batch) p = table ? slot(table, first + q) : single;
        const bool live = p != nullptr;

        float r[R][N];
#pragma unroll
        for (int s = 0; s < R; ++s)
        {
#pragma unroll
            for (int j = 0; j < N; ++j)
            {
                r[s][j] = 0.0f;
                if (j < (s + 1) * L && live && j < n && row[s] < n && j <= row[s])
                    r[s][j] = p[tri_index(lda, upper, row[s], j)];
            }
        }
        int failure = 0;
        lgroup_factor<N, L, 0>(r, row, n, my_stage, failure);
        if (live)
        {
            const int done = failure ? failure - 1 : n;
#pragma unroll
            for (int s = 0; s < R; ++s)
            {
#pragma unroll
                for (int j = 0; j < N; ++j)
                    if (j < (s + 1) * L && j < done && row[s] < n && j <= row[s])
                        p[tri_index(lda, upper, row[s], j)] = r[s][j];
            }
        }
        if (in_batch && l == 0) info[q] = live ? failure : -3;
        __syncwarp();  // the stage is rewritten by the next group
    }
}

// SolveKernel with one lane per matrix.  The warp copies its 32 matrices' lower triangles
// into shared memory in a trapezoid layout: column j keeps rows 4 floor(j / 4) .. N - 1, so
// every column starts on a 16-byte boundary and is copied in 16-byte pieces (four-float
// pieces straddling the diagonal carry a few upper entries that are never read).  The
// per-matrix pitch is 4 modulo 32 floats, so the lanes' 16-byte reads of the same offset in
// different matrices touch different banks.  Lane m then solves matrix m with x in
// registers.  Per right-hand side: the forward sweep x_i = (b_i - sum_{j<i} L(i,j) x_j) /
// L(i,i) takes each x_j into every later row as soon as it is final, which is each row's
// fmaf chain over ascending j; the backward sweep x_i = (x_i - sum_{j>i} L(j,i) x_j) / L(i,i)
// (descending i) is each row's chain over ascending j (cholesky_simt.cpp:93-117).  Both
// read columns of L.
template <int N>
__host__ __device__ constexpr int trap_col(int j)
{
    // floats before column j: sum over earlier columns of N - 4 floor(c / 4)
    return j * N - 4 * ((j / 4) * ((j / 4) - 1) / 2 * 4 + (j / 4) * (j % 4));
}
template <int N>
__host__ __device__ constexpr int trap_size()
{
    return trap_col<N>(N);
}
template <int N>
__host__ __device__ constexpr int trap_pitch()
{
    return (trap_size<N>() + 31 - 4) / 32 * 32 + 4;  // >= size, 4 modulo 32
}
// element (i, j), i >= 4 floor(j / 4), of the trapezoid
template <int N>
__device__ __forceinline__ constexpr int trap_at(int i, int j)
{
    return trap_col<N>(j) + i - 4 * (j / 4);
}

template <int N>
__global__ void __launch_bounds__(32) potrs_lane_kernel(float *a_single, float *const *a_table, int a_first,
                                                        float *b_single, float *const *b_table, int b_first, int n,
                                                        int lda, int ldb, int nrhs, int upper, int count,
                                                        const int *info)
{
    constexpr int P = trap_pitch<N>();
    extern __shared__ __align__(16) float lane_mem[];
    if (info[0] != 0) return;
    const int lane = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x * 32;
    const int64_t q = base + lane;
    const float *mine = nullptr;
    if (q < count) mine = a_table ? slot(a_table, a_first + q) : a_single;
    // 16-byte copies when every column of every matrix starts 16-byte aligned (lower
    // storage, lda % 4 == 0, aligned bases); else element copies
    const bool vec = !upper && (lda & 3) == 0 && lda <= (1 << 25) &&
                     __all_sync(0xffffffffu, (reinterpret_cast<uintptr_t>(mine) & 15u) == 0);
    // The 16-byte pieces a lane copies are the same for every matrix of the warp (one n and
    // lda per call): column j holds pieces 4 floor(j / 4) .. n - 1 rounded up to 4 (inside
    // the column).  Offsets are taken once here; per matrix a lane then issues at most PPL
    // copies with one add each, so the warp streams its 32 triangles back to back.
    constexpr int PPL = (N * (N / 4) + 31) / 32;  // pieces per lane
    unsigned piece_dst[PPL];                      // byte offset in the matrix's trapezoid
    int piece_src[PPL];                           // float offset j * lda + r4 (< 2^31 / 4)
    int piece_bytes[PPL];                         // 0: nothing to copy
#pragma unroll
    for (int it = 0; it < PPL; ++it)
    {
        const int e = lane + 32 * it;
        const int j = e / (N / 4), r4 = (e % (N / 4)) * 4;
        const bool ok = e < N * (N / 4) && j < n && r4 >= 4 * (j / 4) && r4 < n;
        piece_dst[it] = ok ? (unsigned)(trap_at<N>(r4, j) * 4) : 0u;
        piece_src[it] = ok ? j * lda + r4 : 0;
        piece_bytes[it] = ok ? min(4, n - r4) * 4 : 0;
    }
    const unsigned mem0 = (unsigned)__cvta_generic_to_shared(lane_mem);
    for (int mm = 0; mm < 32; ++mm)
    {
        const float *pa =
            reinterpret_cast<const float *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(mine), mm));
        if (!pa) continue;  // uniform: one matrix at a time
        float *dst = lane_mem + mm * P;
        if (vec)
        {
            const unsigned d0 = mem0 + (unsigned)(mm * P * 4);
#pragma unroll
            for (int it = 0; it < PPL; ++it)
                if (piece_bytes[it])
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d0 + piece_dst[it]),
                                 "l"(pa + piece_src[it]), "r"(piece_bytes[it])
                                 : "memory");
        }
        else
        {
            for (int e = lane; e < N * N; e += 32)
            {
                const int j = e / N, i = e % N;
                if (j < n && i < n && i >= j)
                {
                    const unsigned d = (unsigned)__cvta_generic_to_shared(dst + trap_at<N>(i, j));
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d),
                                 "l"(pa + tri_index(lda, upper, i, j))
                                 : "memory");
                }
            }
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();
    float *pb = nullptr;
    if (q < count) pb = b_table ? slot(b_table, b_first + q) : b_single;
    if (!mine || !pb) return;
    const float *tri = lane_mem + lane * P;
    // x_i / L(i, i): the diagonal and its reciprocal are read and formed at the step (they do
    // not depend on x, so they are off the dependent chain)
    auto divide = [&](float v, int i) {
        const float d = tri[trap_at<N>(i, i)];
        return div_by(v, d, div_prepare(d), div_range(d));
    };
    for (int rhs = 0; rhs < nrhs; ++rhs)
    {
        float *xb = pb + (int64_t)rhs * ldb;
        float x[N];
#pragma unroll
        for (int i = 0; i < N; ++i) x[i] = i < n ? xb[i] : 0.0f;
        // forward, column by column
#pragma unroll
        for (int j = 0; j < N; ++j)
        {
            if (j < n)
            {
                x[j] = divide(x[j], j);
#pragma unroll
                for (int i4 = 4 * (j / 4); i4 < N; i4 += 4)
                {
                    const float4 l = *reinterpret_cast<const float4 *>(tri + trap_at<N>(i4, j));
                    if (i4 + 0 > j && i4 + 0 < n) x[i4 + 0] = fma_rn(-l.x, x[j], x[i4 + 0]);
                    if (i4 + 1 > j && i4 + 1 < n) x[i4 + 1] = fma_rn(-l.y, x[j], x[i4 + 1]);
                    if (i4 + 2 > j && i4 + 2 < n) x[i4 + 2] = fma_rn(-l.z, x[j], x[i4 + 2]);
                    if (i4 + 3 > j && i4 + 3 < n) x[i4 + 3] = fma_rn(-l.w, x[j], x[i4 + 3]);
                }
            }
        }
        // backward, a chain per row over ascending j > i
#pragma unroll
        for (int i = N - 1; i >= 0; --i)
        {
            if (i < n)
            {
                float acc = x[i];
#pragma unroll
                for (int j4 = 4 * (i / 4); j4 < N; j4 += 4)
                {
                    const float4 l = *reinterpret_cast<const float4 *>(tri + trap_at<N>(j4, i));
                    if (j4 + 0 > i && j4 + 0 < n) acc = fma_rn(-l.x, x[j4 + 0], acc);
                    if (j4 + 1 > i && j4 + 1 < n) acc = fma_rn(-l.y, x[j4 + 1], acc);
                    if (j4 + 2 > i && j4 + 2 < n) acc = fma_rn(-l.z, x[j4 + 2], acc);
                    if (j4 + 3 > i && j4 + 3 < n) acc = fma_rn(-l.w, x[j4 + 3], acc);
                }
                x[i] = divide(acc, i);
            }
        }
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i < n) xb[i] = x[i];
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

// Lanes per matrix of the grouped factorisation (rows per lane = order / lanes).
constexpr int POTRF_LANES_32 = 16;
constexpr int POTRF_LANES_16 = 8;

template <int N, int L>
cudaError_t potrf_group_n(const RealBatch &a, int upper, int *info, cudaStream_t stream)
{
    constexpr int MPW = 32 / L;
    int64_t warps = (a.count + MPW - 1) / MPW;
    int64_t blocks = (warps * 32 + THREADS - 1) / THREADS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    potrf_group_kernel<N, L><<<(unsigned)blocks, THREADS, 0, stream>>>(a.single, a.table, a.first, a.n, a.ld, upper,
                                                                       a.count, info);
    return cudaGetLastError();
}

template <int N>
cudaError_t potrs_lane_n(const RealBatch &a, const RealBatch &b, int nrhs, int upper, const int *info,
                         cudaStream_t stream)
{
    const size_t smem = (size_t)32 * trap_pitch<N>() * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(potrs_lane_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, (a.count + 31) / 32);
    potrs_lane_kernel<N><<<blocks, 32, smem, stream>>>(a.single, a.table, a.first, b.single, b.table, b.first, a.n,
                                                       a.ld, b.ld, nrhs, upper, a.count, info);
    return cudaGetLastError();
}

__global__ void fill_info_kernel(int *info, int value, int64_t count)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        info[i] = value;
}

// The pointer tables scanned by a grid; each block ORs what it found (1: a null A slot,
// 2: a null B slot) into flags[0] and counts itself in flags[1]; the last block to finish
// writes info[0] (-4 for a null A slot, else -6 for a null B slot, else 0) and clears both
// words for the next launch.
__global__ void __launch_bounds__(256) solve_slot_check_kernel(int *info, float *const *a, float *const *b, int count,
                                                               int *flags)
{
    __shared__ int block_mask;
    if (threadIdx.x == 0) block_mask = 0;
    __syncthreads();
    int mask = 0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
    {
        if (!slot(a, q)) mask |= 1;
        if (!slot(b, q)) mask |= 2;
    }
    mask = (int)__reduce_or_sync(0xffffffffu, (unsigned)mask);
    if ((threadIdx.x & 31) == 0 && mask) atomicOr(&block_mask, mask);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        if (block_mask) atomicOr(&flags[0], block_mask);
        __threadfence();
        if (atomicAdd(&flags[1], 1) == (int)gridDim.x - 1)
        {
            __threadfence();
            const int f = atomicOr(&flags[0], 0);
            info[0] = (f & 1) ? -4 : (f & 2) ? -6 : 0;
            flags[0] = 0;
            flags[1] = 0;
        }
    }
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

cudaError_t launch_solve_slot_check(int *info, float *const *a, float *const *b, int count, int *flags,
                                    cudaStream_t stream)
{
    int64_t blocks = (count + 255) / 256;
    if (blocks > 148) blocks = 148;
    if (blocks < 1) blocks = 1;
    solve_slot_check_kernel<<<(unsigned)blocks, 256, 0, stream>>>(info, a, b, count, flags);
    return cudaGetLastError();
}

cudaError_t launch_potrf_small(const RealBatch &a, int upper, int *info, cudaStream_t stream)
{
    if (a.n <= 8) return potrf_small_n<8, ORDER_SIMT>(a, upper, info, stream);
    if (a.n <= 16) return potrf_group_n<16, POTRF_LANES_16>(a, upper, info, stream);
    return potrf_group_n<32, POTRF_LANES_32>(a, upper, info, stream);
}

cudaError_t launch_potrs_small(const RealBatch &a, const RealBatch &b, int nrhs, int upper, const int *info,
                               cudaStream_t stream)
{
    if (a.count == 1) return potrs_small_n<8>(a, b, nrhs, upper, info, stream);  // one matrix (n <= 8): a sub-warp
    if (a.n <= 8) return potrs_lane_n<8>(a, b, nrhs, upper, info, stream);
    if (a.n <= 16) return potrs_lane_n<16>(a, b, nrhs, upper, info, stream);
    return potrs_lane_n<32>(a, b, nrhs, upper, info, stream);
}

}  // namespace ops_solver
