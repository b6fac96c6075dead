// lu_util.cu -- validation and staging kernels of the real LU family.
//
// launch_finite_scan is the device half of the reference's synchronous finite-value
// check (real_lu_finite_kernel, src/sgetrf/sgetrf_kernel.cpp:98-143): it only reads the
// matrices and raises a flag word; the host reads the flag back and turns it into
// INVALID_VALUE, as CheckFinite (src/utils/real_lu_common.h:90-132) does.
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
__global__ void finite_scan_kernel(float *single, float *const *table, int first, int m, int n, int lda,
                                   int64_t count, int *flag)
{
    // One (matrix, column) job per warp-row of the grid; lanes stride down the column.
    const int64_t jobs = count * n;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    bool bad = false;
    for (int64_t job = warp; job < jobs; job += warps)
    {
        const int64_t q = job / n;
        const int j = (int)(job % n);
        const float *p = table ? slot(table, first + q) : single + q * (int64_t)lda * n;
        if (!p) continue;
        const float *c = p + (int64_t)j * lda;
        for (int i = lane; i < m; i += 32)
        {
            const float v = c[i];
            if (!(fabsf(v) <= 3.402823466e38F)) bad = true;
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flag, 1);
}

__global__ void copy_matrices_kernel(float *s_single, float *const *s_table, int s_first, int lds, float *d_single,
                                     float *const *d_table, int d_first, int ldd, int m, int n, int64_t count)
{
    const int64_t jobs = count * n;
    for (int64_t job = blockIdx.x; job < jobs; job += gridDim.x)
    {
        const int64_t q = job / n;
        const int j = (int)(job % n);
        const float *s = s_table ? slot(s_table, s_first + q) : s_single + q * (int64_t)lds * n;
        float *d = d_table ? slot(d_table, d_first + q) : d_single + q * (int64_t)ldd * n;
        if (!s || !d) continue;
        for (int i = threadIdx.x; i < m; i += blockDim.x) d[i + (int64_t)j * ldd] = s[i + (int64_t)j * lds];
    }
}

__global__ void transpose_kernel(const float *src, int lds, float *dst, int ldd, int rows, int cols)
{
    __shared__ float tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y)
    {
        const int i = bx + threadIdx.x, j = by + r;
        if (i < rows && j < cols) tile[r][threadIdx.x] = src[i + (int64_t)j * lds];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y)
    {
        const int i = by + threadIdx.x, j = bx + r;  // dst(i, j) = src(j, i)
        if (i < cols && j < rows) dst[i + (int64_t)j * ldd] = tile[threadIdx.x][r];
    }
}
__global__ void strided_table_kernel(float **table, float *base, int64_t stride, int count)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x)
        table[q] = base + (int64_t)q * stride;
}
}  // namespace

cudaError_t launch_strided_table(float **table, float *base, int64_t stride, int count, cudaStream_t stream)
{
    int blocks = (count + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    strided_table_kernel<<<blocks, 256, 0, stream>>>(table, base, stride, count);
    return cudaGetLastError();
}

cudaError_t launch_finite_scan(const RealBatch &a, int m, int *flag, cudaStream_t stream)
{
    int64_t jobs = (int64_t)a.count * a.n;
    int64_t blocks = (jobs * 32 + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    finite_scan_kernel<<<(unsigned)blocks, 256, 0, stream>>>(a.single, a.table, a.first, m, a.n, a.ld, a.count, flag);
    return cudaGetLastError();
}

cudaError_t launch_copy_matrices(const RealBatch &src, const RealBatch &dst, int m, cudaStream_t stream)
{
    int64_t jobs = (int64_t)src.count * src.n;
    int64_t blocks = jobs < 148 * 32 ? jobs : 148 * 32;
    if (blocks < 1) blocks = 1;
    int threads = m >= 128 ? 128 : (m >= 64 ? 64 : 32);
    copy_matrices_kernel<<<(unsigned)blocks, threads, 0, stream>>>(src.single, src.table, src.first, src.ld,
                                                                   dst.single, dst.table, dst.first, dst.ld, m,
                                                                   src.n, src.count);
    return cudaGetLastError();
}

cudaError_t launch_transpose(const float *src, int lds, float *dst, int ldd, int rows, int cols, cudaStream_t stream)
{
    dim3 grid((rows + 31) / 32, (cols + 31) / 32);
    transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(src, lds, dst, ldd, rows, cols);
    return cudaGetLastError();
}

}  // namespace ops_solver

namespace ops_solver
{
namespace
{
// Per matrix: info for the inverse above the small orders, in the small path's convention
// (-2 a null A or C slot, -4 a pivot outside [k+1, n], else the first zero diagonal of U,
// 1-based, else 0); C set to the identity where the inverse is computed; fail[q] = info != 0.
__global__ void getri_prepare_kernel(float *a_single, float *const *a_table, const int *ipiv, float *c_single,
                                     float *const *c_table, int n, int lda, int ldc, int count, int *info, int *fail)
{
    __shared__ int bad, zero;
    const int64_t q = blockIdx.x;
    if (q >= count) return;
    const float *A = a_table ? slot(a_table, q) : a_single;
    float *C = c_table ? slot(c_table, q) : c_single;
    if (threadIdx.x == 0)
    {
        bad = 0;
        zero = 0x7fffffff;
    }
    __syncthreads();
    if (A && C)
        for (int k = threadIdx.x; k < n; k += blockDim.x)
        {
            if (ipiv && (ipiv[q * n + k] < k + 1 || ipiv[q * n + k] > n)) bad = 1;
            if (A[(int64_t)k * lda + k] == 0.0f) atomicMin(&zero, k + 1);
        }
    __syncthreads();
    const int v = !(A && C) ? -2 : bad ? -4 : (zero == 0x7fffffff ? 0 : zero);
    if (threadIdx.x == 0)
    {
        info[q] = v;
        fail[q] = v != 0;
    }
    if (v != 0) return;  // uniform
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        C[(int64_t)j * ldc + i] = i == j ? 1.0f : 0.0f;
    }
}

// skip[q * n + r] = fail[q]: the solve's per right-hand side switch
__global__ void getri_skip_kernel(const int *fail, int n, int count, int *skip)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)count * n) return;
    skip[e] = fail[e / n];
}
}  // namespace

cudaError_t launch_getri_blocked(const RealBatch &a, const int *ipiv, const RealBatch &c, int *info, void *scratch,
                                 cudaStream_t stream)
{
    const int n = a.n, count = a.count;
    int *fail = static_cast<int *>(scratch);
    int *skip = fail + count;
    getri_prepare_kernel<<<count, 256, 0, stream>>>(a.single, a.table, ipiv, c.single, c.table, n, a.ld, c.ld, count,
                                                    info, fail);
    const int64_t total = (int64_t)count * n;
    getri_skip_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(fail, n, count, skip);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // C = A^-1 as the solve of A X = I, the identity already in C
    return launch_getrs_blocked(a, ipiv, nullptr, c, n, nullptr, skip, stream);
}

size_t getri_blocked_scratch_bytes(int n, int count) { return ((size_t)count * (n + 1)) * sizeof(int) + 256; }

}  // namespace ops_solver
