// potri.cu -- the inverse from a Cholesky factor, A^-1 = (L L^T)^-1 or (L L^H)^-1, in place
// (aclsolverSpotri, aclsolverCpotri).
//
// The reference forms it as a Cholesky solve against the identity and stores the selected
// triangle of the result (src/cholesky/arch35/cholesky_simt.cpp:220-254: IdentityKernel,
// the solve, InverseStoreKernel; the complex family likewise through its solve,
// src/cpotri/arch35/cpotri.cpp with src/cpotrf/arch35/cpotrf.cpp:16-60).  This build does the
// same with its own solves, so the inverse carries exactly the arithmetic of aclsolverSpotrs /
// aclsolverCpotrs on the identity:
//   prepare: one thread scans the factor's diagonal (real: d > 0 and finite; complex: real
//            part > 0, imaginary part 0, both finite) and sets info to the first failing
//            index + 1, or 0; the grid writes the identity into the n x n workspace;
//   solve:   the library's single-matrix solve on the workspace, skipped when info != 0;
//   store:   when info == 0, the workspace's lower triangle (the inverse is symmetric /
//            Hermitian) goes to the selected triangle of A; a failed factor is left unchanged.
#include "common.cuh"
#include "launch.h"

namespace ops_solver
{
namespace
{
__device__ __forceinline__ bool diagonal_ok(float d) { return d > 0.0f && isfinite(d); }
__device__ __forceinline__ bool diagonal_ok(float2 d) { return d.x > 0.0f && isfinite(d.x) && d.y == 0.0f; }
__device__ __forceinline__ float unit(float) { return 1.0f; }
__device__ __forceinline__ float2 unit(float2) { return make_float2(1.0f, 0.0f); }
__device__ __forceinline__ float nil(float) { return 0.0f; }
__device__ __forceinline__ float2 nil(float2) { return make_float2(0.0f, 0.0f); }
// the value stored at (j, i), j <= i, of the upper triangle from the lower one at (i, j)
__device__ __forceinline__ float mirror(float v) { return v; }
__device__ __forceinline__ float2 mirror(float2 v) { return make_float2(v.x, -v.y); }

template <typename T>
__global__ void __launch_bounds__(256) potri_prepare_kernel(const T *a, int lda, int n, T *w, int *info)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        int first = 0;
        for (int i = 0; i < n; ++i)
            if (!diagonal_ok(a[(int64_t)i * lda + i]))
            {
                first = i + 1;
                break;
            }
        info[0] = first;
    }
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        w[e] = i == j ? unit(T()) : nil(T());
    }
}

template <typename T>
__global__ void __launch_bounds__(256) potri_store_kernel(T *a, int lda, int upper, int n, const T *w, const int *info)
{
    if (info[0] != 0) return;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e % n), j = (int)(e / n);
        if (j > i) continue;
        const T v = w[(int64_t)j * n + i];
        if (upper)
            a[(int64_t)i * lda + j] = mirror(v);
        else
            a[(int64_t)j * lda + i] = v;
    }
}

unsigned grid_for(int n)
{
    const int64_t e = (int64_t)n * n;
    int64_t blocks = (e + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    return (unsigned)(blocks < 1 ? 1 : blocks);
}
}  // namespace

cudaError_t launch_potri_prepare(const float *a, int lda, int n, float *w, int *info, cudaStream_t stream)
{
    potri_prepare_kernel<float><<<grid_for(n), 256, 0, stream>>>(a, lda, n, w, info);
    return cudaGetLastError();
}
cudaError_t launch_potri_store(float *a, int lda, int upper, int n, const float *w, const int *info,
                               cudaStream_t stream)
{
    potri_store_kernel<float><<<grid_for(n), 256, 0, stream>>>(a, lda, upper, n, w, info);
    return cudaGetLastError();
}
cudaError_t launch_cpotri_prepare(const float2 *a, int lda, int n, float2 *w, int *info, cudaStream_t stream)
{
    potri_prepare_kernel<float2><<<grid_for(n), 256, 0, stream>>>(a, lda, n, w, info);
    return cudaGetLastError();
}
cudaError_t launch_cpotri_store(float2 *a, int lda, int upper, int n, const float2 *w, const int *info,
                                cudaStream_t stream)
{
    potri_store_kernel<float2><<<grid_for(n), 256, 0, stream>>>(a, lda, upper, n, w, info);
    return cudaGetLastError();
}

}  // namespace ops_solver
