// selftest.cu -- device checks of arithmetic helpers that the parity contract rests on,
// callable from the tests (not part of the aclsolver interface).
#include "common.cuh"

namespace ops_solver
{
namespace
{
__global__ void divide_kernel(const float *x, const float *d, float *q, int64_t count)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    {
        const float dv = d[i];
        q[i] = div_by(x[i], dv, div_prepare(dv), div_range(dv));
    }
}
}  // namespace
}  // namespace ops_solver

// q[i] = div_by(x[i], d[i]) for device arrays of count floats, on the default stream; 0 or a
// CUDA error code.
extern "C" __attribute__((visibility("default"))) int ops_solver_selftest_divide(const float *x, const float *d,
                                                                                  float *q, long long count)
{
    if (count <= 0) return 0;
    long long blocks = (count + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    ops_solver::divide_kernel<<<(unsigned)blocks, 256>>>(x, d, q, count);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}
