// common.cuh -- device helpers shared by the sm_100a factor-and-solve kernels.
//
// All arithmetic on the plain (FP32) path goes through the explicitly rounded intrinsics
// below so that the compiler can neither contract a multiply and an add into an FMA nor
// split an FMA: the parity contract is bit-for-bit equality with the reference's
// per-element operation order.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ops_solver
{

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float sqrt_rn(float a) { return __fsqrt_rn(a); }
// fma_rn(a, b, c) = a*b + c with one rounding.
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// x / d rounded to nearest even when the reciprocal y = RN(1/d) is at hand (a divisor known
// ahead of a dependent chain): q = RN(x y), then two remainder corrections r = x - d q (one
// FMA), q = RN(q + r y).  After the first, q lies within one ulp of x / d; with y within half
// an ulp of 1/d, Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990; the
// handbook form: Muller et al., Handbook of Floating-Point Arithmetic, the division
// correction theorem) makes the second exactly RN(x / d), provided nothing overflows or
// underflows: d_ok (|d| in [2^-60, 2^60], from div_prepare) and |x| in the same range keep
// every intermediate a normal number.  Other operands (zeros, subnormals, infinities, NaN,
// extreme exponents) take the IEEE division.  Tested against IEEE division in the tests.
__device__ __forceinline__ bool div_range(float v)
{
    const float a = fabsf(v);
    return a >= 0x1p-60f && a <= 0x1p60f;
}
__device__ __forceinline__ float div_prepare(float d) { return __frcp_rn(d); }
__device__ __forceinline__ float div_by(float x, float d, float y, bool d_ok)
{
    if (!d_ok || !div_range(x)) return __fdiv_rn(x, d);
    float q = __fmul_rn(x, y);
    float r = __fmaf_rn(-q, d, x);
    q = __fmaf_rn(r, y, q);
    r = __fmaf_rn(-q, d, x);
    return __fmaf_rn(r, y, q);
}

// Two FP32 lanes in one 64-bit register pair (sm_100 paired FP32 arithmetic): each lane of
// fma2 is an IEEE fma rounded to nearest, i.e. exactly fma_rn on that lane.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi)
{
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float f2_lo(f32x2 v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float f2_hi(f32x2 v) { return __uint_as_float((unsigned)(v >> 32)); }
// d = a * b + d, lane by lane
__device__ __forceinline__ void fma2(f32x2 &d, f32x2 a, f32x2 b)
{
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}

// Copy a rows x cols column-major tile (element (i, k) at src[k * lds + i]) into shared
// memory at dst[k * ldd + i], every thread of the block taking part.  vec: 16-byte cp.async
// (src and dst 16-byte aligned per column, rows, lds and ldd multiples of 4); otherwise
// eight plain loads in flight per thread before their stores.  Entries past rows / cols are
// not written.  Callers wait with tile_wait() and a block barrier.
__device__ __forceinline__ void stage_tile(float *dst, int ldd, const float *src, int64_t lds, int rows, int cols,
                                           bool vec)
{
    const int nt = blockDim.x, t = threadIdx.x;
    if (vec)
    {
        const int per = rows / 4;
        for (int e = t; e < per * cols; e += nt)
        {
            const int k = e / per, i = (e % per) * 4;
            const unsigned d = (unsigned)__cvta_generic_to_shared(dst + k * ldd + i);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src + k * lds + i) : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    else
    {
        const int total = rows * cols;
        for (int e0 = t; e0 < total; e0 += nt * 8)
        {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
            {
                const int e = e0 + u * nt;
                v[u] = e < total ? src[(e / rows) * lds + e % rows] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
            {
                const int e = e0 + u * nt;
                if (e < total) dst[(e / rows) * ldd + e % rows] = v[u];
            }
        }
    }
}
__device__ __forceinline__ void tile_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Matrix slot b of a device pointer table.  Loaded through the read-only path: the
// tables are never written by a kernel.
template <typename T>
__device__ __forceinline__ T *slot(T *const *table, int64_t b)
{
    return reinterpret_cast<T *>(__ldg(reinterpret_cast<const unsigned long long *>(table) + b));
}

// Pivot-search key: larger |a| wins, NaN never wins (key 0); ties are broken separately
// by the smallest row position.  Non-negative float bit patterns order like the values.
__device__ __forceinline__ unsigned pivot_key(float v)
{
    float m = fabsf(v);
    return m == m ? __float_as_uint(m) + 1u : 0u;
}

}  // namespace ops_solver
