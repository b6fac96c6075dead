// complex_lu.cuh -- element arithmetic of the complex64 LU family, written with explicit
// round-to-nearest intrinsics so that no multiply-add is contracted and every kernel gives
// the same bits as the reference's SIMT helpers (paths relative to the reference root):
//   cscore          src/utils/complex_solver_kernel.hpp:48-67    PivotScore
//   csubmul         :69-72                                        SubMul
//   cquotient       :74-86                                        Quotient
//   cscaled_quot    :88-106                                       ScaledQuotient
//   cneeds_scaled   :108-117                                      NeedsScaledNumerator
//   cdivide         :119-143                                      Divide
//   ccomp_submul    src/utils/complex_solver_resident.hpp:21-43   CompensatedSubtract / SubMul
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace ops_solver
{
namespace clu
{
constexpr float FMAX = 3.402823466e38f;

// Abs keeps the sign of a negative zero, as the reference's x < 0 ? -x : x does.
__device__ __forceinline__ float cabs1(float x) { return x < 0.0f ? -x : x; }

__device__ __forceinline__ bool czero(float2 v) { return v.x == 0.0f && v.y == 0.0f; }

// L1 magnitude as an ordered key: NaN 0, zero 1, an overflowing sum halved with its
// exponent extended by one bit.
__device__ __forceinline__ uint32_t cscore(float2 v)
{
    float re = cabs1(v.x), im = cabs1(v.y);
    float s = add_rn(re, im);
    if (!(s >= 0.0f)) return 0u;
    if (s == 0.0f) return 1u;
    if (s > FMAX) return __float_as_uint(add_rn(mul_rn(re, 0.5f), mul_rn(im, 0.5f))) + 0x00800001u;
    return __float_as_uint(s) + 1u;
}

// x - a*b: real fma(a.im, b.im, fma(-a.re, b.re, x.re)), imag fma(-a.im, b.re, fma(-a.re, b.im, x.im)).
__device__ __forceinline__ float2 csubmul(float2 x, float2 a, float2 b)
{
    return make_float2(fma_rn(a.y, b.y, fma_rn(-a.x, b.x, x.x)), fma_rn(-a.y, b.x, fma_rn(-a.x, b.y, x.y)));
}

// Quotient with the divisor's reciprocal 1/den supplied (the same IEEE value the reference
// computes inline; PreparedQuotient, complex_solver_register.hpp:203-214, passes it in too).
__device__ __forceinline__ float cquotient(float ar, float br, float ai, float bi, float den, float den_err,
                                           float reciprocal)
{
    float product = mul_rn(ar, br);
    float other = mul_rn(ai, bi);
    float numerator = add_rn(product, other);
    float part = sub_rn(numerator, product);
    float error = add_rn(add_rn(add_rn(sub_rn(product, sub_rn(numerator, part)), sub_rn(other, part)),
                                fma_rn(ar, br, -product)),
                         fma_rn(ai, bi, -other));
    float result = mul_rn(numerator, reciprocal);
    float remainder = sub_rn(add_rn(fma_rn(-result, den, numerator), error), mul_rn(result, den_err));
    return fma_rn(remainder, reciprocal, result);
}

static __device__ __noinline__ float cscaled_quot(float a, float b, float c, float d, float scale, float den, float den_err)
{
    int ae, be, ce, de, se;
    float am = frexpf(a, &ae), bm = frexpf(b, &be);
    float cm = frexpf(c, &ce), dm = frexpf(d, &de);
    float sm = frexpf(scale, &se);
    int ab = ae + be, cd = ce + de;
    bool zab = a == 0.0f || b == 0.0f, zcd = c == 0.0f || d == 0.0f;
    int e = zab ? cd : zcd ? ab : (ab > cd ? ab : cd);
    am = zab ? 0.0f : ldexpf(am, ab - e);
    cm = zcd ? 0.0f : ldexpf(cm, cd - e);
    float q = cquotient(am, bm, cm, dm, den, den_err, div_rn(1.0f, den));
    return ldexpf(div_rn(q, mul_rn(sm, sm)), e - 2 * se);
}

// The divisor's half of Divide, shared by every numerator divided by the same value
// (the reference's PrepareDivisor computes exactly these terms, complex_solver_register.hpp:183-201).
// inv_s = 1/s when s is a normal power of two, so x * inv_s is the correctly rounded x / s
// (both round the same exact value once); 0 when s must be divided by.  divisor_tiny and
// divisor_ok fold the numerator-independent terms of NeedsScaledNumerator.
struct Divisor
{
    float2 b;
    float s, br, bi, den, err, rcp, inv_s;
    bool divisor_ok, divisor_tiny;
};

__device__ __forceinline__ bool cneeds_scaled(float2 a, const Divisor &d, float ar, float ai)
{
    return cabs1(a.x) <= FMAX && cabs1(a.y) <= FMAX && d.divisor_ok &&
           (cabs1(ar) > 0x1p120f || cabs1(ai) > 0x1p120f || (a.x != 0.0f && cabs1(ar) < 0x1p-100f) ||
            (a.y != 0.0f && cabs1(ai) < 0x1p-100f) || d.divisor_tiny);
}

__device__ __forceinline__ Divisor cprepare(float2 b)
{
    Divisor d;
    d.b = b;
    float s = cabs1(b.x) > cabs1(b.y) ? cabs1(b.x) : cabs1(b.y);
    uint32_t ex = __float_as_uint(s) & 0x7f800000u;
    if (ex != 0) s = __uint_as_float(ex);
    d.s = s;
    d.br = div_rn(b.x, s);
    d.bi = div_rn(b.y, s);
    float first = cabs1(d.br) > cabs1(d.bi) ? d.br : d.bi;
    float second = cabs1(d.br) > cabs1(d.bi) ? d.bi : d.br;
    float square = mul_rn(first, first);
    d.den = fma_rn(second, second, square);
    d.err = add_rn(fma_rn(first, first, -square), fma_rn(second, second, sub_rn(square, d.den)));
    d.rcp = div_rn(1.0f, d.den);
    d.inv_s = ex != 0 && ex <= 0x7e800000u ? __uint_as_float(0x7f000000u - ex) : 0.0f;  // 2^-e for s = 2^e <= 2^126
    d.divisor_ok = s > 0.0f && s <= FMAX;
    d.divisor_tiny = (b.x != 0.0f && cabs1(d.br) < 0x1p-100f) || (b.y != 0.0f && cabs1(d.bi) < 0x1p-100f);
    return d;
}

__device__ __forceinline__ float2 cdivide(float2 a, const Divisor &d)
{
    float ar, ai;
    if (d.inv_s != 0.0f)
    {
        ar = mul_rn(a.x, d.inv_s);
        ai = mul_rn(a.y, d.inv_s);
    }
    else
    {
        ar = div_rn(a.x, d.s);
        ai = div_rn(a.y, d.s);
    }
    if (cneeds_scaled(a, d, ar, ai))
        return make_float2(cscaled_quot(a.x, d.b.x, a.y, d.b.y, d.s, d.den, d.err),
                           cscaled_quot(a.y, d.b.x, -a.x, d.b.y, d.s, d.den, d.err));
    return make_float2(cquotient(ar, d.br, ai, d.bi, d.den, d.err, d.rcp),
                       cquotient(ai, d.br, -ar, d.bi, d.den, d.err, d.rcp));
}

__device__ __forceinline__ float2 cdivide(float2 a, float2 b) { return cdivide(a, cprepare(b)); }

// value - left*right with the rounding error carried into corr.
__device__ __forceinline__ float ccomp_sub(float value, float &corr, float left, float right)
{
    float product = mul_rn(left, right);
    float product_err = fma_rn(left, right, -product);
    float result = sub_rn(value, product);
    float virt = sub_rn(result, value);
    float sum_err = sub_rn(sub_rn(value, sub_rn(result, virt)), add_rn(product, virt));
    corr = add_rn(corr, sub_rn(sum_err, product_err));
    return result;
}

__device__ __forceinline__ void ccomp_submul(float2 &v, float2 &corr, float2 f, float2 s)
{
    v.x = ccomp_sub(v.x, corr.x, f.x, s.x);
    v.x = ccomp_sub(v.x, corr.x, -f.y, s.y);
    v.y = ccomp_sub(v.y, corr.y, f.y, s.x);
    v.y = ccomp_sub(v.y, corr.y, f.x, s.y);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(add_rn(a.x, b.x), add_rn(a.y, b.y)); }
}  // namespace clu
}  // namespace ops_solver
