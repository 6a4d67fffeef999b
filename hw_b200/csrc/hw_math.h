// Scalar math shared bit-for-bit by the CUDA kernels and the CPU oracle.
//
// The reference host path evaluates exp/log through an SSE port of the
// Cephes single-precision routines (src/basecaller/common/simd/xcompile.h:148-152
// -> sse_mathfun.h) and converts float lanes to integers with the x86
// cvtps2dq instruction (common/simd/m512f_SSE.h:126-131, 515-537) followed by
// a plain C++ int32 -> int16 narrowing (common/simd/m512s_SSE.h:101-110).
//
// This header restates those semantics as portable scalar code:
//   * hw_expf / hw_logf follow S. L. Moshier's published Cephes expf/logf
//     method (Cody-Waite range reduction with the ln2 = 0.693359375 -
//     2.12194440e-4 split and the Cephes minimax polynomials).  The
//     polynomial steps are written as explicit fused multiply-adds so that a
//     host compiled with -ffp-contract=off and a device compiled with
//     -fmad=false produce identical bits.  Outside the normal range the
//     results are IEEE-like (0, denormal, inf) rather than clamped.
//   * cvt_rn_i32 mirrors cvtps2dq under round-to-nearest-even: NaN or an
//     out-of-range result yields INT32_MIN ("integer indefinite").
//   * to_i16_wrap narrows by taking the low 16 bits, as the reference does.
//   * f32_to_f16_bits rounds to nearest-even like CUDA's __float2half.
#pragma once

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#include <cuda_fp16.h>
#define HW_HD __host__ __device__ __forceinline__
#else
#define HW_HD static inline
#endif

namespace hwm {

HW_HD float bits_f32(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}

HW_HD uint32_t f32_bits(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}

HW_HD float fma_rn(float a, float b, float c)
{
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

HW_HD float mul_rn(float a, float b)
{
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}

HW_HD float add_rn(float a, float b)
{
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}

// 2^n as a float for n in [-126, 127].
HW_HD float pow2i(int n)
{
    return bits_f32((uint32_t)(n + 127) << 23);
}

// y * 2^n for n in [-252, 254], rounded once (two exact power-of-two factors).
HW_HD float scale2(float y, int n)
{
    const int n1 = n >> 1;
    const int n2 = n - n1;
    return mul_rn(mul_rn(y, pow2i(n1)), pow2i(n2));
}

// Natural exponential, Cephes expf method with fused polynomial steps.
// Written without branches: the special cases (NaN, overflow above
// 88.72283935546875, underflow to 0 below -103.97208404541016) are selected
// after an in-range evaluation, so that several independent calls can be
// interleaved by the compiler.
HW_HD float hw_expf(float x)
{
    const bool isNan = x != x;
    const bool hi = x > 88.72283935546875f;
    const bool lo = x < -103.97208404541016f;
    const float xc = (isNan | hi | lo) ? 0.0f : x;
    const float z = floorf(fma_rn(xc, 1.44269504088896341f, 0.5f));
    float r = fma_rn(z, -0.693359375f, xc);
    r = fma_rn(z, 2.12194440e-4f, r);
    float p = 1.9875691500e-4f;
    p = fma_rn(p, r, 1.3981999507e-3f);
    p = fma_rn(p, r, 8.3334519073e-3f);
    p = fma_rn(p, r, 4.1665795894e-2f);
    p = fma_rn(p, r, 1.6666665459e-1f);
    p = fma_rn(p, r, 5.0000001201e-1f);
    const float r2 = mul_rn(r, r);
    const float y = add_rn(fma_rn(p, r2, r), 1.0f);
    float out = scale2(y, (int)z);
    out = lo ? 0.0f : out;
    out = hi ? bits_f32(0x7f800000u) : out;
    return isNan ? x : out;
}

// Natural logarithm, Cephes logf method with fused polynomial steps.  Also
// branch-free: NaN -> NaN, x < 0 -> NaN, +-0 -> -inf, +inf -> +inf are
// selected after the evaluation; denormals are scaled by 2^32 first.
HW_HD float hw_logf(float x)
{
    const bool isNan = x != x;
    const bool neg = x < 0.0f;
    const bool zero = x == 0.0f;
    uint32_t u = f32_bits(x);
    const bool isInf = u == 0x7f800000u;
    const bool den = u < 0x00800000u;            // denormal (or +0): normalise by 2^32
    u = den ? f32_bits(mul_rn(x, 4294967296.0f)) : u;
    // frexp: x = m * 2^e with m in [0.5, 1)
    int e = (den ? -32 : 0) + (int)((u >> 23) & 0xffu) - 126;
    float m = bits_f32((u & 0x807fffffu) | 0x3f000000u);
    const bool small = m < 0.707106781186547524f;
    e -= small ? 1 : 0;
    m = small ? add_rn(add_rn(m, m), -1.0f) : add_rn(m, -1.0f);
    const float z = mul_rn(m, m);
    float y = 7.0376836292e-2f;
    y = fma_rn(y, m, -1.1514610310e-1f);
    y = fma_rn(y, m, 1.1676998740e-1f);
    y = fma_rn(y, m, -1.2420140846e-1f);
    y = fma_rn(y, m, 1.4249322787e-1f);
    y = fma_rn(y, m, -1.6668057665e-1f);
    y = fma_rn(y, m, 2.0000714765e-1f);
    y = fma_rn(y, m, -2.4999993993e-1f);
    y = fma_rn(y, m, 3.3333331174e-1f);
    y = mul_rn(mul_rn(y, m), z);
    const float fe = (float)e;
    y = fma_rn(fe, -2.12194440e-4f, y);
    y = fma_rn(z, -0.5f, y);
    float r = add_rn(m, y);
    r = fma_rn(fe, 0.693359375f, r);
    r = isInf ? x : r;
    r = zero ? bits_f32(0xff800000u) : r;
    r = neg ? bits_f32(0x7fc00000u) : r;
    return isNan ? x : r;
}

// x86 cvtps2dq under round-to-nearest-even.
HW_HD int32_t cvt_rn_i32(float x)
{
    const float r = rintf(x);
    if (!(r >= -2147483648.0f && r < 2147483648.0f)) return (int32_t)0x80000000u;
    return (int32_t)r;
}

// floorf followed by cvtps2dq (reference floorCastInt).
HW_HD int32_t floor_cast_i32(float x)
{
    const float r = floorf(x);
    if (!(r >= -2147483648.0f && r < 2147483648.0f)) return (int32_t)0x80000000u;
    return (int32_t)r;
}

// Reference float -> int16 lane conversion: round to int32 then keep low 16 bits.
HW_HD int16_t to_i16_wrap(float x)
{
    return (int16_t)(uint16_t)(uint32_t)cvt_rn_i32(x);
}

HW_HD int16_t i16_wrap(int32_t x)
{
    return (int16_t)(uint16_t)(uint32_t)x;
}

// IEEE binary16 round-to-nearest-even encode / exact decode.
HW_HD uint16_t f32_to_f16_bits(float f)
{
#if defined(__CUDA_ARCH__)
    return __half_as_ushort(__float2half_rn(f));
#else
    const uint32_t u = f32_bits(f);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const uint32_t absu = u & 0x7fffffffu;
    if (absu >= 0x7f800000u)                     // inf or nan
        return (uint16_t)(sign | 0x7c00u | (absu > 0x7f800000u ? 0x200u | ((absu >> 13) & 0x3ffu) : 0u));
    if (absu >= 0x477ff000u)                     // rounds to >= 65520 -> inf
        return (uint16_t)(sign | 0x7c00u);
    if (absu < 0x38800000u)                      // result is subnormal or zero
    {
        if (absu < 0x33000000u) return (uint16_t)sign;   // < 2^-25 -> 0
        const uint32_t e = absu >> 23;
        const uint32_t mant = (absu & 0x7fffffu) | 0x800000u;
        const uint32_t shift = 126u - e;                 // 14..24
        uint32_t q = mant >> shift;
        const uint32_t rem = mant & ((1u << shift) - 1u);
        const uint32_t half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (q & 1u))) ++q;
        return (uint16_t)(sign | q);
    }
    uint32_t q = ((absu - 0x38000000u) >> 13);
    const uint32_t rem = absu & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) ++q;
    return (uint16_t)(sign | q);
#endif
}

HW_HD float f16_bits_to_f32(uint16_t h)
{
#if defined(__CUDA_ARCH__)
    return __half2float(__ushort_as_half(h));
#else
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1fu;
    uint32_t m = h & 0x3ffu;
    if (e == 0)
    {
        if (m == 0) return bits_f32(sign);
        int sh = 0;
        while (!(m & 0x400u)) { m <<= 1; ++sh; }
        m &= 0x3ffu;
        return bits_f32(sign | ((uint32_t)(113 - sh) << 23) | (m << 13));
    }
    if (e == 31) return bits_f32(sign | 0x7f800000u | (m << 13));
    return bits_f32(sign | ((e + 112u) << 23) | (m << 13));
#endif
}

// float -> half -> float (the precision the detection model is stored in).
HW_HD float round_f16(float f)
{
    return f16_bits_to_f32(f32_to_f16_bits(f));
}

// Lane-array min/max follow _mm_max_ps/_mm_min_ps: the first operand wins
// only on a strict comparison (common/simd/m512f_SSE.h:370-384), so a NaN in
// either operand yields the second operand.
HW_HD float fmax_sse(float l, float r) { return (l > r) ? l : r; }
HW_HD float fmin_sse(float l, float r) { return (l < r) ? l : r; }
// Scalar std::max / std::min.
HW_HD float fmax_std(float a, float b) { return (a < b) ? b : a; }
HW_HD float fmin_std(float a, float b) { return (b < a) ? b : a; }

// NumericUtil.h:70 satlin, on lane arrays (SSE min/max semantics).
HW_HD float satlin_sse(float a, float b, float x)
{
    const float r = (x - a) / (b - a);
    return fmin_sse(fmax_sse(r, 0.0f), 1.0f);
}

// NumericUtil.h:70 satlin, on scalars (std::min/std::max semantics).
HW_HD float satlin_std(float a, float b, float x)
{
    const float r = (x - a) / (b - a);
    return fmin_std(fmax_std(r, 0.0f), 1.0f);
}

}   // namespace hwm
