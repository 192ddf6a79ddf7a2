// Transcendental and half-precision helpers of the splat rasteriser, usable on
// the host and on the device with bit-identical results.
//
// The reference evaluates exp, log and pow through its shading language's
// library. Those are not reproducible bit for bit on a CPU, and bit-exact
// tile membership and sort keys need both sides to round alike, so this file
// defines its own functions from published methods, built only from
// correctly rounded operations (+ - * /, sqrt, fused multiply-add, rint):
//
//   lrt_exp  Cody & Waite argument reduction x = n ln2 + r, |r| <= ln2/2,
//            with ln 2 split into a float and its float remainder and the
//            reduction done by two fused multiply-adds; e^r by its Taylor
//            series to degree 7 in Horner form (truncation < 0.2 ulp); 2^n
//            applied through the exponent field in at most two exact steps
//            and one final rounding (which also yields subnormal results).
//   lrt_log  x = m 2^e with m in [sqrt(1/2), sqrt 2]; log m = 2 artanh(s),
//            s = (m - 1)/(m + 1), by the artanh series to s^11/11
//            (|s| <= 0.172); e ln 2 added with the split ln 2.
//   lrt_pow  exp(y log x) for x > 0.
//
// Measured against double-precision exp/log they are within 2 ulp (tests).
#pragma once

#include <cstdint>
#include <cstring>
#include <cmath>

#if defined(__CUDACC__)
#include <cuda_fp16.h>
#endif

#if defined(__CUDACC__)
#define LRT_HD __host__ __device__ __forceinline__
#else
#define LRT_HD inline
#endif

namespace lrt {

LRT_HD uint32_t float_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}

LRT_HD float bits_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}

LRT_HD float lrt_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

LRT_HD float lrt_rint(float x) {
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return std::rint(x);
#endif
}

LRT_HD float lrt_exp(float x) {
    if (x != x) return x;
    if (x > 89.0f) return INFINITY;
    if (x < -104.0f) return 0.0f;
    const float n = lrt_rint(x * 1.44269504088896340736f);
    float r = lrt_fma(-n, 0.693147182464599609375f, x);
    r = lrt_fma(-n, -1.904654299957768e-09f, r);
    float p = 1.984126984126984e-4f;
    p = lrt_fma(p, r, 1.388888888888889e-3f);
    p = lrt_fma(p, r, 8.333333333333333e-3f);
    p = lrt_fma(p, r, 4.166666666666666e-2f);
    p = lrt_fma(p, r, 1.666666666666667e-1f);
    p = lrt_fma(p, r, 0.5f);
    p = lrt_fma(p, r, 1.0f);
    p = lrt_fma(p, r, 1.0f);
    int e = static_cast<int>(n);
    if (e > 126) {
        p = p * bits_float(253u << 23);
        e -= 126;
    } else if (e < -125) {
        p = p * bits_float(2u << 23);
        e += 125;
    }
    return p * bits_float(static_cast<uint32_t>(e + 127) << 23);
}

// lrt_exp without its range checks, for -87 <= x <= 88 (where no check
// fires, so the result has the same bits); outside that range it returns an
// unspecified value. For hot loops whose argument is known to be in range.
// On the device n = rint(x log2 e) comes from adding 1.5 * 2^23 (the sum
// rounds to the nearest integer, ties to even, as rint does, for
// |x log2 e| < 2^22), and the sum's low bits are then n itself, so 2^n is one
// shift-add of those bits: no float -> int conversion. The bits are those of
// the form below.
LRT_HD float lrt_exp_in_range(float x) {
#if defined(__CUDA_ARCH__)
    constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23, bits 0x4B400000
    const float t = __fadd_rn(__fmul_rn(x, 1.44269504088896340736f), kMagic);
    const float n = __fsub_rn(t, kMagic);
    float r = __fmaf_rn(-n, 0.693147182464599609375f, x);
    r = __fmaf_rn(-n, -1.904654299957768e-09f, r);
    float p = 1.984126984126984e-4f;
    p = __fmaf_rn(p, r, 1.388888888888889e-3f);
    p = __fmaf_rn(p, r, 8.333333333333333e-3f);
    p = __fmaf_rn(p, r, 4.166666666666666e-2f);
    p = __fmaf_rn(p, r, 1.666666666666667e-1f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    // (bits(t) - 0x4B400000 + 127) << 23 = 2^n's bits, the subtraction folded
    // into the constant (mod 2^32).
    const uint32_t scale = (__float_as_uint(t) << 23) + ((127u - 0x4B400000u) << 23);
    return __fmul_rn(p, __uint_as_float(scale));
#else
    const float n = lrt_rint(x * 1.44269504088896340736f);
    float r = lrt_fma(-n, 0.693147182464599609375f, x);
    r = lrt_fma(-n, -1.904654299957768e-09f, r);
    float p = 1.984126984126984e-4f;
    p = lrt_fma(p, r, 1.388888888888889e-3f);
    p = lrt_fma(p, r, 8.333333333333333e-3f);
    p = lrt_fma(p, r, 4.166666666666666e-2f);
    p = lrt_fma(p, r, 1.666666666666667e-1f);
    p = lrt_fma(p, r, 0.5f);
    p = lrt_fma(p, r, 1.0f);
    p = lrt_fma(p, r, 1.0f);
    const int e = static_cast<int>(n);
    return p * bits_float(static_cast<uint32_t>(e + 127) << 23);
#endif
}

LRT_HD float lrt_log(float x) {
    if (x != x) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int e = 0;
    uint32_t u = float_bits(x);
    if (u < 0x00800000u) {
        x = x * 8388608.0f;
        u = float_bits(x);
        e = -23;
    }
    e += static_cast<int>(u >> 23) - 127;
    float m = bits_float((u & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = lrt_fma(z, 0.0909090909090909f, 0.1111111111111111f);
    p = lrt_fma(p, z, 0.1428571428571429f);
    p = lrt_fma(p, z, 0.2f);
    p = lrt_fma(p, z, 0.3333333333333333f);
    const float t = 2.0f * s;
    const float lm = lrt_fma(t * z, p, t);
    const float fe = static_cast<float>(e);
    return lrt_fma(fe, 0.693147182464599609375f, lrt_fma(fe, -1.904654299957768e-09f, lm));
}

LRT_HD float lrt_pow(float x, float y) { return lrt_exp(y * lrt_log(x)); }

// IEEE binary16 <-> binary32. Decoding is exact; encoding rounds to nearest,
// ties to even (what the reference's f32tof16 does on its devices).
LRT_HD float half_to_float(uint32_t h) {
#if defined(__CUDA_ARCH__)
    return __half2float(__ushort_as_half(static_cast<unsigned short>(h & 0xFFFFu)));
#else
    const uint32_t sign = (h >> 15) & 1u;
    const uint32_t ex = (h >> 10) & 0x1Fu;
    const uint32_t mant = h & 0x3FFu;
    float v;
    if (ex == 0) {
        v = static_cast<float>(mant) * 5.9604644775390625e-08f;
    } else if (ex == 31) {
        v = mant == 0 ? INFINITY : NAN;
    } else {
        v = bits_float(((ex - 15 + 127) << 23) | (mant << 13));
    }
    return sign ? -v : v;
#endif
}

LRT_HD uint32_t float_to_half(float f) {
    const uint32_t u = float_bits(f);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const uint32_t a = u & 0x7FFFFFFFu;
    if (a >= 0x7F800000u) return sign | (a > 0x7F800000u ? 0x7E00u : 0x7C00u);
#if defined(__CUDA_ARCH__)
    // The device's conversion instruction rounds to nearest even too
    // (overflow to infinity, subnormal results exact), so only NaN, whose
    // payload it would keep, takes the line above.
    return __half_as_ushort(__float2half_rn(f));
#else
    if (a >= 0x477FF000u) return sign | 0x7C00u;
    if (a < 0x38800000u) {
        const float v = bits_float(a) * 16777216.0f;
        return sign | static_cast<uint32_t>(lrt_rint(v));
    }
    const uint32_t mant = a & 0x7FFFFFu;
    uint32_t h = ((((a >> 23) - 127 + 15)) << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;
    return sign | h;
#endif
}

LRT_HD float low_half(uint32_t w) { return half_to_float(w & 0xFFFFu); }
LRT_HD float high_half(uint32_t w) { return half_to_float(w >> 16); }

}  // namespace lrt
