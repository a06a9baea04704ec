// fixed_point.cuh -- exact, order-independent sums of FP32 values as 64-bit integer limbs.
//
// A finite x with |x| < 2^62 is trunc(|x| 2^64) split into three limbs, each signed like x: bits
// [0, 32), bits [32, 64) and the integer part. Limb sums are plain integer additions (atomics
// included), so they commute; the 32-bit chunks leave 2^31 additions of headroom. Used for the
// path nodes' radiance and the sum of the per-pixel errors.
#pragma once

#include <cstdint>

namespace nrrs {

constexpr float kFixedMax = 4611686018427387904.0f;  // 2^62: larger values are refused

// trunc(|x| 2^64) as three limbs signed like x; x finite with |x| < 2^62
__device__ __forceinline__ void fixed_limbs(float x, long long l[3]) {
    const unsigned bits = __float_as_uint(x);
    const unsigned e = (bits >> 23) & 0xffu;
    const unsigned long long m = (bits & 0x7fffffu) | (e ? 0x800000u : 0u);
    const int sh = (int)(e ? e : 1u) - 150 + 64;  // |x| 2^64 = m 2^sh
    unsigned __int128 X;
    if (sh >= 0) X = (unsigned __int128)m << sh;
    else X = (-sh) >= 24 ? (unsigned __int128)0 : (unsigned __int128)(m >> (-sh));
    const unsigned long long lo = (unsigned long long)X;
    long long l0 = (long long)(lo & 0xffffffffull);
    long long l1 = (long long)(lo >> 32);
    long long l2 = (long long)(unsigned long long)(X >> 64);
    if (bits >> 31) { l0 = -l0; l1 = -l1; l2 = -l2; }
    l[0] = l0; l[1] = l1; l[2] = l2;
}

// (l0 + l1 2^32 + l2 2^64) 2^-64 rounded to the nearest float, ties to even. The magnitude M
// (< 2^127) is cut to its top 64 bits with the bits below folded into bit 0 (sticky); the
// hardware's correctly rounded u64 -> f32 conversion then rounds exactly as M itself would
// round (the folded bit lies 39 places below the rounding position), and the power-of-two
// scale is exact.
__device__ __forceinline__ float fixed_to_float(long long l0, long long l1, long long l2) {
    using u128 = unsigned __int128;
    const u128 U = ((u128)(__int128)l2 << 64) + ((u128)(__int128)l1 << 32) + (u128)(__int128)l0;
    const unsigned neg = (unsigned)(U >> 127) & 1u;
    const u128 mag = neg ? (u128)0 - U : U;
    const unsigned long long hi = (unsigned long long)(mag >> 64), lo = (unsigned long long)mag;
    float f;
    if (hi == 0) {
        f = __fmul_rn(__ull2float_rn(lo), 0x1p-64f);
    } else {
        const int sh = 64 - __clzll((long long)hi);  // bits of hi: 1..63
        const unsigned long long top = (hi << (64 - sh)) | (lo >> sh) |
                                       ((lo << (64 - sh)) != 0ull ? 1ull : 0ull);
        f = __fmul_rn(__ull2float_rn(top), __uint_as_float((unsigned)(127 + sh - 64) << 23));
    }
    return neg ? -f : f;
}

__device__ __forceinline__ bool fixed_ok(float x) { return fabsf(x) < kFixedMax; }

}  // namespace nrrs
