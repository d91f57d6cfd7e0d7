// les_fix.h -- exact, order-independent global sums (host and device).
//
// The reference sums rhsav, pav and the SOR residual sequentially in FP32
// (press.f95:128-138, 151-160, 186-197), an order no parallel reduction can
// reproduce.  Every global sum here instead converts each FP32 term exactly
// to a signed Q63.64 fixed-point integer (truncating toward zero below
// 2^-64) and adds the integers exactly in 128 bits.  The total does not
// depend on the summation order, so any reduction tree (warp shuffles,
// blocks, a final pass) gives the same bits.  The total T is finished in
// FP64 as ((double)hi * 2^64 + (double)lo) * 2^-64 with hi = T >> 64
// (signed) and lo = T mod 2^64.  A term that is not finite, or has
// |x| >= 2^62, marks the sum bad (the finished value is NaN).
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define LES_HD __host__ __device__ __forceinline__
#else
#define LES_HD inline
#endif

namespace les {

typedef __int128 i128;

struct FixPart {
    unsigned long long lo;
    long long hi;
    int bad;
    int pad;
};

LES_HD i128 fix_term(float x, int &bad) {
#if defined(__CUDA_ARCH__)
    // The same integer without a variable 128-bit shift: |x| = t + f with
    // t = trunc(|x|) and f = |x| - t, both exact in FP32, so
    // trunc(|x| * 2^64) = t * 2^64 + trunc(f * 2^64), each part one
    // truncating conversion (f * 2^64 is a power-of-two scaling, exact).
    const float a = fabsf(x);
    if (!(a < 4.611686018427388e18f)) {  // NaN, inf or >= 2^62
        bad = 1;
        return 0;
    }
    unsigned long long ip = 0ull, fr;
    if (a < 1.0f) {
        fr = __float2ull_rz(a * 18446744073709551616.0f);
    } else {
        const float t = truncf(a);
        ip = __float2ull_rz(t);
        fr = __float2ull_rz((a - t) * 18446744073709551616.0f);
    }
    const i128 m = (i128)(((unsigned __int128)ip << 64) | (unsigned __int128)fr);
    return signbit(x) ? -m : m;
#else
    uint32_t b;
    memcpy(&b, &x, 4);
    const int e = (int)((b >> 23) & 0xffu);
    if (e == 255) {
        bad = 1;
        return 0;
    }
    if (e == 0) return 0;  // zero or subnormal (< 2^-126): truncates to 0
    const int E = e - 127;
    if (E >= 62) {
        bad = 1;
        return 0;
    }
    const unsigned long long mant = (unsigned long long)((b & 0x7fffffu) | 0x800000u);
    const int sh = E + 41;  // x * 2^64 = mant * 2^(E - 23 + 64)
    i128 m;
    if (sh >= 0)
        m = (i128)mant << sh;
    else if (sh > -64)
        m = (i128)(mant >> (-sh));
    else
        m = 0;
    return (b >> 31) ? -m : m;
#endif
}

LES_HD double fix_finish(i128 t, int bad) {
    if (bad) return __builtin_nan("");
    const long long hi = (long long)(t >> 64);
    const unsigned long long lo = (unsigned long long)t;
    const double two64 = 18446744073709551616.0;
    return ((double)hi * two64 + (double)lo) / two64;
}

LES_HD i128 fix_from_part(const FixPart &p) {
    return (i128)(((unsigned __int128)(unsigned long long)p.hi << 64) | (unsigned __int128)p.lo);
}

LES_HD FixPart fix_to_part(i128 t, int bad) {
    FixPart p;
    p.lo = (unsigned long long)t;
    p.hi = (long long)(t >> 64);
    p.bad = bad;
    p.pad = 0;
    return p;
}

}  // namespace les
