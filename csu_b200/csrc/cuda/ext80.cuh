// ext80.cuh -- exact software model of x87 extended-precision arithmetic (64-bit significand,
// round-to-nearest-even), for the device.
//
// The reference accumulates its least-squares gradient in `long double` (solverCalcGrad3,
// solver.c:1041): on x86-64 Linux that is the x87 80-bit format. Its double results are therefore
// round53(round64(...)) of each operation, which plain FP64 (or double-double) arithmetic cannot
// reproduce in every case. The DPLUR blocks difference F(U + 1e-6) - F(U) (implicit.c:692-788) magnify a
// one-ulp difference of the state into a 1e-7 change of the Jacobian, so a last-bit mismatch of a single
// gradient makes implicit histories drift. These routines reproduce the x87 results bit for bit (for
// normal numbers; the reference's gradients never leave that range), so the residual is exact.
//
// A value is (-1)^s * m * 2^e with m normalised to bit 63 (m == 0 is zero). Only +, *, / and the
// conversions used by solverCalcGrad3 are provided. Every operation computes the exact result in 128-bit
// integers and rounds once, which is what the x87 unit does.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define X80_HD __host__ __device__ __forceinline__
#else
#define X80_HD static inline
#endif

namespace csu {

typedef unsigned __int128 u128;

struct X80 {
    unsigned long long m;
    int e;
    int s;
};

X80_HD int x80_clz64(unsigned long long v)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)v);
#else
    return v ? __builtin_clzll(v) : 64;
#endif
}

X80_HD int x80_clz128(u128 v)
{
    unsigned long long hi = (unsigned long long)(v >> 64), lo = (unsigned long long)v;
    return hi ? x80_clz64(hi) : 64 + x80_clz64(lo);
}

X80_HD X80 x80_zero(int s)
{
    X80 r;
    r.m = 0;
    r.e = 0;
    r.s = s;
    return r;
}

X80_HD unsigned long long x80_dbits(double d)
{
#ifdef __CUDA_ARCH__
    return (unsigned long long)__double_as_longlong(d);
#else
    union {
        double d;
        unsigned long long u;
    } c;
    c.d = d;
    return c.u;
#endif
}

X80_HD double x80_bitsd(unsigned long long b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    union {
        double d;
        unsigned long long u;
    } c;
    c.u = b;
    return c.d;
#endif
}

// exact conversion of a double
X80_HD X80 x80_from_double(double d)
{
    unsigned long long b = x80_dbits(d);
    X80 r;
    r.s = (int)(b >> 63);
    int E = (int)((b >> 52) & 0x7ff);
    unsigned long long F = b & ((1ULL << 52) - 1);
    if (E == 0) {
        if (F == 0) return x80_zero(r.s);
        int lz = x80_clz64(F);
        r.m = F << lz;
        r.e = -1074 - lz;
    } else {
        r.m = (F | (1ULL << 52)) << 11;
        r.e = E - 1075 - 11;
    }
    return r;
}

// round a non-zero 128-bit magnitude M * 2^e (plus a sticky bit below it) to a 64-bit significand
X80_HD X80 x80_round(int s, u128 M, int e, bool sticky)
{
    int lz = x80_clz128(M);
    M <<= lz;
    e -= lz;
    unsigned long long hi = (unsigned long long)(M >> 64), lo = (unsigned long long)M;
    const unsigned long long half = 1ULL << 63;
    bool up = lo > half || (lo == half && (sticky || (hi & 1)));
    if (up) {
        hi++;
        if (hi == 0) {
            hi = half;
            e++;
        }
    }
    X80 r;
    r.m = hi;
    r.e = e + 64;
    r.s = s;
    return r;
}

X80_HD X80 x80_neg(X80 a)
{
    a.s ^= 1;
    return a;
}

X80_HD X80 x80_add(X80 a, X80 b)
{
    if (a.m == 0) {
        if (b.m == 0) return x80_zero(a.s & b.s);
        return b;
    }
    if (b.m == 0) return a;
    if (a.e < b.e || (a.e == b.e && a.m < b.m)) {
        X80 t = a;
        a = b;
        b = t;
    }
    int d = a.e - b.e;
    u128 A = (u128)a.m << 64;
    u128 B;
    bool sticky = false;
    if (d == 0) {
        B = (u128)b.m << 64;
    } else if (d < 128) {
        u128 full = (u128)b.m << 64;
        B = full >> d;
        sticky = (full << (128 - d)) != 0;
    } else {
        B = 0;
        sticky = true;
    }
    if (a.s == b.s) {
        u128 S = A + B;
        if (S < A) { // carry out of bit 127
            sticky = sticky || (S & 1);
            S = (S >> 1) | ((u128)1 << 127);
            return x80_round(a.s, S, a.e - 64 + 1, sticky);
        }
        return x80_round(a.s, S, a.e - 64, sticky);
    }
    u128 D = A - B;
    if (sticky) D -= 1; // the shifted-out part of B is borrowed, the remainder stays sticky
    if (D == 0 && !sticky) return x80_zero(0);
    return x80_round(a.s, D, a.e - 64, sticky);
}

X80_HD X80 x80_mul(X80 a, X80 b)
{
    if (a.m == 0 || b.m == 0) return x80_zero(a.s ^ b.s);
    u128 P = (u128)a.m * b.m;
    return x80_round(a.s ^ b.s, P, a.e + b.e, false);
}

// a / b, b != 0: 67 quotient bits by restoring division, remainder as sticky
X80_HD X80 x80_div(X80 a, X80 b)
{
    if (a.m == 0) return x80_zero(a.s ^ b.s);
    unsigned long long am = a.m, bm = b.m;
    u128 Q = am >= bm ? 1 : 0;
    u128 r = am >= bm ? (u128)(am - bm) : (u128)am;
    for (int i = 0; i < 66; i++) {
        r <<= 1;
        Q <<= 1;
        if (r >= bm) {
            r -= bm;
            Q |= 1;
        }
    }
    return x80_round(a.s ^ b.s, Q, a.e - b.e - 66, r != 0);
}

// Reciprocal for dividing by a fixed normalised 64-bit significand d (Moller & Granlund, "Improved division
// by invariant integers", 2011): v = floor((2^128 - 1) / d) - 2^64. Computed once per divisor.
X80_HD unsigned long long x80_recip(unsigned long long d)
{
    u128 all = ~(u128)0;
    return (unsigned long long)(all / d - ((u128)1 << 64));
}

// floor((u1 * 2^64 + u0) / d) and remainder, for u1 < d (their Algorithm 4, two products)
X80_HD unsigned long long x80_udiv_pre(unsigned long long u1, unsigned long long u0, unsigned long long d,
                                       unsigned long long v, unsigned long long* rem)
{
    u128 q = (u128)v * u1;
    q += ((u128)u1 << 64) | u0;
    unsigned long long q1 = (unsigned long long)(q >> 64) + 1, q0 = (unsigned long long)q;
    unsigned long long r = u0 - q1 * d;
    if (r > q0) {
        q1--;
        r += d;
    }
    if (r >= d) {
        q1++;
        r -= d;
    }
    *rem = r;
    return q1;
}

// a / b with v = x80_recip(b.m): same result as x80_div, in two invariant-divisor steps
X80_HD X80 x80_div_pre(X80 a, X80 b, unsigned long long v)
{
    if (a.m == 0) return x80_zero(a.s ^ b.s);
    unsigned long long d = b.m, n = a.m, r, r2;
    unsigned long long Q1 = n >= d ? 1 : 0;
    unsigned long long u1 = n - Q1 * d;
    unsigned long long q = x80_udiv_pre(u1, 0, d, v, &r);
    unsigned long long q2 = x80_udiv_pre(r, 0, d, v, &r2);
    u128 M = ((u128)Q1 << 127) | ((u128)q << 63) | (q2 >> 1);
    bool sticky = (q2 & 1) || r2 != 0;
    return x80_round(a.s ^ b.s, M, a.e - b.e - 127, sticky);
}

// round to double (nearest even); normal range exact, outside it via scaling
X80_HD double x80_to_double(X80 x)
{
    if (x.m == 0) return x.s ? -0.0 : 0.0;
    unsigned long long m53 = x.m >> 11, rem = x.m & 0x7ffULL;
    int e = x.e + 11;
    if (rem > 0x400ULL || (rem == 0x400ULL && (m53 & 1))) {
        m53++;
        if (m53 == (1ULL << 53)) {
            m53 >>= 1;
            e++;
        }
    }
    int E = e + 52 + 1023;
    if (E <= 0 || E >= 2047) {
        double v = (double)m53;
        // rare: scale in two steps to avoid intermediate overflow
        int h = e / 2;
#ifdef __CUDA_ARCH__
        v = ldexp(ldexp(v, h), e - h);
#else
        v = __builtin_ldexp(__builtin_ldexp(v, h), e - h);
#endif
        return x.s ? -v : v;
    }
    unsigned long long bits = ((unsigned long long)x.s << 63) | ((unsigned long long)E << 52) |
                              (m53 & ((1ULL << 52) - 1));
    return x80_bitsd(bits);
}

} // namespace csu
