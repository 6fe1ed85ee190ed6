// lsqdd.cuh -- certified fast evaluation of the reference's extended-precision least-squares solve.
//
// solverCalcGrad3 (solver.c:1031-1074) sums double products in x87 `long double` and solves the 2x2
// normal equations there:  dUx = (c A - b B) / (a c - b b),  dUy = (-b A + a B) / (a c - b b), each result
// rounded to double. ext80.cuh reproduces that bit for bit with 128-bit integer arithmetic, which is exact
// but costs ~1,000 integer instructions per gradient component.
//
// This header evaluates the same quantity in double-double arithmetic (FP64 pipes, error-free
// transformations with explicit fma) together with a rigorous bound E on the distance between the
// double-double value and the value the x87 sequence produces before its final rounding to double:
//
//   - the sums A, B are reproduced exactly (x87_sum_add: each step rounded to 64 bits in FP64 with
//     error-free transformations and an exact round-to-nearest-even on the 64-bit grid);
//   - every later x87 operation rounds to a 64-bit significand, relative error <= u = 2^-64: the two
//     products and the difference add u * |term| each, the division u * |q|;
//   - the double-double evaluation itself is accurate to ~2^-100 relative (Joldes, Muller & Popescu,
//     "Tight and rigorous error bounds for basic building blocks of double-word arithmetic", ACM TOMS
//     2017), covered here by a 2^-96 term.
//
// If the interval [q - E, q + E] around the double-double value q contains no rounding boundary of
// double precision (a midpoint between two consecutive doubles), the x87 result rounds to the same
// double as q, namely RN(q): the component is certified and returned. Otherwise (about one component in
// a hundred on solver meshes: strong cancellation in the numerator, or q close to a midpoint)
// lsq_exact_numerator computes the numerator exactly as x87 would, then the x87 division's rounding to 64
// bits from the double-double quotient and its bound, and the store to double exactly; what that cannot
// decide (a quotient within 2^-100 of a boundary of the 64-bit grid: none in millions of random
// components) the caller recomputes with ext80.cuh. Either way the result is the reference's bit pattern.
#pragma once
#include <math.h>
#include <string.h>

#include "ext80.cuh"

namespace csu {

struct DD {
    double h, l;
};

X80_HD double dd_bits2d(unsigned long long b)
{
    double d;
    memcpy(&d, &b, 8);
    return d;
}

X80_HD unsigned long long dd_d2bits(double d)
{
    unsigned long long b;
    memcpy(&b, &d, 8);
    return b;
}

// Knuth's TwoSum: s + e == a + b exactly
X80_HD DD dd_two_sum(double a, double b)
{
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    DD r = {s, e};
    return r;
}

// Dekker's FastTwoSum (|a| >= |b| or a == 0)
X80_HD DD dd_fast_two_sum(double a, double b)
{
    double s = a + b;
    double e = b - (s - a);
    DD r = {s, e};
    return r;
}

// a * b == p + e exactly (fma computes a*b - p without intermediate rounding)
X80_HD DD dd_two_prod(double a, double b)
{
    double p = a * b;
    double e = fma(a, b, -p);
    DD r = {p, e};
    return r;
}

// AccurateDWPlusDW (relative error <= 3u^2 even under cancellation)
X80_HD DD dd_add(DD a, DD b)
{
    DD s = dd_two_sum(a.h, b.h);
    DD t = dd_two_sum(a.l, b.l);
    double c = s.l + t.h;
    DD v = dd_fast_two_sum(s.h, c);
    double w = t.l + v.l;
    return dd_fast_two_sum(v.h, w);
}

X80_HD DD dd_neg(DD a)
{
    DD r = {-a.h, -a.l};
    return r;
}

// DWTimesDW (relative error <= 7u^2)
X80_HD DD dd_mul(DD a, DD b)
{
    DD p = dd_two_prod(a.h, b.h);
    double t = a.h * b.l;
    t = t + a.l * b.h;
    double c = p.l + t;
    return dd_fast_two_sum(p.h, c);
}

// An x87 value as an exact double-double (normal range only; m has bit 63 set or is zero).
X80_HD DD dd_from_x80(X80 x)
{
    DD r;
    if (x.m == 0) {
        r.h = 0.0;
        r.l = 0.0;
        return r;
    }
    double hi = ldexp((double)(x.m >> 11), x.e + 11);
    double lo = ldexp((double)(x.m & 0x7ffULL), x.e);
    r = dd_fast_two_sum(hi, lo);
    if (x.s) r = dd_neg(r);
    return r;
}

// 1/d to ~2^-104 relative: one Newton correction of the FP64 reciprocal.
X80_HD DD dd_recip(DD d)
{
    double r = 1.0 / d.h;
    double e = fma(-d.h, r, 1.0);
    e = e - d.l * r;
    return dd_fast_two_sum(r, e * r);
}

// RN64 of the exact total h + r.h + r.l + e, |e| <= err, where h = RN53 of (nearly) the total and r is
// normalised (|r.l| <= ulp(r.h) / 2) with |r| <~ ulp(h): the 64-bit grid in h's binade has spacing
// G = ulp(h) / 2^11 (half of it just below a power of two). Returns the rounded value as an exact
// double-double. ok is cleared when the rounding cannot be decided: the remainder within |r.l| + err of a
// midpoint with err > 0, or a magnitude outside the range where G is a normal double.
X80_HD DD x87_round(double h, DD r, double err, bool& ok)
{
    if (h == 0.0) {
        if (r.l != 0.0 || err != 0.0) ok = false;
        DD z = {r.h, 0.0};
        return z;
    }
    unsigned long long bits = dd_d2bits(h);
    unsigned long long ex = (bits >> 52) & 0x7ffULL;
    if (ex <= 64ULL || ex >= 0x7c0ULL) {
        ok = false;
        DD z = {h, 0.0};
        return z;
    }
    double G = dd_bits2d((ex - 63ULL) << 52);
    bool pow2 = (bits & 0xfffffffffffffULL) == 0;
    if (pow2 && r.h != 0.0 && ((r.h < 0.0) != (h < 0.0))) G *= 0.5;
    // r.h to a multiple of G, ties to even (|r.h| < 2^51 G); an exact tie is broken by r.l
    double C = 0x1.8p52 * G;
    double q = (r.h + C) - C;
    double d = r.h - q;
    double hg = 0.5 * G;
    if (err == 0.0) {
        if (d == hg && r.l > 0.0) q += G;
        if (d == -hg && r.l < 0.0) q -= G;
    } else if (!(hg - fabs(d) > fabs(r.l) + err)) {
        ok = false;
    }
    return dd_fast_two_sum(h, q);
}

// First two terms of the reference's `long double` accumulation (solver.c:1066-1070), exactly:
// A = 0; A += p1; A += p2 gives RN64(p1 + p2) (0 + p1 is exact and +0 for a zero p1).
X80_HD DD x87_sum2(double p1, double p2, bool& ok)
{
    DD t = dd_two_sum(p1 + 0.0, p2);
    DD r = {t.l, 0.0};
    return x87_round(t.h, r, 0.0, ok);
}

// One more step, A += p: s is an x87 value held as an exact double-double (s.h = RN53(s), s.l the
// remaining <= 11 bits); returns RN64(s + p) in the same form.
X80_HD DD x87_sum_add(DD s, double p, bool& ok)
{
    DD t = dd_two_sum(s.h, p);
    DD w = dd_two_sum(t.l, s.l);
    DD v = dd_two_sum(t.h, w.h);
    DD r = dd_two_sum(v.l, w.l); // s + p == v.h + r.h + r.l exactly
    return x87_round(v.h, r, 0.0, ok);
}

// RN64(a * b) for x87 values held as exact double-doubles: the exact product is the sum of four exact
// partial products (a.l and b.l carry at most 11 bits, so a.h * b.l and a.l * b.h fit in 64 bits and
// a.l * b.l in 22); the smallest parts enter through a tail with a rounding bound.
X80_HD DD x87_mul(DD a, DD b, bool& ok)
{
    DD p = dd_two_prod(a.h, b.h);
    if (p.h == 0.0) {
        DD z = {p.h, 0.0};
        return z;
    }
    DD m1 = dd_two_prod(a.h, b.l);
    DD m2 = dd_two_prod(a.l, b.h);
    double m3 = a.l * b.l;
    DD s1 = dd_two_sum(m1.h, m2.h);
    DD s2 = dd_two_sum(p.l, s1.h);
    double tail = ((s2.l + s1.l) + (m1.l + m2.l)) + m3;
    double terr = 0x1p-50 * (((fabs(s2.l) + fabs(s1.l)) + (fabs(m1.l) + fabs(m2.l))) + fabs(m3));
    DD v = dd_two_sum(p.h, s2.h);
    DD r = dd_two_sum(v.l, tail);
    return x87_round(v.h, r, terr, ok);
}

// RN64(a + b) for x87 values held as exact double-doubles.
X80_HD DD x87_add(DD a, DD b, bool& ok)
{
    DD s = dd_two_sum(a.h, b.h);
    DD f = dd_two_sum(a.l, b.l);
    DD g = dd_two_sum(s.l, f.h);
    DD v = dd_two_sum(s.h, g.h);  // a + b == v.h + v.l + g.l + f.l exactly
    DD t = dd_two_sum(g.l, f.l);
    DD r = dd_two_sum(v.l, t.h);  // a + b == v.h + r.h + r.l + t.l exactly
    return x87_round(v.h, r, fabs(t.l), ok);
}

// The double a `long double` division of two doubles stores, RN53(RN64(n / d)) (the reference's SST
// diagonal solves, implicit.c:341-342): h = RN53(n / d) with its exact remainder gives the quotient as a
// double-double to ~2^-106, rounded on the 64-bit grid (bound 2^-100 |h|); its high part is the store.
// ok is cleared when that rounding cannot be decided (or for zero, non-finite and extreme quotients).
X80_HD double x87_div_d(double n, double d, bool& ok)
{
    double h = n / d;
    if (n == 0.0) return h; // +-0 in x87 as in double
    if (h == 0.0 || !(fabs(h) <= 1.7976931348623157e308)) {
        ok = false;
        return h;
    }
    double r = fma(-h, d, n); // n - h d exactly
    DD t = {r / d, 0.0};
    DD q64 = x87_round(h, t, 0x1p-100 * fabs(h), ok);
    return q64.h;
}

// q as the double RN53(q) if [q - E, q + E] holds no rounding boundary of double precision.
X80_HD bool dd_round_certified(DD q, double E, double* out)
{
    double h = q.h, l = q.l;
    double ah = fabs(h);
    if (!(ah >= 0x1p-960 && ah <= 0x1p+960)) return false;
    unsigned long long bits = dd_d2bits(h);
    unsigned long long ex = (bits >> 52) & 0x7ffULL;
    double ulp = dd_bits2d((ex - 52ULL) << 52);
    bool pow2 = (bits & 0xfffffffffffffULL) == 0;
    bool toward0 = l == 0.0 || ((l < 0.0) != (h < 0.0));
    double half = (pow2 && toward0) ? 0.25 * ulp : 0.5 * ulp;
    if (!(half - fabs(l) > E)) return false;
    *out = h;
    return true;
}

// Certified RN53(x87: (k1 * X - k2 * Y) / det) for exact x87 sums X, Y and exact x87 constants k1, k2,
// with R = 1/det to ~2^-103, from a double-double evaluation and an error bound: the x87 errors left are
// the two products and the difference (u each, relative to their operands) and the division (u |q|).
// Cheap; fails under strong cancellation in the numerator (then use lsq_exact_numerator).
X80_HD bool lsq_certified(DD k1, DD k2, DD R, DD X, DD Y, double* out)
{
    if (X.h == 0.0 && Y.h == 0.0) {
        // both sums are +0 (an x87 sum that starts at +0 never becomes -0): the quotient is +0 (det > 0)
        *out = 0.0;
        return true;
    }
    const double u = 0x1p-64;
    DD t1 = dd_mul(k1, X), t2 = dd_mul(k2, Y);
    // t1 - t2 with the sloppy double-word sum: its error, <= 2^-104 (|t1| + |t2|), is covered below
    DD s = dd_two_sum(t1.h, -t2.h);
    DD N = dd_two_sum(s.h, s.l + (t1.l - t2.l));
    DD q = dd_mul(N, R);
    double aR = fabs(R.h), aq = fabs(q.h);
    double terms = fabs(k1.h) * fabs(X.h) + fabs(k2.h) * fabs(Y.h);
    double E = (u * (terms + fabs(N.h)) * aR + u * aq) * (1.0 + 0x1p-20) + 0x1p-95 * (terms * aR + aq);
    return dd_round_certified(q, E, out);
}

// The same when lsq_certified cannot decide: the x87 numerator RN64(RN64(k1 X) - RN64(k2 Y)) computed
// exactly (x87_mul, x87_add), then the x87 division itself: RN64(N / det) decided on the 64-bit grid from
// the double-double quotient N R (relative error <= 2^-103 (R) + 7 2^-106 (dd_mul) < 2^-102, bounded here by
// 2^-100 |q|), and its store to double, RN53 of that 64-bit value, done exactly by the hardware addition in
// x87_round's result (s = RN(h + q) of an exact sum). Undecidable only when the quotient lies within
// 2^-100 of a midpoint of the 64-bit grid. A zero numerator is +0 in x87 (k1 > 0 and the sums are never
// -0), and so is the quotient.
X80_HD bool lsq_exact_numerator(DD k1, DD k2, DD R, DD X, DD Y, double* out)
{
    bool ok = true;
    DD P1 = x87_mul(k1, X, ok);
    DD P2 = x87_mul(k2, Y, ok);
    P2.h = -P2.h;
    P2.l = -P2.l;
    DD N = x87_add(P1, P2, ok);
    if (!ok) return false;
    if (N.h == 0.0) {
        *out = 0.0;
        return true;
    }
    DD q = dd_mul(N, R);
    DD r = {q.l, 0.0};
    DD q64 = x87_round(q.h, r, 0x1p-100 * fabs(q.h), ok);
    if (!ok) return false;
    *out = q64.h;
    return true;
}

} // namespace csu
