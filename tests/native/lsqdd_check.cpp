// Host check of csu_b200/csrc/cuda/lsqdd.cuh against the x86-64 host's x87 long double:
//  1. the FP64 emulation of single x87 operations (accumulation step, product, sum of x87 values) on
//     random, tie-prone, power-of-two and cancelling operands: results equal bit for bit whenever the
//     emulation reports success, and it reports success almost always;
//  2. the reference's least-squares formula (solverCalcGrad3, solver.c:1031-1074): every component that
//     the certified double-double solve or the exact-numerator solve returns equals the x87 result.
// Prints counts; exit status 1 on any mismatch.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "../../csu_b200/csrc/cuda/lsqdd.cuh"

using namespace csu;

static DD dd_of(long double v)
{
    double h = (double)v;
    DD r = {h, (double)(v - (long double)h)};
    return r;
}

static long double ld_of(DD d) { return (long double)d.h + (long double)d.l; }

static bool same(long double a, long double b)
{
    return a == b && std::signbit(a) == std::signbit(b);
}

int main(int argc, char** argv)
{
    long n = argc > 1 ? atol(argv[1]) : 200000;
    std::mt19937_64 rng(987654321);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::uniform_int_distribution<int> E(-30, 30);
    std::uniform_int_distribution<int> S(-80, 20);
    long bad_op = 0, undecided_op = 0, ops = 0;
    auto rnd64 = [&]() {
        long double v = (long double)U(rng) * ldexpl(1.0L, E(rng));
        return v + (long double)U(rng) * ldexpl(fabsl(v), -55); // all 64 significand bits
    };
    for (long i = 0; i < 4 * n; i++) {
        long double sv = rnd64();
        int ge;
        frexpl(sv, &ge);
        long double G = ldexpl(1.0L, ge - 64); // spacing of 64-bit significands at sv
        double p = ldexp(U(rng), S(rng)) * (double)fabsl(sv);
        if (i % 7 == 0) p = (double)ldexpl(floorl(ldexpl(sv, 70)) + 0.5L, -70);
        if (i % 11 == 0) p = -(double)sv;
        if (i % 13 == 1) // just off a midpoint: the tie needs the low part
            p = (double)(0.5L * G * (1.0L + ((rng() & 1) ? 1 : -1) * ldexpl(1.0L, -52))) * ((rng() & 1) ? 1 : -1);
        if (i % 13 == 2) { // power of two minus a fraction of the spacing
            sv = ldexpl(1.0L, ge) * (sv < 0 ? -1 : 1);
            long double G2 = ldexpl(1.0L, ge + 1 - 64);
            long double f = 0.25L + 0.5L * (long double)U(rng) * 0.999L;
            p = -(double)(f * G2) * (sv < 0 ? -1 : 1);
        }
        // accumulation step
        bool ok = true;
        DD r = x87_sum_add(dd_of(sv), p, ok);
        ops++;
        if (!ok) undecided_op++;
        else if (!same(ld_of(r), sv + (long double)p)) bad_op++;
        // first two terms
        double p2 = ldexp(U(rng), S(rng) / 2);
        ok = true;
        r = x87_sum2(p, p2, ok);
        ops++;
        if (!ok) undecided_op++;
        else if (!same(ld_of(r), ((long double)0 + (long double)p) + (long double)p2)) bad_op++;
        // product and sum of two x87 values (sums near cancellation every third case)
        long double tv = rnd64();
        if (i % 3 == 0) tv = -sv * (1 + ldexpl(1.0L, -40 - (int)(rng() % 20)) * (long double)U(rng));
        if (i % 5 == 0) tv = sv * ldexpl(1.0L, (int)(rng() % 40) - 20) * (1 + (long double)U(rng) * 1e-3L);
        ok = true;
        r = x87_mul(dd_of(sv), dd_of(tv), ok);
        ops++;
        if (!ok) undecided_op++;
        else if (!same(ld_of(r), sv * tv) && !(r.h == 0 && sv * tv == 0)) bad_op++;
        ok = true;
        r = x87_add(dd_of(sv), dd_of(tv), ok);
        ops++;
        if (!ok) undecided_op++;
        else if (!(ld_of(r) == sv + tv)) bad_op++;
    }
    // full formula
    long bad = 0, tried = 0, cert1 = 0, cert2 = 0, bad_sum = 0;
    for (long i = 0; i < n; i++) {
        int kind = (int)(i % 5);
        int nn = 3 + (int)(rng() & 1);
        double x[5], y[5], u[5];
        double scale = ldexp(1.0, E(rng) / 3);
        x[0] = U(rng) * 10;
        y[0] = U(rng) * 10;
        double u0 = U(rng) * ldexp(1.0, E(rng) / 2);
        double gx = U(rng), gy = U(rng);
        if (kind == 4) gx *= 1e-9; // field varying along y only: strong cancellation in the x numerator
        u[0] = u0;
        for (int j = 1; j <= nn; j++) {
            x[j] = x[0] + U(rng) * scale;
            y[j] = y[0] + U(rng) * scale;
            if (kind == 0) u[j] = U(rng) * ldexp(1.0, E(rng) / 2);
            else if (kind == 1 || kind == 4)
                u[j] = u0 + (gx * (x[j] - x[0]) + gy * (y[j] - y[0])) * (1 + 1e-12 * U(rng));
            else if (kind == 2) u[j] = u0 * (1 + 1e-14 * U(rng));
            else u[j] = (rng() & 3) ? u0 : u0 * (1 + 1e-9 * U(rng));
        }
        long double a = 0, b = 0, c = 0, A = 0, B = 0;
        double px[4], py[4];
        for (int j = 1; j <= nn; j++) {
            double dx = x[j] - x[0], dy = y[j] - y[0], du = u[j] - u[0];
            a += dx * dx;
            b += dx * dy;
            c += dy * dy;
            A += dx * du;
            B += dy * du;
            px[j - 1] = dx * du;
            py[j - 1] = dy * du;
        }
        long double det = a * c - b * b;
        double rx = (c * A - b * B) / det;
        double ry = (-b * A + a * B) / det;
        bool ok = true;
        DD ax = x87_sum2(px[0], px[1], ok), ay = x87_sum2(py[0], py[1], ok);
        for (int j = 2; j < nn; j++) {
            ax = x87_sum_add(ax, px[j], ok);
            ay = x87_sum_add(ay, py[j], ok);
        }
        if (!ok || ld_of(ax) != A || ld_of(ay) != B) {
            if (bad_sum < 10) printf("sum mismatch kind %d\n", kind);
            bad_sum++;
            continue;
        }
        DD ka = dd_of(a), kb = dd_of(b), kc = dd_of(c);
        DD R = dd_recip(dd_of(det));
        for (int comp = 0; comp < 2; comp++) {
            double q, want = comp ? ry : rx;
            DD k1 = comp ? ka : kc, X = comp ? ay : ax, Y = comp ? ax : ay;
            tried++;
            if (lsq_certified(k1, kb, R, X, Y, &q)) cert1++;
            else if (lsq_exact_numerator(k1, kb, R, X, Y, &q)) cert2++;
            else continue;
            if (memcmp(&q, &want, 8) != 0) {
                if (bad < 10) printf("mismatch kind %d comp %d: %.17g vs %.17g\n", kind, comp, q, want);
                bad++;
            }
        }
    }
    printf("ops=%ld undecided=%ld op_mismatches=%ld | components=%ld certified=%.4f exact_numerator=%.4f "
           "left=%.5f mismatches=%ld sum_mismatches=%ld\n",
           ops, undecided_op, bad_op, tried, (double)cert1 / tried, (double)cert2 / tried,
           1.0 - (double)(cert1 + cert2) / tried, bad, bad_sum);
    return (bad || bad_sum || bad_op) ? 1 : 0;
}
