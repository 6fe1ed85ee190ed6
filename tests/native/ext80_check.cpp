// Host check of csu_b200/csrc/cuda/ext80.cuh against the x86-64 host's x87 long double: the primitive
// operations on random operands, and the reference's least-squares gradient formula
// (solverCalcGrad3, solver.c:1031-1074) evaluated both ways. Prints the number of mismatches.
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <random>
#include "../../csu_b200/csrc/cuda/ext80.cuh"

using namespace csu;

static long double to_ld(X80 x)
{
    if (x.m == 0) return x.s ? -0.0L : 0.0L;
    long double v = ldexpl((long double)x.m, x.e);
    return x.s ? -v : v;
}

static X80 from_ld(long double v)
{
    if (v == 0) return x80_zero(std::signbit(v) ? 1 : 0);
    int e;
    long double f = frexpl(fabsl(v), &e);
    X80 r;
    r.m = (unsigned long long)ldexpl(f, 64);
    r.e = e - 64;
    r.s = v < 0;
    return r;
}

static bool same(long double a, long double b)
{
    return memcmp(&a, &b, 10) == 0 || (a == 0 && b == 0 && std::signbit(a) == std::signbit(b));
}

int main(int argc, char** argv)
{
    long n = argc > 1 ? atol(argv[1]) : 200000;
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::uniform_int_distribution<int> E(-40, 40);
    auto rnd = [&]() { return ldexp(U(rng), E(rng)); };
    long bad_add = 0, bad_mul = 0, bad_div = 0, bad_cvt = 0, bad_grad = 0;
    for (long i = 0; i < n; i++) {
        double x = rnd(), y = rnd();
        long double lx = (long double)x + (long double)rnd() * 1e-3L;
        long double ly = (long double)y * (1 + 1e-9L * (long double)rnd());
        X80 X = from_ld(lx), Y = from_ld(ly);
        if (!same(to_ld(X), lx)) bad_cvt++;
        if (!same(to_ld(x80_add(X, Y)), lx + ly)) bad_add++;
        if (!same(to_ld(x80_add(X, x80_neg(Y))), lx - ly)) bad_add++;
        if (!same(to_ld(x80_mul(X, Y)), lx * ly)) bad_mul++;
        if (ly != 0 && !same(to_ld(x80_div(X, Y)), lx / ly)) bad_div++;
        if (ly != 0 && !same(to_ld(x80_div_pre(X, Y, x80_recip(Y.m))), lx / ly)) bad_div++;
        double dx = x80_to_double(X);
        if (dx != (double)lx) bad_cvt++;
        // near-cancellation additions
        long double lz = -lx * (1 + 1e-17L * (long double)rnd());
        if (!same(to_ld(x80_add(X, from_ld(lz))), lx + lz)) bad_add++;
        // solverCalcGrad3: x/y offsets of 3-4 neighbours, values u
        int nn = 3 + (int)(rng() & 1);
        double ddx[4], ddy[4], du[4];
        long double a = 0, b = 0, c = 0, A = 0, B = 0;
        double scale = ldexp(1.0, E(rng) / 4);
        for (int j = 0; j < nn; j++) {
            ddx[j] = U(rng) * scale;
            ddy[j] = U(rng) * scale;
            du[j] = U(rng) * ldexp(1.0, E(rng) / 4);
            a += ddx[j] * ddx[j];
            b += ddx[j] * ddy[j];
            c += ddy[j] * ddy[j];
            A += ddx[j] * du[j];
            B += ddy[j] * du[j];
        }
        double gx = (c * A - b * B) / (a * c - b * b);
        double gy = (-b * A + a * B) / (a * c - b * b);
        X80 XA = x80_zero(0), XB = x80_zero(0);
        for (int j = 0; j < nn; j++) {
            XA = x80_add(XA, x80_from_double(ddx[j] * du[j]));
            XB = x80_add(XB, x80_from_double(ddy[j] * du[j]));
        }
        X80 Xa = from_ld(a), Xb = from_ld(b), Xc = from_ld(c), Xd = from_ld(a * c - b * b);
        double hx = x80_to_double(x80_div(x80_add(x80_mul(Xc, XA), x80_neg(x80_mul(Xb, XB))), Xd));
        double hy = x80_to_double(x80_div_pre(x80_add(x80_mul(x80_neg(Xb), XA), x80_mul(Xa, XB)), Xd, x80_recip(Xd.m)));
        if (memcmp(&gx, &hx, 8) != 0 || memcmp(&gy, &hy, 8) != 0) bad_grad++;
    }
    printf("n=%ld add=%ld mul=%ld div=%ld cvt=%ld grad=%ld\n", n, bad_add, bad_mul, bad_div, bad_cvt, bad_grad);
    return (bad_add || bad_mul || bad_div || bad_cvt || bad_grad) ? 1 : 0;
}
