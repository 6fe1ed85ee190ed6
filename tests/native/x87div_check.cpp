// x87_div_d (lsqdd.cuh), the double a `long double` division of two doubles stores -- the quotients of the
// reference's SST diagonal solve (implicit.c:341-342) -- against this x86-64 host's x87: random operands
// over wide exponent ranges, near-midpoint quotients (n = d * (q + half an ulp) perturbed by a few ulps),
// exact quotients, and mixed signs. Prints the counts; exit status 1 on any mismatch.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../csu_b200/csrc/cuda/lsqdd.cuh"

using namespace csu;

static double x87(double n, double d)
{
    volatile long double q = (long double)n / (long double)d;
    return (double)q;
}

int main(int argc, char** argv)
{
    const long N = argc > 1 ? atol(argv[1]) : 1000000;
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::uniform_int_distribution<int> ex(-40, 40);
    long tried = 0, decided = 0, bad = 0, naive = 0;
    auto check = [&](double n, double d) {
        if (d == 0.0) return;
        bool ok = true;
        double q = x87_div_d(n, d, ok);
        double want = x87(n, d);
        tried++;
        if (!(n / d == want) && !std::isnan(want)) naive++; // where double rounding shows
        if (!ok) return; // the caller falls back to the integer model
        decided++;
        if (!(q == want) && !(std::isnan(q) && std::isnan(want))) {
            if (bad < 10) printf("mismatch n=%a d=%a got %a want %a\n", n, d, q, want);
            bad++;
        }
    };
    for (long i = 0; i < N; i++) {
        double n = std::ldexp(u(rng), ex(rng)), d = std::ldexp(u(rng), ex(rng));
        check(n, d);
        // near the midpoint between two doubles: q + half an ulp, nudged by a few ulps of n
        double q = n / d;
        if (std::isfinite(q) && q != 0.0) {
            double h = std::nextafter(q, 2 * q) - q;
            double nm = (q + 0.5 * h) * d;
            for (int k = -2; k <= 2; k++) {
                double nk = nm;
                for (int s = 0; s < (k < 0 ? -k : k); s++) nk = std::nextafter(nk, k < 0 ? -INFINITY : INFINITY);
                check(nk, d);
            }
            check(q * d, d); // often an exact quotient
        }
    }
    printf("tried=%ld decided=%ld undecided=%ld mismatches=%ld naive_differs=%ld\n", tried, decided,
           tried - decided, bad, naive);
    return bad ? 1 : 0;
}
