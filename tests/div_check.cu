// Host build (nvcc, no device code runs) of the quotient helpers of
// sc_common.cuh: quot_in_range at the edges of its range, and div_rcp (a
// product by the correctly rounded reciprocal with one FMA correction)
// against the IEEE quotient on random operands, including quotients near
// the ends of the range where the helper falls back to a division and
// subnormal dividends (whose quotients by divisors of at least 2^-70 fall
// below the range, so the remainder of every fast quotient is exact).
// Prints: <edge failures> <quotients> <mismatches> <fast-path quotients>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <random>

#include "sc_common.cuh"

int main(int argc, char** argv) {
    const long n = argc > 1 ? std::atol(argv[1]) : 1000000;
    int edge = 0;
    const double lo = std::ldexp(1.0, -899), hi = std::ldexp(1.0, 900);
    const double inf = std::numeric_limits<double>::infinity(), nan = std::numeric_limits<double>::quiet_NaN();
    const struct {
        double q;
        bool in;
    } cases[] = {{lo, true},   {std::nextafter(lo, 0.0), false}, {-lo, true}, {hi, false},
                 {std::nextafter(hi, 0.0), true}, {-std::nextafter(hi, 0.0), true}, {0.0, false},
                 {-0.0, false}, {std::numeric_limits<double>::denorm_min(), false}, {inf, false},
                 {-inf, false}, {nan, false}, {1.0, true}, {-3.5e-200, true}, {7.0e250, true}};
    for (const auto& c : cases) edge += sc::quot_in_range(c.q) != c.in;
    std::mt19937_64 g(2026);
    // divisors in the callers' range (|b| >= 2^-70: mesh spacings, c dt,
    // gamma), dividends from subnormal to near overflow
    std::uniform_real_distribution<double> e(-1000.0, 1000.0), eb(-70.0, 300.0), m(1.0, 2.0), s(-1.0, 1.0);
    long bad = 0, fast = 0;
    for (long i = 0; i < n; ++i) {
        const double b = (s(g) < 0 ? -1.0 : 1.0) * m(g) * std::ldexp(1.0, (int)eb(g));
        // quotient exponents spread over the whole range, edges included
        const double a = (s(g) < 0 ? -1.0 : 1.0) * m(g) * std::ldexp(1.0, (int)e(g)) * std::fabs(b);
        const double rb = 1.0 / b;
        const double q = sc::div_rcp(a, b, rb), ref = a / b;
        bad += std::memcmp(&q, &ref, sizeof q) != 0;
        fast += sc::quot_in_range(a * rb);
    }
    std::printf("%d %ld %ld %ld\n", edge, n, bad, fast);
    return 0;
}
