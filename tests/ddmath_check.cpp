// Host build of the device double-double log / atan (sc_ddmath.cuh) checked
// against quad precision rounded once (libquadmath).  Prints one line:
//   <n> <log mismatches> <atan mismatches> <libm log mismatches> <libm atan mismatches>
// Arguments are log-uniform over the ranges the Green's function produces.
#include <quadmath.h>

#include <cstdio>
#include <cstdlib>
#include <random>

#include "sc_ddmath.cuh"

int main(int argc, char** argv) {
    const long n = argc > 1 ? std::atol(argv[1]) : 1000000;
    std::mt19937_64 g(12345);
    std::uniform_real_distribution<double> el(-30.0, 30.0), ea(-22.0, 22.0), sg(-1.0, 1.0);
    long bl = 0, ba = 0, ll = 0, la = 0;
    for (long i = 0; i < n; ++i) {
        const double x = std::exp(el(g));
        const double lq = (double)logq((__float128)x);
        bl += sc::ddm::log_dd(x) != lq;
        ll += std::log(x) != lq;
        const double y = (sg(g) < 0 ? -1.0 : 1.0) * std::exp(ea(g));
        const double aq = (double)atanq((__float128)y);
        ba += sc::ddm::atan_dd(y) != aq;
        la += std::atan(y) != aq;
    }
    // a few exact cases
    bl += sc::ddm::log_dd(1.0) != 0.0;
    ba += sc::ddm::atan_dd(0.0) != 0.0;
    ba += sc::ddm::atan_dd(1.0) != (double)atanq((__float128)1.0);
    ba += sc::ddm::atan_dd(-1.0) != (double)atanq((__float128)-1.0);
    std::printf("%ld %ld %ld %ld %ld\n", n, bl, ba, ll, la);
    return 0;
}
