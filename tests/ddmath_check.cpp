// Host build of the device double-double log / atan (sc_ddmath.cuh) checked
// against quad precision rounded once (libquadmath).  Prints one line:
//   <n> <log mismatches> <atan mismatches> <libm log mismatches> <libm atan mismatches>
//   <log quick != full> <atan quick != full> <log quick accepted> <atan quick accepted>
//   <Green's-function arguments> <of them decided by the quick phases>
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
    long bl = 0, ba = 0, ll = 0, la = 0, dl = 0, da = 0, ql = 0, qa = 0;
    for (long i = 0; i < n; ++i) {
        const double x = std::exp(el(g));
        const double lq = (double)logq((__float128)x);
        const double l = sc::ddm::log_dd(x);
        bl += l != lq;
        ll += std::log(x) != lq;
        dl += l != sc::ddm::log_dd_full(x);
        double r;
        ql += sc::ddm::log_quick(x, r);
        const double y = (sg(g) < 0 ? -1.0 : 1.0) * std::exp(ea(g));
        const double aq = (double)atanq((__float128)y);
        const double t = sc::ddm::atan_dd(y);
        ba += t != aq;
        la += std::atan(y) != aq;
        da += t != sc::ddm::atan_dd_full(y);
        // outside [2^-30, 2^30] the quick phase is not tried: count as decided
        qa += !(std::fabs(y) >= 9.3132257461547852e-10 && std::fabs(y) <= 1073741824.0) || sc::ddm::atan_quick(y, r);
    }
    // every table interval of both reductions, edges included, where the
    // quick phases' error is largest (log near 1 +- 1/128, atan near j/64)
    std::uniform_real_distribution<double> w(-1.0 / 128, 1.0 / 128);
    for (long i = 0; i < n / 4; ++i) {
        const double x = (45 + (int)(i % 47)) / 64.0 + w(g);
        if (x > 0.0) {
            const double lq = (double)logq((__float128)x);
            const double l = sc::ddm::log_dd(x);
            bl += l != lq;
            dl += l != sc::ddm::log_dd_full(x);
        }
        double y = (i % 65) / 64.0 + w(g);
        if (i & 1) y = 1.0 / y;
        if (y != 0.0 && std::fabs(y) < 1e300) {
            const double t = sc::ddm::atan_dd(y);
            ba += t != (double)atanq((__float128)y);
            da += t != sc::ddm::atan_dd_full(y);
        }
    }
    // a few exact cases
    bl += sc::ddm::log_dd(1.0) != 0.0;
    ba += sc::ddm::atan_dd(0.0) != 0.0;
    ba += sc::ddm::atan_dd(1.0) != (double)atanq((__float128)1.0);
    ba += sc::ddm::atan_dd(-1.0) != (double)atanq((__float128)-1.0);
    // the arguments the integrated Green's function evaluates: ln(x + r) and
    // atan(x y / (z r)) at the cell-corner offsets of a 40^3 grid with
    // unequal spacings (FFTPoissonSolver.cpp:472-493)
    long garg = 0, gquick = 0;
    const double h[3] = {1.1e-4, 0.9e-4, 3.7e-4};
    for (int i = 0; i < 40; ++i)
        for (int j = 0; j < 40; ++j)
            for (int k = 0; k < 40; ++k) {
                const double x = i * h[0] - h[0] / 2, y = j * h[1] - h[1] / 2, z = k * h[2] - h[2] / 2;
                const double r = std::sqrt(x * x + y * y + z * z);
                double o;
                const double log_args[3] = {x + r, y + r, z + r};
                const double atan_args[3] = {x * y / (z * r), x * z / (y * r), y * z / (x * r)};
                for (int m = 0; m < 3; ++m) {
                    garg += 2;
                    gquick += sc::ddm::log_quick(log_args[m], o);
                    gquick += sc::ddm::atan_quick(atan_args[m], o);
                }
            }
    std::printf("%ld %ld %ld %ld %ld %ld %ld %ld %ld %ld %ld\n", n, bl, ba, ll, la, dl, da, ql, qa, garg, gquick);
    return 0;
}
