// sc_ddmath.cuh -- natural logarithm and arctangent evaluated in
// double-double arithmetic and rounded once to double.
//
// The integrated Green's function (FFTPoissonSolver.cpp:472-493) cancels
// eight antiderivative values per mesh point, so a one-ulp difference in a
// single log or atan moves the field by about 1e-11 of its maximum.  Two
// libraries that round differently (glibc on the host, CUDA on the device)
// therefore disagree at that level.  These versions carry about 2^-100 of
// relative accuracy until the last rounding, so they return the correctly
// rounded result except when the exact value lies within roughly 2^-20 ulp
// of a rounding boundary; they use only +, -, *, /, sqrt-free fma, and table
// reads, and give the same bits on the host and on the device.
//
// Methods:
//   * error-free transformations TwoSum (Knuth), Fast2Sum (Dekker) and
//     TwoProd by fused multiply-add; double-double add / multiply / divide
//     after Dekker (1971) and the QD library's "accurate" variants.
//   * log: x = 2^k m, m in [sqrt(1/2), sqrt(2)); c = round(64 m) / 64;
//     log x = k log 2 + log c + log1p((m - c) / c)  (table-driven, after
//     Tang, "Table-driven implementation of the logarithm function", 1990).
//   * atan: s = |x| or 1/|x|; c = round(64 s) / 64;
//     atan s = atan c + atan((s - c) / (1 + s c)); pi/2 - atan(1/|x|) for |x| > 1.
//   Tables of log(j/64) and atan(j/64) as (hi, lo) pairs come from mpmath at
//   200 bits (gen_ddmath_tables.py).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define SC_DDM_HD __host__ __device__ __forceinline__
#define SC_DDM_TABLE static __device__ const
#else
#define SC_DDM_HD static inline
#define SC_DDM_TABLE static const
#endif

#include "sc_ddmath_tables.h"

namespace sc {
namespace ddm {

struct dd {
    double hi, lo;
};

SC_DDM_HD dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return dd{s, e};
}

// requires |a| >= |b| (or a == 0)
SC_DDM_HD dd fast_two_sum(double a, double b) {
    const double s = a + b;
    const double e = b - (s - a);
    return dd{s, e};
}

SC_DDM_HD dd two_prod(double a, double b) {
    const double p = a * b;
    return dd{p, fma(a, b, -p)};
}

SC_DDM_HD dd neg(dd a) { return dd{-a.hi, -a.lo}; }

// "Sloppy" double-double addition: relative error about 2^-105 (|a| + |b|) /
// |a + b|.  Every sum below either has no cancellation, or (the residuals of
// div) only needs its result to 2^-53 relative.
SC_DDM_HD dd add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return fast_two_sum(s.hi, s.lo);
}

SC_DDM_HD dd mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return fast_two_sum(p.hi, p.lo);
}

SC_DDM_HD dd mul_d(dd a, double b) {
    dd p = two_prod(a.hi, b);
    p.lo += a.lo * b;
    return fast_two_sum(p.hi, p.lo);
}

// a / b from one hardware division: q1 = a.hi (1 / b.hi) is within a few ulp
// of the quotient, and two correction terms from the exact residuals
// a - b (q1 + q2) bring the result to about 2^-100 relative.
SC_DDM_HD dd div(dd a, dd b) {
    const double inv = 1.0 / b.hi;
    const double q1 = a.hi * inv;
    dd r = add(a, neg(mul_d(b, q1)));
    const double q2 = r.hi * inv;
    r = add(r, neg(mul_d(b, q2)));
    const double q3 = r.hi * inv;
    return add(fast_two_sum(q1, q2), dd{q3, 0.0});
}

SC_DDM_HD dd tab(const double (*t)[2], int i) { return dd{t[i][0], t[i][1]}; }

// log(x) for finite normal x > 0; other inputs go to the library function.
SC_DDM_HD double log_dd(double x) {
    if (!(x >= 2.2250738585072014e-308) || !(x <= 1.7976931348623157e308)) return log(x);
    uint64_t bits;
    memcpy(&bits, &x, sizeof bits);
    int k = (int)(bits >> 52) - 1023;
    bits = (bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    double m;
    memcpy(&m, &bits, sizeof m);  // [1, 2)
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        k += 1;
    }
    const int j = (int)rint(m * 64.0);  // 45 .. 91
    const double c = (double)j / 64.0;
    const double u = m - c;  // exact (Sterbenz)
    // t = u / c: th from the tabulated reciprocal, tl from the exact residual
    const double rc = kLogRcp[j - kLogJ0];
    const double th = u * rc;
    const double tl = fma(-th, c, u) * rc;
    const dd t = fast_two_sum(th, tl);     // |t| < 0.0112
    // log1p t = t - t^2/2 + t^3/3 + t^4 (-1/4 + t/5 - ... - t^8/12)
    const double h = t.hi;
    double p = -1.0 / 12.0;
    p = p * h + 1.0 / 11.0;
    p = p * h - 1.0 / 10.0;
    p = p * h + 1.0 / 9.0;
    p = p * h - 1.0 / 8.0;
    p = p * h + 1.0 / 7.0;
    p = p * h - 1.0 / 6.0;
    p = p * h + 1.0 / 5.0;
    p = p * h - 1.0 / 4.0;
    const dd t2 = mul(t, t);
    const dd t3 = mul(t2, t);
    const double h2 = h * h;
    dd s = add(t, dd{-0.5 * t2.hi, -0.5 * t2.lo});
    s = add(s, mul(t3, dd{kThirdHi, kThirdLo}));
    s = add(s, dd{(h2 * h2) * p, 0.0});
    const double kd = (double)k;
    dd r = add(dd{kd * kLn2Hi, 0.0}, two_prod(kd, kLn2Lo));
    r = add(r, dd{kd * kLn2Lo2, 0.0});
    r = add(r, tab(kLogTab, j - kLogJ0));
    r = add(r, s);
    return r.hi;
}

// atan(x) for finite x; NaN and infinities go to the library function.
SC_DDM_HD double atan_dd(double x) {
    const double a = fabs(x);
    if (!(a <= 1.7976931348623157e308)) return atan(x);
    if (a < 9.3132257461547852e-10) return x;  // |x| < 2^-30: x^3/3 is below half an ulp of x
    // s = min(a, 1/a); c = j/64 near s; atan s = atan c + atan t with
    //   a <= 1: t = (a - c) / (1 + a c)
    //   a >  1: t = (1/a - c) / (1 + c/a) = (1 - a c) / (a + c)
    // numerator and denominator are exact double-doubles (TwoProd, TwoSum).
    const bool inv = a > 1.0;
    const double s = inv ? 1.0 / a : a;
    const int j = (int)rint(s * 64.0);  // 0 .. 64
    const double c = (double)j / 64.0;
    dd num, den;
    if (inv) {
        const dd ac = two_prod(a, c);
        num = add(dd{1.0, 0.0}, neg(ac));
        den = two_sum(a, c);
    } else {
        num = dd{a - c, 0.0};  // exact (Sterbenz, or c = 0)
        den = add(dd{1.0, 0.0}, two_prod(a, c));
    }
    const dd t = div(num, den);  // |t| < 2^-7
    // atan t = t - t^3/3 + t^5 (1/5 - t^2/7 + t^4/9 - t^6/11)
    const double h = t.hi, h2 = h * h;
    double p = -1.0 / 11.0;
    p = p * h2 + 1.0 / 9.0;
    p = p * h2 - 1.0 / 7.0;
    p = p * h2 + 1.0 / 5.0;
    const dd t3 = mul(mul(t, t), t);
    dd r = add(t, mul(t3, dd{-kThirdHi, -kThirdLo}));
    r = add(r, dd{(h2 * h2 * h) * p, 0.0});
    r = add(r, tab(kAtanTab, j));
    if (inv) r = add(dd{kPiHalfHi, kPiHalfLo}, neg(r));
    return x < 0.0 ? -r.hi : r.hi;
}

}  // namespace ddm
}  // namespace sc
