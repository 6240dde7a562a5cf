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
SC_DDM_HD double log_dd_full(double x) {
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
SC_DDM_HD double atan_dd_full(double x) {
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

// ---------------------------------------------------------------- quick phase
// Ziv's strategy (as in CRlibm, Daramy-Loirat et al.): a cheaper evaluation
// whose result hi + lo carries a relative error below kQuickEps; when that
// error cannot move the value across a rounding boundary, hi is the
// correctly rounded result, otherwise the full double-double evaluation
// above decides.  log and atan of a double other than log 1, atan 0 are
// transcendental, never exactly halfway between two doubles.  The quick
// phase accepts only values at least 2^-10 ulp from a boundary, where the
// full evaluation is correctly rounded too, so both phases give the same
// bits.
//
// Error budget of both quick phases, relative to the result v: the
// argument reduction t = th + tl is exact to 2^-103; the polynomial tail
// above the last exactly summed term is below 2^-14.5 |v| and is evaluated
// with a relative error under 2^-51; the low-order words (at most about
// ten, each below 2^-14.5 |v|) are added in double with at most 2^-53 of
// their partial sums per addition.  Together about 2^-65 |v| at worst (the
// largest error seen against quad precision, over 2e7 arguments spread over
// every table interval, is 2^-65.5); the test allows 2^-63.
constexpr double kQuickEps = 0x1p-63;

// RN(hi + lo + d) == hi for every |d| <= eps |hi|, with |lo| <= ulp(hi) / 2
// and hi normal; powers of two (a smaller ulp below) are left to the full
// evaluation.
SC_DDM_HD bool rounds_to_hi(double hi, double lo, double eps) {
    uint64_t b;
    memcpy(&b, &hi, sizeof b);
    if ((b & 0x000fffffffffffffull) == 0) return false;
    b &= 0x7ff0000000000000ull;
    if (b < 0x07b0000000000000ull) return false;  // |hi| < 2^-900: left to the full evaluation
    double half_ulp;
    memcpy(&half_ulp, &b, sizeof half_ulp);
    half_ulp *= 0x1p-53;
    return fabs(lo) + eps * fabs(hi) < half_ulp;
}

// Quick log: the reduction of log_dd_full; log1p t = t - t^2/2 + t^3 q(t)
// with t^2 exact (TwoProd) and t^3 q(t) in double; k log2 + log c + th -
// th^2/2 by exact TwoSums, the rest as one double.
SC_DDM_HD bool log_quick(double x, double& out) {
    uint64_t bits;
    memcpy(&bits, &x, sizeof bits);
    int k = (int)(bits >> 52) - 1023;
    bits = (bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    double m;
    memcpy(&m, &bits, sizeof m);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        k += 1;
    }
    const int j = (int)rint(m * 64.0);
    const double c = (double)j / 64.0;
    const double u = m - c;
    const double rc = kLogRcp[j - kLogJ0];
    const double th = u * rc;
    const double tl = fma(-th, c, u) * rc;  // |t| < 2^-6.49
    // q(t) = 1/3 - t/4 + t^2/5 - ... + t^8/11 (terms to t^11 of log1p)
    double q = fma(th, 1.0 / 11.0, -1.0 / 10.0);
    q = fma(th, q, 1.0 / 9.0);
    q = fma(th, q, -1.0 / 8.0);
    q = fma(th, q, 1.0 / 7.0);
    q = fma(th, q, -1.0 / 6.0);
    q = fma(th, q, 1.0 / 5.0);
    q = fma(th, q, -1.0 / 4.0);
    q = fma(th, q, 1.0 / 3.0);
    const double p = th * th, pe = fma(th, th, -p);
    const double cubic = (p * th) * q;
    const double kd = (double)k;
    const dd s1 = two_sum(kd * kLn2Hi, kLogTab[j - kLogJ0][0]);
    const dd s2 = two_sum(s1.hi, th);
    const dd s3 = two_sum(s2.hi, -0.5 * p);
    double lo = -(th * tl) - 0.5 * pe;
    lo += tl;
    lo += kLogTab[j - kLogJ0][1];
    lo += kd * kLn2Lo;
    lo += s1.lo + s2.lo + s3.lo;
    lo += cubic;
    const dd r = fast_two_sum(s3.hi, lo);
    if (!rounds_to_hi(r.hi, r.lo, kQuickEps)) return false;
    out = r.hi;
    return true;
}

// Reciprocal of d in [1, 2^31] to about 2^-52: the float reciprocal and two
// Newton steps.
SC_DDM_HD double rcp_approx(double d) {
    double r = (double)(1.0f / (float)d);
    r = fma(r, fma(-d, r, 1.0), r);
    r = fma(r, fma(-d, r, 1.0), r);
    return r;
}

// Quick atan for 2^-30 <= |x| <= 2^30: the reduction of atan_dd_full with
// t = num / den to 2^-103 from one approximate reciprocal and the exact
// residual, atan t = t + t^3 p(t^2) in double, atan c + th by TwoSum (and
// pi/2 - that for |x| > 1).
SC_DDM_HD bool atan_quick(double x, double& out) {
    const double a = fabs(x);
    const bool inv = a > 1.0;
    // j = round(64 s), s = min(a, 1/a); a float 1/a may pick the neighbour
    // of round(64/a), which keeps |t| below 2^-6.99
    const int j = inv ? (int)rintf(64.0f / (float)a) : (int)rint(a * 64.0);
    const double c = (double)j / 64.0;
    double nh, nl, dh, dl;
    if (inv) {
        // 1 - a c may cancel to far below a c's low word: renormalise
        const dd ac = two_prod(a, c);
        const dd n = two_sum(1.0, -ac.hi);
        const dd nn = two_sum(n.hi, n.lo - ac.lo);
        nh = nn.hi;
        nl = nn.lo;
        const dd d = two_sum(a, c);
        dh = d.hi;
        dl = d.lo;
    } else {
        nh = a - c;  // exact (Sterbenz, or c = 0)
        nl = 0.0;
        const dd ac = two_prod(a, c);
        const dd d = two_sum(1.0, ac.hi);
        dh = d.hi;
        dl = d.lo + ac.lo;
    }
    const double rd = rcp_approx(dh);
    const double th = nh * rd;
    const double res = fma(-th, dh, nh) + (nl - th * dl);
    const double tl = res * rd;
    // atan t - t = t^3 (-1/3 + t^2/5 - t^4/7 + t^6/9 - t^8/11)
    const double h2 = th * th;
    double pq = fma(h2, -1.0 / 11.0, 1.0 / 9.0);
    pq = fma(h2, pq, -1.0 / 7.0);
    pq = fma(h2, pq, 1.0 / 5.0);
    pq = fma(h2, pq, -1.0 / 3.0);
    const double tail = (h2 * th) * pq;
    const dd s1 = two_sum(kAtanTab[j][0], th);
    double lo = tl + tail;
    lo += kAtanTab[j][1];
    lo += s1.lo;
    double hi = s1.hi;
    if (inv) {
        const dd s2 = two_sum(kPiHalfHi, -hi);
        lo = (kPiHalfLo - lo) + s2.lo;
        hi = s2.hi;
    }
    const dd r = fast_two_sum(hi, lo);
    if (!rounds_to_hi(r.hi, r.lo, kQuickEps)) return false;
    out = x < 0.0 ? -r.hi : r.hi;
    return true;
}

// Correctly rounded log and atan (the quick phase, else the full evaluation).
SC_DDM_HD double log_dd(double x) {
    double r;
    if (x >= 2.2250738585072014e-308 && x <= 1.7976931348623157e308 && x != 1.0 && log_quick(x, r)) return r;
    return log_dd_full(x);
}

SC_DDM_HD double atan_dd(double x) {
    const double a = fabs(x);
    double r;
    if (a >= 9.3132257461547852e-10 && a <= 1073741824.0 && atan_quick(x, r)) return r;
    return atan_dd_full(x);
}

}  // namespace ddm
}  // namespace sc
