// sc_exact.cuh -- order-independent (exact) sums of doubles on the device.
//
// Every double v with |v| < 2^55 becomes the 128-bit integer
// trunc(v * 2^72); integer addition is exact and associative, so a sum over
// particles does not depend on the order the particles are visited in (the
// particle arrays are reordered by cell every few steps).  The total is
// rounded to a double once.  Parts below 2^-72 (2e-22) are dropped, far
// below the rounding of any sum the step forms.
#pragma once

#include <cstdint>

namespace sc {

using i128 = __int128;
using u128 = unsigned __int128;

constexpr int kExFrac = 72;

__device__ __forceinline__ i128 ex_from(double v) {
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    const int e = (int)((bits >> 52) & 0x7ff);
    if (e == 0) return 0;  // zero or subnormal
    const unsigned long long m = (bits & 0xfffffffffffffull) | (1ull << 52);
    // v = m * 2^(e - 1075); fixed = m * 2^(e - 1075 + kExFrac)
    const int sh = e - 1075 + kExFrac;
    u128 mag;
    if (sh >= 0)
        mag = sh < 75 ? ((u128)m << sh) : ((u128)m << 74);  // |v| >= 2^55 saturates (out of contract)
    else
        mag = sh > -53 ? (u128)(m >> (-sh)) : (u128)0;
    return (bits >> 63) ? -(i128)mag : (i128)mag;
}

// correctly rounded double of x * 2^-kExFrac
__device__ __forceinline__ double ex_to_double(i128 x) {
    const bool neg = x < 0;
    const u128 m = neg ? (u128)(-x) : (u128)x;
    const unsigned long long hi = (unsigned long long)(m >> 64), lo = (unsigned long long)m;
    double r;
    if (hi == 0) {
        r = __ull2double_rn(lo);
    } else {
        const int lz = __clzll(hi);
        const unsigned long long top = lz ? ((hi << lz) | (lo >> (64 - lz))) : hi;
        const unsigned long long rest = lo << lz;
        unsigned long long mant = top >> 11;
        const unsigned long long rem = top & 0x7ffull;
        if (rem > 0x400ull || (rem == 0x400ull && (rest != 0 || (mant & 1ull)))) mant += 1;
        r = ldexp((double)mant, 75 - lz);
    }
    return ldexp(neg ? -r : r, -kExFrac);
}

__device__ __forceinline__ i128 ex_shfl_down(i128 v, int off) {
    const u128 u = (u128)v;
    const unsigned long long lo = __shfl_down_sync(0xffffffffu, (unsigned long long)u, off);
    const unsigned long long hi = __shfl_down_sync(0xffffffffu, (unsigned long long)(u >> 64), off);
    return (i128)(((u128)hi << 64) | lo);
}

// ---------------------------------------------------------------- deposit
// Exact sums of the scattered charges: each charge v (|v| <= |q dt|) becomes
// the integer t = rint(v * 2^(52 - E)) with 2^E > 2 |q dt|, so |t| < 2^51;
// the sums are integer additions, exact, so any order gives the same total,
// which is rounded to a double once.  The rounding of t is at most 2^-52 of
// one particle's charge.
constexpr int kFxFrac = 52;

__device__ __forceinline__ int fx_exponent(double qdt) { return qdt != 0.0 ? ilogb(qdt) + 2 : 0; }

// correctly rounded double of the 128-bit accumulator (lo, hi), times unit
__device__ __forceinline__ double acc_to_double(unsigned long long lo, unsigned long long hi, double unit) {
    const long long shi = (long long)hi;
    if (shi == ((long long)lo < 0 ? -1 : 0)) return __ll2double_rn((long long)lo) * unit;  // fits in 64 bits
    const bool neg = shi < 0;
    unsigned long long mlo = lo, mhi = hi;
    if (neg) {
        mlo = ~mlo + 1ull;
        mhi = ~mhi + (mlo == 0 ? 1ull : 0ull);
    }
    const int lz = __clzll(mhi);
    const unsigned long long top = lz ? ((mhi << lz) | (mlo >> (64 - lz))) : mhi;
    const unsigned long long rest = mlo << lz;
    unsigned long long mant = top >> 11;
    const unsigned long long rem = top & 0x7ffull;
    if (rem > 0x400ull || (rem == 0x400ull && (rest != 0 || (mant & 1ull)))) mant += 1;
    const double r = ldexp((double)mant, 75 - lz);
    return (neg ? -r : r) * unit;
}

// The charge density of one node from its accumulator (L, H) = H 2^32 + L:
// (exact node sum) / dT * tmp2 (PartBunch.cpp:496, :510-511).  Only a
// product and a quotient: no contraction can change its rounding.
__device__ __forceinline__ double node_density(ulonglong2 a, double unit, double dT, double tmp2) {
    const i128 w = (i128)(long long)a.y * (i128)4294967296 + (i128)a.x;
    double s = acc_to_double((unsigned long long)w, (unsigned long long)(w >> 64), unit);
    s /= dT;
    s *= tmp2;
    return s;
}

}  // namespace sc
