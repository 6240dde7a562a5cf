// Test infrastructure (oracle pinning).  A stand-in for IPPL's random
// number generator (which pulls in the field library): getQuaternion draws
// from it only for anti-parallel vectors, a case the pinning inputs avoid
// and the product reports as an error.
#pragma once
struct PinRandom {
    unsigned long long s = 0x9e3779b97f4a7c15ull;
    double operator()() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (double)(s >> 11) * 0x1p-53;
    }
};
static PinRandom IpplRandom;
