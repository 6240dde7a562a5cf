// Test infrastructure (oracle pinning).  A stand-in for IPPL's Inform
// stream (which needs the parallel runtime): CoordinateSystemTrafo only
// names it in its printing helpers.
#pragma once
#include <iostream>
class Inform {
public:
    std::ostream& getStream() { return std::cout; }
};
