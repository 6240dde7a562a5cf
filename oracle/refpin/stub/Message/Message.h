// Test infrastructure (oracle pinning).  A stand-in for IPPL's
// Message/Message.h, whose real header needs MPI: the reference's Vektor,
// Tenzor and PETE expression headers only name the message class in their
// (unused here) serialisation members, and call ERRORMSG / Ippl::abortAllNodes
// on dimension errors that 3-D code never reaches.  The reference's header
// chain also declares IPPL's output stream, which its users name.
#pragma once
#include <cstdlib>
#include <iostream>

#include "Utility/Inform.h"
using std::endl;
class Message {
public:
    template <class T> Message& put(const T&) { return *this; }
    template <class T> Message& get(T&) { return *this; }
    Message& setCopy(bool) { return *this; }
};
template <class T> inline void putMessage(Message&, const T&) {}
template <class I> inline void putMessage(Message&, I, I) {}
template <class T> inline void getMessage(Message&, T&) {}
template <class I> inline void getMessage(Message&, I, I) {}
#define ERRORMSG(x) (std::cerr << x)
struct Ippl {
    static void abortAllNodes(const char* = nullptr) { std::abort(); }
    static void abort(const char* = nullptr, int = 0) { std::abort(); }
};
