// Boost.Random API shim: the reference's CPU solvers only declare a time-seeded
// boost::random::mt19937 (reference code/PrunedDP++/src/main.cpp:7-8) and never
// draw from it on the solver path.  std::mt19937 has the same published
// definition (Matsumoto & Nishimura 1998, 32-bit MT19937).
#pragma once
#include <cstdint>
#include <ctime>
#include <random>
namespace boost {
namespace random {
typedef std::mt19937 mt19937;
}  // namespace random
}  // namespace boost
