// Forced-included ahead of the Lucid reference sources (g++ -include).  The
// reference calls std::ldexpf (math/random.hpp:119), which libc++ (the
// reference's Apple Clang toolchain) declares in namespace std and GCC 13's
// libstdc++ does not; it is the C library's ldexpf either way.
#pragma once
#include <cmath>
#include <math.h>
namespace std {
using ::ldexpf;
}
