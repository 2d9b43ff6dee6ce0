// Oracle (test infrastructure only): stand-in for the reference's
// src/basic/types.h, with just what src/assemble/assembler.h uses, so that
// the reference's own assembler<N>::applyCoeff_ compiles here.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <numeric>
#include <stdexcept>
#include <unordered_set>
#include <vector>

using label = int;
using scalar = double;

#ifndef STK_ThrowAssert
#define STK_ThrowAssert(expr) \
  do {                        \
    if (!(expr)) throw std::runtime_error("STK_ThrowAssert: " #expr); \
  } while (0)
#endif
#ifndef STK_ThrowAssertMsg
#define STK_ThrowAssertMsg(expr, msg) STK_ThrowAssert(expr)
#endif
