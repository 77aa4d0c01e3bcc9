// Force-included when compiling the reference's host sources on Linux / g++.
// Test infrastructure only (oracle/build_ref.py).
//
// * The reference calls std::sqrtf / std::cosf / std::sinf / std::fabsf, which
//   MSVC provides and libstdc++ does not; they are forwarded to the C library.
// * Src/math.h:365 seeds the sample-table engine from std::random_device; the
//   oracle needs a reproducible table, so that name is redirected to a device
//   that returns the seed set by ref_set_seed() (ref_host_driver.cpp).
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <random>
#include <string>

namespace std {
inline float sqrtf(float x) { return ::sqrtf(x); }
inline float cosf(float x) { return ::cosf(x); }
inline float sinf(float x) { return ::sinf(x); }
inline float fabsf(float x) { return ::fabsf(x); }
struct fornos_seeded_device {
  unsigned int operator()();
};
}  // namespace std
using std::isnan;

#define random_device fornos_seeded_device
