// Host stand-in for <cuda_runtime.h>, so that fornos_b200/csrc/fk_device.cuh
// compiles with g++ for the box-test fuzzer: the device qualifiers vanish and
// each IEEE-rounded intrinsic becomes the same single operation in host
// float arithmetic (SSE, no contraction: build with -ffp-contract=off).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#define __device__
#define __host__
#define __forceinline__ inline

struct float4 {
  float x, y, z, w;
};
struct int2 {
  int x, y;
};
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }

inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
inline float __frcp_rn(float a) { return 1.0f / a; }
inline float __fsqrt_rn(float a) { return std::sqrt(a); }
inline float __fmaf_rn(float a, float b, float c) { return std::fma(a, b, c); }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __ddiv_rn(double a, double b) { return a / b; }
inline float __double2float_rn(double a) { return (float)a; }
inline float __int_as_float(int v) { float f; std::memcpy(&f, &v, 4); return f; }
inline int __float_as_int(float f) { int v; std::memcpy(&v, &f, 4); return v; }
using std::fabs;
inline float fabsf(float a) { return std::fabs(a); }
inline float fminf(float a, float b) { return std::fmin(a, b); }
inline float fmaxf(float a, float b) { return std::fmax(a, b); }
