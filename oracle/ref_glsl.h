// GLSL 4.30 vocabulary for compiling the reference's compute shaders
// (Shaders/*.comp) as C++ on the host.  Used only by oracle/build_ref.py, which
// rewrites each shader's declarations (buffers, uniforms, in/out parameters) and
// compiles it against this header into oracle/_ref.  Test infrastructure only.
//
// Semantics follow the arithmetic contract of the oracle: binary32 operations in
// source order without contraction, correctly rounded division and sqrt,
// min/max = fminf/fmaxf, normalize(v) = v * (1 / sqrt(dot(v, v))), dot summed
// left to right.  vec3 is 16 bytes so that std430 arrays of vec3 and structs of
// vec3 (Shaders/ao_step0.comp:7-13) have the layout the host uploads
// (Src/meshmapping.h:15-31, Src/solver_ao.h:75-81).
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>

namespace glsl {

typedef unsigned int uint;

struct dvec3;

struct alignas(16) vec3 {
  float x, y, z;
  vec3() : x(0), y(0), z(0) {}
  vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  explicit vec3(const dvec3& d);
};

struct alignas(16) vec4 {
  float x, y, z, w;
  vec4() : x(0), y(0), z(0), w(0) {}
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  vec3 yzw() const { return vec3(y, z, w); }
};

struct dvec3 {
  double x, y, z;
  dvec3() : x(0), y(0), z(0) {}
  dvec3(double a, double b, double c) : x(a), y(b), z(c) {}
  dvec3(const vec3& v) : x(v.x), y(v.y), z(v.z) {}
};

inline vec3::vec3(const dvec3& d) : x((float)d.x), y((float)d.y), z((float)d.z) {}

struct uvec3 { uint x, y, z; };

inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3 operator*(const vec3& a, float k) { return vec3(a.x * k, a.y * k, a.z * k); }
inline vec3 operator*(float k, const vec3& a) { return vec3(k * a.x, k * a.y, k * a.z); }
inline vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline vec3& operator+=(vec3& a, const vec3& b) { a = a + b; return a; }
inline dvec3 operator-(const dvec3& a, const dvec3& b) { return dvec3(a.x - b.x, a.y - b.y, a.z - b.z); }

inline float abs(float v) { return std::fabs(v); }
inline vec3 abs(const vec3& v) { return vec3(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double dot(const dvec3& a, const dvec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
  return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }

extern thread_local uvec3 gl_GlobalInvocationID;

}  // namespace glsl
