// Rules of the surface-area inner tree, shared by the host builder
// (fk_tree.cpp) and the device builder (fk_sah.cu) so both produce the same
// records bit for bit.
//
// The tree is a function of the leaf set alone: a node's split depends only
// on which leaves it holds (min / max and integer sums do not depend on
// order), partitions are stable so every node's leaves stay in flattened-index
// order, and the fallback split (no candidate plane) takes the first half in
// that order.  Floats are merged in the total order of their keys (-0 below
// +0), so signed zeros cannot make the two builders disagree either.
#pragma once
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define FK_SAH_HD __host__ __device__ __forceinline__
#else
#define FK_SAH_HD inline
#endif

namespace fk {
namespace sah {

constexpr int kBins = 32;
// Leaf boxes with a coordinate that is not finite or not below this in
// magnitude get no rebuilt tree (centres, extents and bin positions of the
// others cannot overflow).
constexpr float kMaxCoord = 1e30f;

// Order-preserving key of a float: unsigned order of keys = total order of
// floats with -0 below +0.
FK_SAH_HD uint32_t key(float f) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  std::memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

FK_SAH_HD float unkey(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}

FK_SAH_HD uint32_t kmin(uint32_t a, uint32_t b) { return a < b ? a : b; }
FK_SAH_HD uint32_t kmax(uint32_t a, uint32_t b) { return a > b ? a : b; }

FK_SAH_HD float centre(float lo, float hi) { return 0.5f * (lo + hi); }

FK_SAH_HD float bin_scale(float extent) { return extent > 0.0f ? (float)kBins / extent : 0.0f; }

// Bin of a centre coordinate; NaN (a zero offset times an infinite scale)
// goes to bin 0 and infinity to the last bin.
FK_SAH_HD int bin_of(float c, float cmin, float scale) {
  const float v = (c - cmin) * scale;
  return v >= (float)(kBins - 1) ? kBins - 1 : (v > 0.0f ? (int)v : 0);
}

// Half the surface area of a box (all three face pairs), in double.
FK_SAH_HD double half_area(float lx, float hx, float ly, float hy, float lz, float hz) {
  double x = (double)hx - lx, y = (double)hy - ly, z = (double)hz - lz;
  x = x > 0.0 ? x : 0.0;
  y = y > 0.0 ? y : 0.0;
  z = z > 0.0 ? z : 0.0;
  return x * y + y * z + z * x;
}

FK_SAH_HD bool coord_ok(float x) { return x > -kMaxCoord && x < kMaxCoord; }

// Cost of splitting after bin q: left box area x left triangles + the right
// side's cost; a candidate needs triangles on the left and a non-zero right
// cost.  Candidates are compared axis by axis (x, y, z), bin by bin, and the
// first strict minimum wins.

}  // namespace sah
}  // namespace fk
