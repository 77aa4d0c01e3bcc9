// Arithmetic of BVH::createBinary (Src/bvh.cpp:128-314) shared by the host
// build (fk_bvh.cpp) and the device build (fk_bvh_dev.cu), so that both give
// the same nodes bit for bit.
#pragma once
#include <cfloat>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define FK_BVH_HD __host__ __device__ __forceinline__
#else
#define FK_BVH_HD inline
#endif

namespace fk {
namespace bvh {

FK_BVH_HD bool negative(float x) {
#ifdef __CUDA_ARCH__
  return (__float_as_uint(x) >> 31) != 0;
#else
  uint32_t u;
  std::memcpy(&u, &x, 4);
  return (u >> 31) != 0;
#endif
}

// The build's min and max: the smaller / larger operand; a NaN operand loses
// (both NaN: the first); zeros of opposite sign give -0 for both.  That is
// what std::fmin / std::fmax return on the x86-64 hosts of this build
// (glibc's AVX-512 variants), written out so that it holds on every host and
// on the device.  Both are commutative and associative, so a fold over a set
// does not depend on its order: the extreme value, and -0 when that extreme
// is a zero and the set holds a -0.
FK_BVH_HD float fmin(float x, float y) {
  if (x < y) return x;
  if (y < x) return y;
  if (x == y) return negative(x) ? x : y;
  return (x != x) ? y : x;
}
FK_BVH_HD float fmax(float x, float y) {
  if (x > y) return x;
  if (y > x) return y;
  if (x == y) return negative(x) ? x : y;
  return (x != x) ? y : x;
}

// Bucket of a centroid coordinate (Src/bvh.cpp:146-150): 16 buckets over the
// centroid extent; a NaN position goes to bucket 0.
FK_BVH_HD uint32_t bucket(float c, float lo, float ext) {
  const float r = ((c - lo) / ext) * 15.99f;
  if (r != r) return 0;
  const uint32_t k = (uint32_t)r;
  return k > 15 ? 15 : k;
}

// Split cost of Src/bvh.cpp:63-68 (x*y appears twice in the area term).
FK_BVH_HD float cost(float ex, float ey, float ez, int n) {
  return float(n) * (2.0f * (ex * ey + ex * ez + ex * ey));
}

// Split choice of Src/bvh.cpp:128-203 from the 16 buckets per axis: bucket
// boxes (lo / hi per axis) and triangle counts, the node's triangle count n
// and its centroid box.  Sweeps each axis (right-side boxes grown from the
// last bucket, the left side grown bucket by bucket, the first strict minimum
// of the 15 proper splits), takes the cheapest axis (x, then y, then z on ties)
// and returns the split value at that bucket's upper boundary.  The all-left
// step (bucket 15) has an empty right side: its cost is NaN and it never wins
// (the reference reads past its table there).
FK_BVH_HD void pick_split(const float (*blo)[16][3], const float (*bhi)[16][3], const uint32_t (*cnt)[16], int n,
                          const float* clo, const float* chi, int* axis, float* value) {
  float best_cost[3];
  int best_idx[3];
  for (int a = 0; a < 3; ++a) {
    float rlo[15][3], rhi[15][3];
    for (int q = 0; q < 3; ++q) {
      rlo[14][q] = blo[a][15][q];
      rhi[14][q] = bhi[a][15][q];
    }
    for (int k = 13; k >= 0; --k)
      for (int q = 0; q < 3; ++q) {  // join(right[k + 1], bucket k + 1)
        rlo[k][q] = fmin(blo[a][k + 1][q], rlo[k + 1][q]);
        rhi[k][q] = fmax(bhi[a][k + 1][q], rhi[k + 1][q]);
      }
    float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    int nl = 0, nr = n;
    float best = FLT_MAX;
    int bi = 0;
    for (int k = 0; k < 15; ++k) {
      nl += (int)cnt[a][k];
      nr -= (int)cnt[a][k];
      for (int q = 0; q < 3; ++q) {  // join(left, bucket k)
        llo[q] = fmin(blo[a][k][q], llo[q]);
        lhi[q] = fmax(bhi[a][k][q], lhi[q]);
      }
      const float c = cost(lhi[0] - llo[0], lhi[1] - llo[1], lhi[2] - llo[2], nl) +
                      cost(rhi[k][0] - rlo[k][0], rhi[k][1] - rlo[k][1], rhi[k][2] - rlo[k][2], nr);
      if (c < best) {
        best = c;
        bi = k;
      }
    }
    best_cost[a] = best;
    best_idx[a] = bi;
  }
  int ax;
  if (best_cost[0] <= best_cost[1] && best_cost[0] <= best_cost[2]) ax = 0;
  else if (best_cost[1] <= best_cost[0] && best_cost[1] <= best_cost[2]) ax = 1;
  else ax = 2;
  *axis = ax;
  *value = clo[ax] + (chi[ax] - clo[ax]) / 16.0f * float(best_idx[ax] + 1);
}

}  // namespace bvh
}  // namespace fk
