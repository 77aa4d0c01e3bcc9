// Inner-tree layouts of the ordered traversals, built on the host from the
// flattened leaves of BVH::createBinary (Src/bvh.cpp:283-314, flattened by
// Src/meshmapping.cpp:62-125).  The leaves and their boxes are never changed:
// a traversal's result depends only on them, because an inner box is a union
// of its children's boxes and the slab test is monotone in the box, so any
// inner tree over the same leaves prunes only what the leaves' own tests
// would reject.
#include <algorithm>
#include <array>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "fk_internal.h"

namespace fk {
namespace {

struct Box {
  float lo[3], hi[3];
};

Box merge(const Box& a, const Box& b) {
  Box r;
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = std::min(a.lo[k], b.lo[k]);
    r.hi[k] = std::max(a.hi[k], b.hi[k]);
  }
  return r;
}

Box empty_box() {
  Box b;
  for (int k = 0; k < 3; ++k) {
    b.lo[k] = 3.4e38f;
    b.hi[k] = -3.4e38f;
  }
  return b;
}

// Half the surface area (all three face pairs, in double).
double half_area(const Box& b) {
  const double x = std::max(0.0, (double)b.hi[0] - b.lo[0]), y = std::max(0.0, (double)b.hi[1] - b.lo[1]),
               z = std::max(0.0, (double)b.hi[2] - b.lo[2]);
  return x * y + y * z + z * x;
}

void put_record(std::vector<float4>& wide, uint32_t rec, const Box& L, int32_t refL, int32_t cntL, const Box& R,
                int32_t refR, int32_t cntR) {
  float4* w = &wide[4 * (size_t)rec];
  w[0] = make_float4(L.lo[0], L.hi[0], L.lo[1], L.hi[1]);
  w[1] = make_float4(R.lo[0], R.hi[0], R.lo[1], R.hi[1]);
  w[2] = make_float4(L.lo[2], L.hi[2], R.lo[2], R.hi[2]);
  int32_t ints[4] = {refL, refR, cntL, cntR};
  float f[4];
  std::memcpy(f, ints, 16);
  w[3] = make_float4(f[0], f[1], f[2], f[3]);
}

struct Leaf {
  Box box;
  float c[3];      // box centre
  uint32_t flat;   // flattened node index
  uint32_t tris;
};

struct SahBuilder {
  std::vector<Leaf>& leaves;
  std::vector<float4>& wide;  // L - 1 records for L leaves, preallocated
  std::atomic<uint32_t> depth{1};
  static constexpr int kBins = 32;
  static constexpr uint32_t kParallelLeaves = 16384;  // smaller subtrees build on the calling thread

  // Builds the subtree over leaves [b, e) (e - b >= 2) into records
  // [rec, rec + e - b - 1): its root at rec, the left subtree (leaves [b, m))
  // from rec + 1, the right one from rec + (m - b).  Disjoint subtrees write
  // disjoint records, so the two halves of a large node build on two threads.
  // Returns the subtree's box; `level` counts the root as 1.
  Box build(uint32_t rec, uint32_t b, uint32_t e, uint32_t level) {
    const uint32_t m = split(b, e);
    Box boxes[2];
    int32_t refs[2], cnts[2];
    const uint32_t lo[2] = {b, m}, hi[2] = {m, e};
    const uint32_t kids[2] = {rec + 1, rec + (m - b)};
    std::thread side;
    for (int s = 0; s < 2; ++s) {
      if (hi[s] - lo[s] == 1) {
        const Leaf& l = leaves[lo[s]];
        boxes[s] = l.box;
        refs[s] = -(int32_t)l.flat - 1;
        cnts[s] = (int32_t)l.tris;
        raise_depth(level + 1);
        continue;
      }
      refs[s] = (int32_t)kids[s];
      cnts[s] = 0;
      if (s == 0 && hi[1] - lo[1] > 1 && hi[0] - lo[0] >= kParallelLeaves) {
        side = std::thread([this, &boxes, &kids, &lo, &hi, level] { boxes[0] = build(kids[0], lo[0], hi[0], level + 1); });
      } else {
        boxes[s] = build(kids[s], lo[s], hi[s], level + 1);
      }
    }
    if (side.joinable()) side.join();
    put_record(wide, rec, boxes[0], refs[0], cnts[0], boxes[1], refs[1], cnts[1]);
    return merge(boxes[0], boxes[1]);
  }

  void raise_depth(uint32_t d) {
    uint32_t cur = depth.load();
    while (d > cur && !depth.compare_exchange_weak(cur, d)) {
    }
  }

  // Binned SAH over box centres on all three axes (cost = half area x
  // triangles); partitions [b, e) and returns the split point.
  uint32_t split(uint32_t b, uint32_t e) {
    float cmin[3] = {3.4e38f, 3.4e38f, 3.4e38f}, cmax[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (uint32_t i = b; i < e; ++i)
      for (int k = 0; k < 3; ++k) {
        cmin[k] = std::min(cmin[k], leaves[i].c[k]);
        cmax[k] = std::max(cmax[k], leaves[i].c[k]);
      }
    double best = 1e300;
    int best_axis = -1, best_bin = 0;
    float scale[3];
    for (int k = 0; k < 3; ++k) {
      const float ext = cmax[k] - cmin[k];
      scale[k] = ext > 0.0f ? (float)kBins / ext : 0.0f;
    }
    for (int k = 0; k < 3; ++k) {
      if (!(scale[k] > 0.0f)) continue;
      std::array<Box, kBins> bb;
      std::array<double, kBins> bn{};
      bb.fill(empty_box());
      for (uint32_t i = b; i < e; ++i) {
        int q = (int)((leaves[i].c[k] - cmin[k]) * scale[k]);
        q = std::min(std::max(q, 0), kBins - 1);
        bb[q] = merge(bb[q], leaves[i].box);
        bn[q] += leaves[i].tris;
      }
      std::array<double, kBins> right_cost{};
      Box acc = empty_box();
      double n = 0;
      for (int q = kBins - 1; q > 0; --q) {
        acc = merge(acc, bb[q]);
        n += bn[q];
        right_cost[q] = n > 0 ? half_area(acc) * n : 0.0;
      }
      acc = empty_box();
      n = 0;
      for (int q = 0; q < kBins - 1; ++q) {
        acc = merge(acc, bb[q]);
        n += bn[q];
        if (n == 0 || right_cost[q + 1] == 0) continue;
        const double cost = half_area(acc) * n + right_cost[q + 1];
        if (cost < best) {
          best = cost;
          best_axis = k;
          best_bin = q;
        }
      }
    }
    uint32_t m = (b + e) / 2;
    if (best_axis >= 0) {
      const int k = best_axis;
      auto it = std::partition(leaves.begin() + b, leaves.begin() + e, [&](const Leaf& l) {
        int q = (int)((l.c[k] - cmin[k]) * scale[k]);
        q = std::min(std::max(q, 0), kBins - 1);
        return q <= best_bin;
      });
      m = (uint32_t)(it - leaves.begin());
      if (m == b || m == e) m = (b + e) / 2;
    }
    return m;
  }
};

}  // namespace

uint32_t build_sah_wide(const float4* lo, const float4* hi, const uint32_t* jump, uint32_t nn,
                        std::vector<float4>& wide) {
  std::vector<Leaf> leaves;
  for (uint32_t i = 0; i < nn; ++i) {
    if (jump[i] != i + 1) continue;
    Leaf l;
    l.box = {{lo[i].x, lo[i].y, lo[i].z}, {hi[i].x, hi[i].y, hi[i].z}};
    for (int k = 0; k < 3; ++k) l.c[k] = 0.5f * (l.box.lo[k] + l.box.hi[k]);
    l.flat = i;
    uint32_t s, e;
    std::memcpy(&s, &lo[i].w, 4);
    std::memcpy(&e, &hi[i].w, 4);
    l.tris = (e - s) / 3;
    leaves.push_back(l);
  }
  wide.clear();
  if (leaves.size() < 2) return 1;
  wide.resize(4 * (leaves.size() - 1));
  SahBuilder sb{leaves, wide};
  sb.build(0, 0, (uint32_t)leaves.size(), 1);
  return sb.depth.load();
}

void collapse_wide4(const std::vector<float4>& wide, std::vector<float4>& wide4, uint32_t& n4, uint32_t& depth4) {
  struct Ent {
    float lo[3], hi[3];
    int32_t ref;
  };
  wide4.clear();
  n4 = 0;
  depth4 = 0;
  if (wide.empty()) return;
  auto child = [&](uint32_t r, int k) {
    const float4* w = &wide[4 * (size_t)r];
    Ent e;
    if (k == 0) {
      e = {{w[0].x, w[0].z, w[2].x}, {w[0].y, w[0].w, w[2].y}, 0};
      std::memcpy(&e.ref, &w[3].x, 4);
    } else {
      e = {{w[1].x, w[1].z, w[2].z}, {w[1].y, w[1].w, w[2].w}, 0};
      std::memcpy(&e.ref, &w[3].y, 4);
    }
    return e;
  };
  std::vector<uint32_t> list{0};  // 2-wide records that become 4-wide nodes
  std::vector<uint32_t> lvl{1};
  std::vector<std::array<Ent, 4>> kids;
  std::vector<int> counts;
  for (size_t q = 0; q < list.size(); ++q) {
    std::array<Ent, 4> e{};
    int m = 0;
    for (int k = 0; k < 2; ++k) {
      Ent c = child(list[q], k);
      if (c.ref >= 0) {
        e[m++] = child((uint32_t)c.ref, 0);
        e[m++] = child((uint32_t)c.ref, 1);
      } else {
        e[m++] = c;
      }
    }
    for (int k = 0; k < m; ++k)
      if (e[k].ref >= 0) {
        const uint32_t r = (uint32_t)e[k].ref;
        e[k].ref = (int32_t)list.size();
        list.push_back(r);
        lvl.push_back(lvl[q] + 1);
      }
    for (int k = m; k < 4; ++k) e[k] = e[0];
    kids.push_back(e);
    counts.push_back(m);
    depth4 = std::max(depth4, lvl[q]);
  }
  n4 = (uint32_t)list.size();
  wide4.resize(8 * (size_t)n4);
  for (uint32_t k = 0; k < n4; ++k) {
    float4* w = &wide4[8 * (size_t)k];
    const auto& e = kids[k];
    for (int a = 0; a < 3; ++a) {
      w[2 * a] = make_float4(e[0].lo[a], e[1].lo[a], e[2].lo[a], e[3].lo[a]);
      w[2 * a + 1] = make_float4(e[0].hi[a], e[1].hi[a], e[2].hi[a], e[3].hi[a]);
    }
    float f[4];
    int32_t ints[4] = {e[0].ref, e[1].ref, e[2].ref, e[3].ref};
    std::memcpy(f, ints, 16);
    w[6] = make_float4(f[0], f[1], f[2], f[3]);
    int32_t cnt[4] = {counts[k], 0, 0, 0};
    std::memcpy(f, cnt, 16);
    w[7] = make_float4(f[0], f[1], f[2], f[3]);
  }
}

}  // namespace fk
