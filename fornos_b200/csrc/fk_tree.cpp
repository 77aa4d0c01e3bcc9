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
#include <system_error>
#include <thread>
#include <vector>

#include "fk_internal.h"
#include "fk_sah_rules.h"

namespace fk {
namespace {

using sah::key;
using sah::kmax;
using sah::kmin;
using sah::unkey;

// Box as float keys (fk_sah_rules.h): merging is a key min / max.
struct KBox {
  uint32_t lo[3], hi[3];
};

KBox merge(const KBox& a, const KBox& b) {
  KBox r;
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = kmin(a.lo[k], b.lo[k]);
    r.hi[k] = kmax(a.hi[k], b.hi[k]);
  }
  return r;
}

KBox empty_box() {
  KBox b;
  for (int k = 0; k < 3; ++k) {
    b.lo[k] = 0xffffffffu;
    b.hi[k] = 0u;
  }
  return b;
}

double half_area(const KBox& b) {
  return sah::half_area(unkey(b.lo[0]), unkey(b.hi[0]), unkey(b.lo[1]), unkey(b.hi[1]), unkey(b.lo[2]),
                        unkey(b.hi[2]));
}

void put_record(std::vector<float4>& wide, uint32_t rec, const KBox& L, int32_t refL, int32_t cntL, const KBox& R,
                int32_t refR, int32_t cntR) {
  float4* w = &wide[4 * (size_t)rec];
  w[0] = make_float4(unkey(L.lo[0]), unkey(L.hi[0]), unkey(L.lo[1]), unkey(L.hi[1]));
  w[1] = make_float4(unkey(R.lo[0]), unkey(R.hi[0]), unkey(R.lo[1]), unkey(R.hi[1]));
  w[2] = make_float4(unkey(L.lo[2]), unkey(L.hi[2]), unkey(R.lo[2]), unkey(R.hi[2]));
  int32_t ints[4] = {refL, refR, cntL, cntR};
  float f[4];
  std::memcpy(f, ints, 16);
  w[3] = make_float4(f[0], f[1], f[2], f[3]);
}

struct Leaf {
  KBox box;
  float c[3];      // box centre
  uint32_t flat;   // flattened node index
  uint32_t tris;
};

struct SahBuilder {
  std::vector<Leaf>& leaves;  // flattened-index order; every node's range stays in that order
  std::vector<float4>& wide;  // L - 1 records for L leaves, preallocated
  std::atomic<uint32_t> depth{1};
  static constexpr int kBins = sah::kBins;
  static constexpr uint32_t kParallelLeaves = 16384;  // smaller subtrees build on the calling thread

  // Builds the subtree over leaves [b, e) (e - b >= 2) into records
  // [rec, rec + e - b - 1): its root at rec, the left subtree (leaves [b, m))
  // from rec + 1, the right one from rec + (m - b).  Disjoint subtrees write
  // disjoint records, so the two halves of a large node build on two threads.
  // Returns the subtree's box; `level` counts the root as 1.
  KBox build(uint32_t rec, uint32_t b, uint32_t e, uint32_t level) {
    const uint32_t m = split(b, e);
    KBox boxes[2];
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
        try {
          side = std::thread([this, &boxes, &kids, &lo, &hi, level] { boxes[0] = build(kids[0], lo[0], hi[0], level + 1); });
        } catch (const std::system_error&) {  // no thread to be had: built here
          boxes[0] = build(kids[0], lo[0], hi[0], level + 1);
        }
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

  // Binned surface-area split of [b, e) over box centres on all three axes
  // (cost = half area x triangles, fk_sah_rules.h); stably partitions the
  // range and returns the split point.
  uint32_t split(uint32_t b, uint32_t e) {
    uint32_t cmin_k[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, cmax_k[3] = {0u, 0u, 0u};
    for (uint32_t i = b; i < e; ++i)
      for (int k = 0; k < 3; ++k) {
        cmin_k[k] = kmin(cmin_k[k], key(leaves[i].c[k]));
        cmax_k[k] = kmax(cmax_k[k], key(leaves[i].c[k]));
      }
    float cmin[3], scale[3];
    for (int k = 0; k < 3; ++k) {
      cmin[k] = unkey(cmin_k[k]);
      scale[k] = sah::bin_scale(unkey(cmax_k[k]) - cmin[k]);
    }
    double best = 1e300;
    int best_axis = -1, best_bin = 0;
    uint32_t best_left = 0;
    for (int k = 0; k < 3; ++k) {
      if (!(scale[k] > 0.0f)) continue;
      std::array<KBox, kBins> bb;
      std::array<uint32_t, kBins> bt{}, bc{};
      bb.fill(empty_box());
      for (uint32_t i = b; i < e; ++i) {
        const int q = sah::bin_of(leaves[i].c[k], cmin[k], scale[k]);
        bb[q] = merge(bb[q], leaves[i].box);
        bt[q] += leaves[i].tris;
        bc[q] += 1;
      }
      std::array<double, kBins> right_cost{};
      KBox acc = empty_box();
      uint32_t n = 0;
      for (int q = kBins - 1; q > 0; --q) {
        acc = merge(acc, bb[q]);
        n += bt[q];
        right_cost[q] = n > 0 ? half_area(acc) * (double)n : 0.0;
      }
      acc = empty_box();
      n = 0;
      uint32_t count = 0;
      for (int q = 0; q < kBins - 1; ++q) {
        acc = merge(acc, bb[q]);
        n += bt[q];
        count += bc[q];
        if (n == 0 || right_cost[q + 1] == 0.0) continue;
        const double cost = half_area(acc) * (double)n + right_cost[q + 1];
        if (cost < best) {
          best = cost;
          best_axis = k;
          best_bin = q;
          best_left = count;
        }
      }
    }
    if (best_axis < 0) return b + (e - b) / 2;  // no candidate plane: first half in flattened order
    const int k = best_axis;
    const float cm = cmin[k], sc = scale[k];
    std::stable_partition(leaves.begin() + b, leaves.begin() + e,
                          [&](const Leaf& l) { return sah::bin_of(l.c[k], cm, sc) <= best_bin; });
    return b + best_left;
  }
};

}  // namespace

uint32_t build_sah_wide(const float4* lo, const float4* hi, const uint32_t* jump, uint32_t nn,
                        std::vector<float4>& wide) {
  std::vector<Leaf> leaves;
  wide.clear();
  for (uint32_t i = 0; i < nn; ++i) {
    if (jump[i] != i + 1) continue;
    const float l3[3] = {lo[i].x, lo[i].y, lo[i].z}, h3[3] = {hi[i].x, hi[i].y, hi[i].z};
    Leaf l;
    for (int k = 0; k < 3; ++k) {
      if (!sah::coord_ok(l3[k]) || !sah::coord_ok(h3[k])) return 0;  // no rebuilt tree for this scene
      l.box.lo[k] = key(l3[k]);
      l.box.hi[k] = key(h3[k]);
      l.c[k] = sah::centre(l3[k], h3[k]);
    }
    l.flat = i;
    uint32_t s, e;
    std::memcpy(&s, &lo[i].w, 4);
    std::memcpy(&e, &hi[i].w, 4);
    l.tris = (e - s) / 3;
    leaves.push_back(l);
  }
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

extern "C" int fk_diag_sah_host(const fk_bvh_node* nodes, uint32_t nn, float* records, uint32_t capacity,
                                uint32_t* count, uint32_t* depth) {
  if (!nodes || nn == 0) return FK_ERR_INVALID;
  std::vector<float4> lo(nn), hi(nn);
  std::vector<uint32_t> jump(nn);
  for (uint32_t i = 0; i < nn; ++i) {
    const fk_bvh_node& n = nodes[i];
    if (n.jump <= i || n.jump > nn || n.start > n.end || (n.jump == i + 1) != (n.end > n.start)) return FK_ERR_INVALID;
    float fs, fe;
    std::memcpy(&fs, &n.start, 4);
    std::memcpy(&fe, &n.end, 4);
    lo[i] = make_float4(n.aabb_min[0], n.aabb_min[1], n.aabb_min[2], fs);
    hi[i] = make_float4(n.aabb_max[0], n.aabb_max[1], n.aabb_max[2], fe);
    jump[i] = n.jump;
  }
  std::vector<float4> wide;
  const uint32_t d = fk::build_sah_wide(lo.data(), hi.data(), jump.data(), nn, wide);
  const uint32_t n = (uint32_t)(wide.size() / 4);
  if (count) *count = n;
  if (depth) *depth = d;
  if (records) {
    if (capacity < n) return FK_ERR_INVALID;
    std::memcpy(records, wide.data(), sizeof(float4) * wide.size());
  }
  return FK_OK;
}
