// Host side of the scene upload (fk_layout.h): three passes over node ranges,
// one host thread per range, and a scan in node order for the tree depth
// (on a thread of its own beside the last two passes when there are several
// ranges).  A range whose thread cannot be started runs on the calling thread.
//
//   1. each range checks its nodes, writes their device layout and counts
//      leaves and inner nodes; the first defect of each range is kept, so
//      the earliest over all ranges is the one a scan in node order meets;
//   2. from the counts' prefix sums, each range numbers its inner records
//      and lists its leaves;
//   3. each range writes its inner nodes' records, which read both children
//      (the right child lies anywhere after the left subtree, so this pass is
//      bound by cache misses and gains the most from the threads).
#include "fk_layout.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <system_error>
#include <thread>

#include "fk_sah_rules.h"

namespace fk {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr float kFilterLimit = 16777216.0f;  // 2^24: box coordinates the filtered box tests accept

struct RangeScan {
  uint32_t bad = kNone;    // first node outside the array, with a partial triangle, or with children and triangles
  bool mixed = false;      // that node has both children and triangles
  uint32_t split = kNone;  // first inner node whose children do not split its subtree
  uint32_t leaves = 0, inner = 0;
  bool sah_ok = true, coords_ok = true;
};

// fn(t, a, b) over [0, nn) cut into `threads` ranges in node order; the
// calling thread takes the last range, and any range whose thread could not
// be started.
template <typename F>
void over_ranges(unsigned threads, uint32_t nn, F&& fn) {
  std::vector<std::thread> pool;
  pool.reserve(threads);
  for (unsigned t = 0; t < threads; ++t) {
    const uint32_t a = (uint32_t)((uint64_t)nn * t / threads), b = (uint32_t)((uint64_t)nn * (t + 1) / threads);
    if (t + 1 < threads) {
      try {
        pool.emplace_back([&fn, t, a, b] { fn(t, a, b); });
        continue;
      } catch (const std::system_error&) {
      }
    }
    fn(t, a, b);
  }
  for (auto& th : pool) th.join();
}

size_t up16(size_t b) { return (b + 15) & ~(size_t)15; }

float as_float(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

}  // namespace

size_t layout_bytes(uint32_t nn) {
  return 2 * 16 * (size_t)nn + up16(4 * (size_t)nn) + 64 * (size_t)(nn / 2) + up16(4 * (size_t)nn);
}

std::string layout_nodes(const fk_bvh_node* nodes, uint32_t nn, uint32_t nc, void* arena, NodeLayout& out,
                         unsigned threads) {
  if (!nodes || nn == 0 || !arena) return "fk_scene_upload: empty or malformed scene";
  unsigned T = threads;
  if (T == 0) T = nn < (1u << 16) ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  T = std::min<unsigned>(T, nn);
  char* at = static_cast<char*>(arena);
  float* const lo = out.lo = reinterpret_cast<float*>(at);
  float* const hi = out.hi = reinterpret_cast<float*>(at + 16 * (size_t)nn);
  uint32_t* const jump = out.jump = reinterpret_cast<uint32_t*>(at + 32 * (size_t)nn);
  float* const wide = out.wide = reinterpret_cast<float*>(at + 32 * (size_t)nn + up16(4 * (size_t)nn));
  int32_t* const wide_of = reinterpret_cast<int32_t*>(at + 32 * (size_t)nn + up16(4 * (size_t)nn) +
                                                      64 * (size_t)(nn / 2));

  std::vector<RangeScan> scan(T);
  over_ranges(T, nn, [&](unsigned t, uint32_t a, uint32_t b) {
    RangeScan& r = scan[t];
    for (uint32_t i = a; i < b; ++i) {
      const fk_bvh_node& n = nodes[i];
      if (n.start > n.end || n.end > nc || n.start % 3 || n.end % 3 || n.jump <= i || n.jump > nn) {
        r.bad = i;
        return;
      }
      const bool leaf = n.jump == i + 1;
      if (leaf != (n.end > n.start)) {
        r.bad = i;
        r.mixed = true;
        return;
      }
      float* L = lo + 4 * (size_t)i;
      float* H = hi + 4 * (size_t)i;
      L[0] = n.aabb_min[0], L[1] = n.aabb_min[1], L[2] = n.aabb_min[2], L[3] = as_float(n.start);
      H[0] = n.aabb_max[0], H[1] = n.aabb_max[1], H[2] = n.aabb_max[2], H[3] = as_float(n.end);
      jump[i] = n.jump;
      for (int k = 0; k < 3; ++k)
        r.coords_ok = r.coords_ok && std::fabs(n.aabb_min[k]) < kFilterLimit &&
                      std::fabs(n.aabb_max[k]) < kFilterLimit && n.aabb_min[k] <= n.aabb_max[k];
      if (leaf) {
        ++r.leaves;
        for (int k = 0; k < 3; ++k) r.sah_ok = r.sah_ok && sah::coord_ok(n.aabb_min[k]) && sah::coord_ok(n.aabb_max[k]);
      } else {
        ++r.inner;
        // children i + 1 and c = nodes[i + 1].jump must split [i + 1, n.jump):
        // c inside it and c's subtree ending where node i's ends (i + 1 < n.jump
        // <= nn, so both reads stay in the array)
        const uint32_t c = nodes[i + 1].jump;
        if (r.split == kNone && (c >= n.jump || nodes[c].jump != n.jump)) r.split = i;
      }
    }
  });
  for (const RangeScan& r : scan)  // ranges in node order: the first defect over all of them
    if (r.bad != kNone)
      return "fk_scene_upload: node " + std::to_string(r.bad) +
             (r.mixed ? " mixes children and triangles" : " is malformed");
  if (nodes[0].jump != nn) return "fk_scene_upload: node 0 does not span the array";
  for (const RangeScan& r : scan)
    if (r.split != kNone) return "fk_scene_upload: node " + std::to_string(r.split) + " children inconsistent";

  std::vector<uint32_t> leaf_base(T), wide_base(T);
  uint32_t leaves = 0, inner = 0;
  out.sah_ok = out.coords_ok = true;
  for (unsigned t = 0; t < T; ++t) {
    leaf_base[t] = leaves;
    wide_base[t] = inner;
    leaves += scan[t].leaves;
    inner += scan[t].inner;
    out.sah_ok = out.sah_ok && scan[t].sah_ok;
    out.coords_ok = out.coords_ok && scan[t].coords_ok;
  }
  // a checked tree is a full binary tree: nn = 2 x inner + 1
  if (inner > nn / 2) return "fk_scene_upload: empty or malformed scene";
  out.leaves = leaves;
  out.wide_count = inner;
  out.leaf_ids.resize(leaves);
  // With the structure checked, node i's subtree is [i, jump[i]) and the
  // subtrees nest, so the inner nodes whose subtree still holds node i (a
  // stack of their ends) are its ancestors.  The scan reads only the skip
  // pointers: with several ranges it runs beside the record passes.
  uint32_t depth = 1;
  auto depth_scan = [&] {
    std::vector<uint32_t> ends;
    for (uint32_t i = 0; i < nn; ++i) {
      while (!ends.empty() && ends.back() <= i) ends.pop_back();
      depth = std::max(depth, (uint32_t)ends.size() + 1);
      if (jump[i] != i + 1) ends.push_back(jump[i]);
    }
  };
  std::thread depth_thread;
  if (T > 1) {
    try {
      depth_thread = std::thread(depth_scan);
    } catch (const std::system_error&) {
    }
  }
  over_ranges(T, nn, [&](unsigned t, uint32_t a, uint32_t b) {
    uint32_t l = leaf_base[t], w = wide_base[t];
    for (uint32_t i = a; i < b; ++i) {
      if (jump[i] == i + 1) {
        wide_of[i] = -1;
        out.leaf_ids[l++] = i;
      } else {
        wide_of[i] = (int32_t)w++;
      }
    }
  });
  over_ranges(T, nn, [&](unsigned, uint32_t a, uint32_t b) {
    for (uint32_t i = a; i < b; ++i) {
      if (wide_of[i] < 0) continue;
      const uint32_t c[2] = {i + 1, jump[i + 1]};
      int32_t ints[4];
      for (int k = 0; k < 2; ++k) {
        const bool inner_child = wide_of[c[k]] >= 0;
        ints[k] = inner_child ? wide_of[c[k]] : -(int32_t)c[k] - 1;
        ints[2 + k] = inner_child ? 0 : (int32_t)((nodes[c[k]].end - nodes[c[k]].start) / 3);
      }
      const fk_bvh_node& A = nodes[c[0]];
      const fk_bvh_node& B = nodes[c[1]];
      float* w = wide + 16 * (size_t)wide_of[i];
      w[0] = A.aabb_min[0], w[1] = A.aabb_max[0], w[2] = A.aabb_min[1], w[3] = A.aabb_max[1];
      w[4] = B.aabb_min[0], w[5] = B.aabb_max[0], w[6] = B.aabb_min[1], w[7] = B.aabb_max[1];
      w[8] = A.aabb_min[2], w[9] = A.aabb_max[2], w[10] = B.aabb_min[2], w[11] = B.aabb_max[2];
      std::memcpy(w + 12, ints, 16);
    }
  });
  if (depth_thread.joinable()) depth_thread.join();
  else depth_scan();
  out.depth = depth;
  return {};
}

}  // namespace fk
