// Checks fk::layout_nodes (fornos_b200/csrc/fk_layout.cpp) against a
// sequential restatement of the scene upload's checks and layout, on a node
// file and on seeded mutations of it, for several thread counts.
//
//   check <nodes.bin> <corner count> <mutations> <seed>
//
// nodes.bin: fk_bvh_node records.  Prints "cases N mismatches M" last and
// exits non-zero on a mismatch.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../fornos_b200/csrc/fk_layout.h"
#include "../../fornos_b200/csrc/fk_sah_rules.h"

namespace {

struct Plain {
  std::string err;
  std::vector<float> lo, hi, wide;
  std::vector<uint32_t> jump, leaf_ids;
  uint32_t leaves = 0, nw = 0, depth = 1;
  bool sah_ok = true, coords_ok = true;
};

float as_float(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// One pass after another, in node order, each stopping at its first defect.
Plain plain(const std::vector<fk_bvh_node>& nodes, uint32_t nc) {
  Plain p;
  const uint32_t nn = (uint32_t)nodes.size();
  if (nn == 0) {
    p.err = "fk_scene_upload: empty or malformed scene";
    return p;
  }
  p.lo.assign(4 * (size_t)nn, 0.0f);
  p.hi.assign(4 * (size_t)nn, 0.0f);
  p.jump.assign(nn, 0);
  for (uint32_t i = 0; i < nn; ++i) {
    const fk_bvh_node& n = nodes[i];
    if (n.start > n.end || n.end > nc || n.start % 3 || n.end % 3 || n.jump <= i || n.jump > nn) {
      p.err = "fk_scene_upload: node " + std::to_string(i) + " is malformed";
      return p;
    }
    const bool leaf = n.jump == i + 1;
    if (leaf != (n.end > n.start)) {
      p.err = "fk_scene_upload: node " + std::to_string(i) + " mixes children and triangles";
      return p;
    }
    p.leaves += leaf;
    if (leaf) {
      p.leaf_ids.push_back(i);
      for (int a = 0; a < 3; ++a)
        p.sah_ok = p.sah_ok && fk::sah::coord_ok(n.aabb_min[a]) && fk::sah::coord_ok(n.aabb_max[a]);
    }
    for (int a = 0; a < 3; ++a) {
      p.lo[4 * i + a] = n.aabb_min[a];
      p.hi[4 * i + a] = n.aabb_max[a];
    }
    p.lo[4 * i + 3] = as_float(n.start);
    p.hi[4 * i + 3] = as_float(n.end);
    p.jump[i] = n.jump;
  }
  if (nodes[0].jump != nn) {
    p.err = "fk_scene_upload: node 0 does not span the array";
    return p;
  }
  std::vector<int32_t> wide_of(nn, -1);
  for (uint32_t i = 0; i < nn; ++i)
    if (nodes[i].jump != i + 1) {
      const uint32_t r = nodes[i + 1].jump;
      if (i + 1 >= nn || r >= nodes[i].jump || nodes[r].jump != nodes[i].jump) {
        p.err = "fk_scene_upload: node " + std::to_string(i) + " children inconsistent";
        return p;
      }
      wide_of[i] = (int32_t)p.nw++;
    }
  p.wide.assign(16 * (size_t)p.nw, 0.0f);
  std::vector<uint32_t> depth(nn, 1);
  for (uint32_t i = 0; i < nn; ++i) {
    p.depth = depth[i] > p.depth ? depth[i] : p.depth;
    if (wide_of[i] < 0) continue;
    const uint32_t c[2] = {i + 1, nodes[i + 1].jump};
    depth[c[0]] = depth[c[1]] = depth[i] + 1;
    int32_t ints[4];
    for (int k = 0; k < 2; ++k) {
      ints[k] = wide_of[c[k]] >= 0 ? wide_of[c[k]] : -(int32_t)c[k] - 1;
      ints[2 + k] = wide_of[c[k]] >= 0 ? 0 : (int32_t)((nodes[c[k]].end - nodes[c[k]].start) / 3);
    }
    const fk_bvh_node& L = nodes[c[0]];
    const fk_bvh_node& R = nodes[c[1]];
    float* w = &p.wide[16 * (size_t)wide_of[i]];
    const float v[12] = {L.aabb_min[0], L.aabb_max[0], L.aabb_min[1], L.aabb_max[1],
                         R.aabb_min[0], R.aabb_max[0], R.aabb_min[1], R.aabb_max[1],
                         L.aabb_min[2], L.aabb_max[2], R.aabb_min[2], R.aabb_max[2]};
    std::memcpy(w, v, 48);
    std::memcpy(w + 12, ints, 16);
  }
  for (uint32_t i = 0; i < nn; ++i)
    for (int a = 0; a < 3; ++a)
      p.coords_ok = p.coords_ok && std::fabs(nodes[i].aabb_min[a]) < 16777216.0f &&
                    std::fabs(nodes[i].aabb_max[a]) < 16777216.0f && nodes[i].aabb_min[a] <= nodes[i].aabb_max[a];
  return p;
}

bool same(const Plain& p, const std::string& err, const fk::NodeLayout& l, uint32_t nn) {
  if (p.err != err) return false;
  if (!err.empty()) return true;
  auto eq = [](const void* a, const void* b, size_t bytes) { return bytes == 0 || std::memcmp(a, b, bytes) == 0; };
  return p.leaves == l.leaves && p.nw == l.wide_count && p.depth == l.depth && p.sah_ok == l.sah_ok &&
         p.coords_ok == l.coords_ok && p.leaf_ids == l.leaf_ids && eq(p.lo.data(), l.lo, 16 * (size_t)nn) &&
         eq(p.hi.data(), l.hi, 16 * (size_t)nn) && eq(p.jump.data(), l.jump, 4 * (size_t)nn) &&
         eq(p.wide.data(), l.wide, 64 * (size_t)p.nw);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::vector<fk_bvh_node> base;
  fk_bvh_node n;
  while (std::fread(&n, sizeof n, 1, f) == 1) base.push_back(n);
  std::fclose(f);
  const uint32_t nc = (uint32_t)std::stoul(argv[2]);
  const int mutations = std::stoi(argv[3]);
  std::mt19937 rng((uint32_t)std::stoul(argv[4]));
  long cases = 0, mismatches = 0, errors = 0;
  auto run = [&](const std::vector<fk_bvh_node>& nodes) {
    const Plain p = plain(nodes, nc);
    errors += !p.err.empty();
    for (unsigned threads : {1u, 2u, 3u, 7u, 16u, 0u}) {
      fk::NodeLayout l;
      struct alignas(16) Word { unsigned char b[16]; };
      std::vector<Word> arena(fk::layout_bytes((uint32_t)nodes.size()) / 16);
      const std::string err = fk::layout_nodes(nodes.data(), (uint32_t)nodes.size(), nc, arena.data(), l, threads);
      ++cases;
      if (!same(p, err, l, (uint32_t)nodes.size())) {
        if (++mismatches <= 5)
          std::printf("mismatch: %zu nodes, threads %u: '%s' against '%s'\n", nodes.size(), threads, err.c_str(),
                      p.err.c_str());
      }
    }
  };
  run(base);
  const uint32_t nn = (uint32_t)base.size();
  const float odd[] = {NAN, INFINITY, -INFINITY, 16777216.0f, -16777216.0f, 1e30f, -0.0f, 3.0f};
  for (int m = 0; m < mutations; ++m) {
    std::vector<fk_bvh_node> nodes = base;
    const int edits = 1 + (int)(rng() % 3);
    for (int e = 0; e < edits; ++e) {
      fk_bvh_node& x = nodes[rng() % nn];
      switch (rng() % 9) {
        case 0: x.jump = (uint32_t)(rng() % (nn + 2)); break;                   // anywhere, past the end included
        case 1: x.jump = x.jump + (rng() % 2 ? 1u : 0xFFFFFFFFu); break;        // off by one
        case 2: x.start = (uint32_t)(rng() % (nc + 4)); break;
        case 3: x.end = (uint32_t)(rng() % (nc + 4)); break;
        case 4: x.end = x.start; break;                                        // a leaf without triangles
        case 5: x.end = x.start + 3 * (1 + rng() % 4); break;                  // an inner node with triangles
        case 6: x.aabb_min[rng() % 3] = odd[rng() % 8]; break;
        case 7: x.aabb_max[rng() % 3] = odd[rng() % 8]; break;
        default: std::swap(x.aabb_min[rng() % 3], x.aabb_max[rng() % 3]); break;  // faces out of order
      }
    }
    run(nodes);
  }
  std::printf("cases %ld mismatches %ld rejected %ld\n", cases, mismatches, errors);
  return mismatches ? 1 : 0;
}
