// BVH build and flatten on the host: BVH::createBinary (Src/bvh.cpp:128-314)
// and fillMeshData (Src/meshmapping.cpp:62-125).
//
// The tree is the reference's, node for node: 16 centroid buckets per axis,
// the reference's cost formula, the split at a bucket boundary, an order-
// preserving partition, leaves of <= max_tris triangles or at max_depth, boxes
// kept as (center, half size) and rebuilt from the children after recursion.
// The top levels are built by parallel tasks; every node's inputs (its
// triangle list in original order) are the same as in the sequential build, so
// the result is identical.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <system_error>
#include <thread>

#include "fk_bvh_rules.h"
#include "fk_internal.h"

namespace {

struct Box {
  float lo[3], hi[3];
};
inline Box empty_box() {
  Box b;
  for (int a = 0; a < 3; ++a) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; }
  return b;
}
// min / max below are fk::bvh::fmin / fmax (fk_bvh_rules.h): order does not
// matter, so these folds equal the device build's parallel ones.
// addPoint (Src/bvh.cpp:31-35).
inline void add_point(Box& b, const float* p) {
  for (int a = 0; a < 3; ++a) { b.lo[a] = fk::bvh::fmin(p[a], b.lo[a]); b.hi[a] = fk::bvh::fmax(p[a], b.hi[a]); }
}
// min(acc, triangle bounds) of the partition loop (Src/bvh.cpp:240-247).
inline void grow_acc(Box& b, const float* lo, const float* hi) {
  for (int a = 0; a < 3; ++a) { b.lo[a] = fk::bvh::fmin(b.lo[a], lo[a]); b.hi[a] = fk::bvh::fmax(b.hi[a], hi[a]); }
}
inline Box join(const Box& a, const Box& b) {
  Box r = a;
  for (int k = 0; k < 3; ++k) { r.lo[k] = fk::bvh::fmin(b.lo[k], r.lo[k]); r.hi[k] = fk::bvh::fmax(b.hi[k], r.hi[k]); }
  return r;
}
// Src/bvh.cpp:63-68 (x*y appears twice in the reference's area term).
inline float cost_of(const Box& b, int n) {
  return fk::bvh::cost(b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2], n);
}

// Per-triangle values the build reads repeatedly.
struct Pre {
  float p[3][3];  // corners
  float cdiv[3];  // (p0 + p1 + p2) / 3.0f       (bucketing, Src/bvh.cpp:139)
  float cmul[3];  // (p0 + p1 + p2) * (1.0f/3.0f) (partition, Src/bvh.cpp:227)
};

using Node = fk_bvh_tree_node;

// Threads for one pass of the build over n triangles: one below 2^18, else
// as many as the host has (16 at most) with at least 2^17 triangles each.
unsigned pass_threads(uint32_t n) {
  if (n < (1u << 18)) return 1;
  const unsigned hw = std::thread::hardware_concurrency();
  return std::max(1u, std::min(std::min(hw ? hw : 1u, 16u), n >> 17));
}

// fn(k, x, y) over [b, e) cut into T chunks in order; the calling thread takes
// the last chunk, and any chunk whose thread cannot be started.
template <typename F>
void over_chunks(uint32_t b, uint32_t e, unsigned T, F&& fn) {
  std::vector<std::thread> pool;
  pool.reserve(T);
  for (unsigned k = 0; k < T; ++k) {
    const uint32_t x = b + (uint32_t)((uint64_t)(e - b) * k / T);
    const uint32_t y = b + (uint32_t)((uint64_t)(e - b) * (k + 1) / T);
    if (k + 1 < T) {
      try {
        pool.emplace_back([&fn, k, x, y] { fn(k, x, y); });
        continue;
      } catch (const std::system_error&) {
      }
    }
    fn(k, x, y);
  }
  for (auto& th : pool) th.join();
}

// Bucket counts and triangle bounds of one axis choice (Src/bvh.cpp:139-170).
struct Bins {
  uint32_t cnt[3][16];
  float blo[3][16][3], bhi[3][16][3];
  void clear() {
    for (int a = 0; a < 3; ++a)
      for (int k = 0; k < 16; ++k) {
        cnt[a][k] = 0;
        for (int q = 0; q < 3; ++q) {
          blo[a][k][q] = FLT_MAX;
          bhi[a][k][q] = -FLT_MAX;
        }
      }
  }
  void merge(const Bins& o) {
    for (int a = 0; a < 3; ++a)
      for (int k = 0; k < 16; ++k) {
        cnt[a][k] += o.cnt[a][k];
        for (int q = 0; q < 3; ++q) {
          blo[a][k][q] = fk::bvh::fmin(o.blo[a][k][q], blo[a][k][q]);
          bhi[a][k][q] = fk::bvh::fmax(o.bhi[a][k][q], bhi[a][k][q]);
        }
      }
  }
};

// Large ranges run their passes (centroid bounds, buckets, partition) over
// chunks on several threads: counts add up and the bounds are min / max folds
// whose order does not matter, and the chunks' sides are joined in chunk order,
// so the tree is the sequential build's, bit for bit.
struct Build {
  const Pre* pre;
  std::vector<uint32_t>& order;
  size_t max_tris, max_depth;
  int par_depth;

  // Returns (axis, split value) of Src/bvh.cpp:128-203.
  Box centroid_bounds(uint32_t x, uint32_t y) const {
    Box c = empty_box();
    for (uint32_t i = x; i < y; ++i) add_point(c, pre[order[i]].cdiv);
    return c;
  }
  void fill_bins(uint32_t x, uint32_t y, const Box& cb, const float* ext, Bins& B) const {
    B.clear();
    for (uint32_t i = x; i < y; ++i) {
      const Pre& p = pre[order[i]];
      for (int a = 0; a < 3; ++a) {
        const uint32_t q = fk::bvh::bucket(p.cdiv[a], cb.lo[a], ext[a]);
        B.cnt[a][q]++;
        for (int c = 0; c < 3; ++c)
          for (int r = 0; r < 3; ++r) {
            B.blo[a][q][r] = fk::bvh::fmin(p.p[c][r], B.blo[a][q][r]);
            B.bhi[a][q][r] = fk::bvh::fmax(p.p[c][r], B.bhi[a][q][r]);
          }
      }
    }
  }

  void choose(uint32_t b, uint32_t e, int* axis, float* value) const {
    const unsigned T = pass_threads(e - b);
    Box cb;
    float ext[3];
    if (T == 1) {
      cb = centroid_bounds(b, e);
      for (int a = 0; a < 3; ++a) ext[a] = cb.hi[a] - cb.lo[a];
      Bins B;
      fill_bins(b, e, cb, ext, B);
      fk::bvh::pick_split(B.blo, B.bhi, B.cnt, (int)(e - b), cb.lo, cb.hi, axis, value);
      return;
    }
    std::vector<Box> cbs(T);
    over_chunks(b, e, T, [&](unsigned k, uint32_t x, uint32_t y) { cbs[k] = centroid_bounds(x, y); });
    cb = cbs[0];
    for (unsigned k = 1; k < T; ++k) cb = join(cb, cbs[k]);
    for (int a = 0; a < 3; ++a) ext[a] = cb.hi[a] - cb.lo[a];
    std::vector<Bins> bins(T);
    over_chunks(b, e, T, [&](unsigned k, uint32_t x, uint32_t y) { fill_bins(x, y, cb, ext, bins[k]); });
    for (unsigned k = 1; k < T; ++k) bins[0].merge(bins[k]);
    fk::bvh::pick_split(bins[0].blo, bins[0].bhi, bins[0].cnt, (int)(e - b), cb.lo, cb.hi, axis, value);
  }

  static void set_box(Node& n, const Box& b) {
    for (int a = 0; a < 3; ++a) {
      n.c[a] = (b.lo[a] + b.hi[a]) * 0.5f;
      n.s[a] = (b.hi[a] - b.lo[a]) * 0.5f;
    }
  }

  // Builds the subtree over order[b, e) whose node `ni` already holds its
  // box; nodes are appended to `out`.
  void divide(std::vector<Node>& out, int32_t ni, uint32_t b, uint32_t e, size_t depth) {
    out[ni].first = b;
    out[ni].count = e - b;
    if ((size_t)(e - b) <= max_tris || depth >= max_depth) {
      out[ni].subtree = e - b;
      return;
    }
    int axis;
    float split;
    choose(b, e, &axis, &split);
    // Order-preserving partition (triangles keep their relative order on each
    // side).  A large range splits in chunks, each into its own two sides; the
    // left sides then go back in chunk order, followed by the right sides.
    std::vector<uint32_t> right;
    Box lb = empty_box(), rb = empty_box();
    uint32_t w = b;
    auto side_of = [&](uint32_t t, Box& l, Box& r, bool& left) {
      const Pre& p = pre[t];
      float lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        lo[a] = fk::bvh::fmin(p.p[0][a], fk::bvh::fmin(p.p[1][a], p.p[2][a]));
        hi[a] = fk::bvh::fmax(p.p[0][a], fk::bvh::fmax(p.p[1][a], p.p[2][a]));
      }
      left = p.cmul[axis] <= split;
      grow_acc(left ? l : r, lo, hi);
    };
    const unsigned T = pass_threads(e - b);
    if (T == 1) {
      for (uint32_t i = b; i < e; ++i) {
        const uint32_t t = order[i];
        bool left;
        side_of(t, lb, rb, left);
        if (left) order[w++] = t;
        else right.push_back(t);
      }
    } else {
      struct Sides {
        std::vector<uint32_t> left, right;
        Box lb, rb;
      };
      std::vector<Sides> parts(T);
      over_chunks(b, e, T, [&](unsigned k, uint32_t x, uint32_t y) {
        Sides& s = parts[k];
        s.lb = s.rb = empty_box();
        for (uint32_t i = x; i < y; ++i) {
          const uint32_t t = order[i];
          bool left;
          side_of(t, s.lb, s.rb, left);
          (left ? s.left : s.right).push_back(t);
        }
      });
      for (Sides& s : parts) {
        std::copy(s.left.begin(), s.left.end(), order.begin() + w);
        w += (uint32_t)s.left.size();
        lb = join(lb, s.lb);
        rb = join(rb, s.rb);
      }
      right.reserve(e - w);
      for (Sides& s : parts) right.insert(right.end(), s.right.begin(), s.right.end());
    }
    if (w == b || w == e) {  // Src/bvh.cpp:248-256: cannot split, stays a leaf
      std::copy(right.begin(), right.end(), order.begin() + w);
      out[ni].subtree = e - b;
      return;
    }
    std::copy(right.begin(), right.end(), order.begin() + w);
    std::vector<uint32_t>().swap(right);
    out[ni].count = 0;
    Node L, R;
    set_box(L, lb);
    set_box(R, rb);
    int32_t li, ri;
    if ((int)depth < par_depth && (e - b) > 65536) {
      std::vector<Node> lv(1, L), rv(1, R);
      std::thread th;
      try {
        th = std::thread([&] { divide(lv, 0, b, w, depth + 1); });
      } catch (const std::system_error&) {  // no thread to be had: the left half here, first
        divide(lv, 0, b, w, depth + 1);
      }
      divide(rv, 0, w, e, depth + 1);
      if (th.joinable()) th.join();
      li = (int32_t)out.size();
      append(out, lv);
      ri = (int32_t)out.size();
      append(out, rv);
    } else {
      li = (int32_t)out.size();
      out.push_back(L);
      ri = (int32_t)out.size();
      out.push_back(R);
      divide(out, li, b, w, depth + 1);
      divide(out, ri, w, e, depth + 1);
    }
    out[ni].kid[0] = li;
    out[ni].kid[1] = ri;
    const Node& A = out[li];
    const Node& B = out[ri];
    Box u;
    for (int a = 0; a < 3; ++a) {
      u.lo[a] = fk::bvh::fmin(A.c[a] - A.s[a], B.c[a] - B.s[a]);
      u.hi[a] = fk::bvh::fmax(A.c[a] + A.s[a], B.c[a] + B.s[a]);
      out[ni].c[a] = (u.hi[a] + u.lo[a]) * 0.5f;
      out[ni].s[a] = (u.hi[a] - u.lo[a]) * 0.5f;
    }
    out[ni].subtree = A.subtree + B.subtree;
  }

  static void append(std::vector<Node>& out, const std::vector<Node>& sub) {
    int32_t off = (int32_t)out.size();
    for (Node n : sub) {
      if (n.kid[0] >= 0) { n.kid[0] += off; n.kid[1] += off; }
      out.push_back(n);
    }
  }
};

// Walks the fillMeshData recursion: emits nodes / corners through callbacks.
// A leaf's corners in the flattened arrays: from corner `corner`, the
// corners of triangles order[first .. first + count).
struct LeafRun {
  uint32_t corner, first, count;
};

struct Flatten {
  const fk_bvh& t;
  fk_bvh_node* nodes;
  std::vector<LeafRun>* runs;  // the leaves' corner runs, written after the walk (or null: counts only)
  uint32_t n_nodes = 0, n_corners = 0;

  void visit(int32_t ni) {
    const Node& n = t.nodes[ni];
    bool kids = n.kid[0] >= 0;
    if (!kids && n.count == 0) return;
    if (kids) {
      const Node& a = t.nodes[n.kid[0]];
      const Node& b = t.nodes[n.kid[1]];
      if (a.subtree > 0 && b.subtree == 0) { visit(n.kid[0]); return; }
      if (b.subtree > 0 && a.subtree == 0) { visit(n.kid[1]); return; }
    }
    uint32_t me = n_nodes++;
    uint32_t start = n_corners;
    if (!kids) {
      if (runs) runs->push_back({n_corners, n.first, n.count});
      n_corners += 3 * n.count;
    }
    if (nodes) {
      fk_bvh_node& d = nodes[me];
      for (int a = 0; a < 3; ++a) {
        d.aabb_min[a] = n.c[a] - n.s[a];
        d.aabb_max[a] = n.c[a] + n.s[a];
      }
      d.start = start;
      d.end = n_corners;
    }
    if (kids) {
      visit(n.kid[0]);
      visit(n.kid[1]);
    }
    if (nodes) nodes[me].jump = n_nodes;
  }
};

}  // namespace

extern "C" {

int fk_bvh_build(const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, fk_bvh** out) {
  if (!mesh || !out || max_tris == 0) return FK_ERR_INVALID;
  const uint32_t nf = mesh->triangle_count();
  std::unique_ptr<Pre[]> pre(new (std::nothrow) Pre[nf ? nf : 1]);
  if (!pre) return FK_ERR_NOMEM;
  over_chunks(0, nf, pass_threads(nf), [&](unsigned, uint32_t x, uint32_t y) {
    for (uint32_t f = x; f < y; ++f) {
      const float* p[3];
      for (int k = 0; k < 3; ++k)
        p[k] = &mesh->positions[3 * (size_t)mesh->vertices[3 * (size_t)mesh->triangles[3 * (size_t)f + k]]];
      Pre& q = pre[f];
      for (int a = 0; a < 3; ++a) {
        float s = p[0][a] + p[1][a] + p[2][a];
        q.cdiv[a] = s / 3.0f;
        q.cmul[a] = s * (1.0f / 3.0f);
        for (int k = 0; k < 3; ++k) q.p[k][a] = p[k][a];
      }
    }
  });
  fk_bvh* t = new (std::nothrow) fk_bvh();
  if (!t) return FK_ERR_NOMEM;
  t->triangle_count = nf;
  t->order.resize(nf);
  for (uint32_t i = 0; i < nf; ++i) t->order[i] = i;
  // Root box over all positions (Src/bvh.cpp:287-297), including unreferenced ones.
  Box rb = empty_box();
  for (uint32_t i = 0; i < mesh->position_count(); ++i) {
    const float* p = &mesh->positions[3 * (size_t)i];
    grow_acc(rb, p, p);
  }
  Node root;
  Build::set_box(root, rb);
  t->nodes.reserve(nf / 2 + 16);
  t->nodes.push_back(root);
  unsigned hw = std::thread::hardware_concurrency();
  int par = 0;
  while ((1u << par) < (hw ? hw : 1) && par < 6) ++par;
  Build b{pre.get(), t->order, max_tris, max_depth, par};
  b.divide(t->nodes, 0, 0, nf, 0);
  *out = t;
  return FK_OK;
}

int fk_bvh_free(fk_bvh* bvh) {
  delete bvh;
  return FK_OK;
}

int fk_bvh_flatten_sizes(const fk_bvh* bvh, uint32_t* node_count, uint32_t* corner_count) {
  if (!bvh || !node_count || !corner_count) return FK_ERR_INVALID;
  Flatten f{*bvh, nullptr, nullptr};
  f.visit(0);
  *node_count = f.n_nodes;
  *corner_count = f.n_corners;
  return FK_OK;
}

int fk_bvh_flatten(const fk_bvh* bvh, const fk_mesh* mesh, fk_bvh_node* nodes, float* pos4, float* nrm4) {
  if (!bvh || !mesh || !nodes || !pos4 || !nrm4) return FK_ERR_INVALID;
  if (mesh->triangle_count() != bvh->triangle_count) return FK_ERR_INVALID;
  uint32_t nn = (uint32_t)(mesh->normals.size() / 3);
  for (uint32_t v = 0; v < mesh->vertex_count(); ++v)
    if (mesh->vertices[3 * (size_t)v + 2] >= nn) return FK_ERR_INVALID;
  // the walk numbers the nodes and the leaves' corner runs in depth-first
  // order; the corners (the bulk of the bytes) are then written run by run
  // over chunks on several threads
  std::vector<LeafRun> runs;
  Flatten f{*bvh, nodes, &runs};
  f.visit(0);
  over_chunks(0, (uint32_t)runs.size(), pass_threads(bvh->triangle_count), [&](unsigned, uint32_t x, uint32_t y) {
    for (uint32_t r = x; r < y; ++r) {
      const LeafRun& run = runs[r];
      uint32_t c = run.corner;
      for (uint32_t i = 0; i < run.count; ++i) {
        const uint32_t tri = bvh->order[run.first + i];
        for (int k = 0; k < 3; ++k, ++c) {
          const uint32_t* v = &mesh->vertices[3 * (size_t)mesh->triangles[3 * (size_t)tri + k]];
          const float* p = &mesh->positions[3 * (size_t)v[0]];
          const float* q = &mesh->normals[3 * (size_t)v[2]];
          float* dp = pos4 + 4 * (size_t)c;
          float* dn = nrm4 + 4 * (size_t)c;
          dp[0] = p[0], dp[1] = p[1], dp[2] = p[2], dp[3] = 0.0f;
          dn[0] = q[0], dn[1] = q[1], dn[2] = q[2], dn[3] = 0.0f;
        }
      }
    }
  });
  return FK_OK;
}

}  // extern "C"
