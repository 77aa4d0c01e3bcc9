// CPU oracle for the Fornos texture-baking path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product is
// compared against; it is never linked into, imported by, or called from the
// product library (fornos_b200/).  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load it.
//
// It restates, in plain sequential C++, the reference's algorithm for the path:
//   * host preprocessing   Src/mesh.cpp:627-768   (face / vertex / welded normals,
//                                                  tangent space)
//   * UV rasterisation     Src/compute.cpp:75-193, 195-349 (raster, hybrid raster)
//   * map compaction       Src/compute.cpp:372-416
//   * BVH build            Src/bvh.cpp:128-314    (16-bucket SAH-style binary split)
//   * BVH flatten          Src/meshmapping.cpp:62-125 (skip-pointer DFS layout)
//   * sample table         Src/math.h:314-382     (Hammersley + cosine hemisphere)
//   * the 13 compute shaders, Shaders/*.comp, as per-texel / per-sample functions.
//
// Arithmetic contract (shared with the CUDA kernels and with the reference sources
// compiled under oracle/_ref): IEEE-754 binary32 operations evaluated in source
// order, no FMA contraction (-ffp-contract=off), correctly rounded division and
// square root, min/max = fminf/fmaxf (a NaN operand loses), normalize(v) =
// v * (1 / sqrt(dot(v, v))) as in Src/math.h:110-113, dot = (x*x' + y*y') + z*z'.
// The mesh-mapping barycentric is evaluated in binary64 exactly as
// Shaders/meshmapping_nobackfaces.comp:48-62 declares it.
//
// Parity is pinned by tests/test_oracle_vs_reference.py against the reference's own
// sources (Src/bvh.cpp, Src/compute.cpp, Src/meshmapping.cpp, Src/mesh.cpp,
// Src/math.h and Shaders/*.comp) compiled by oracle/build_ref.py into oracle/_ref,
// and by the committed fixtures in tests/golden/ generated from that build.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- vector math
struct F2 { float x, y; };
struct F3 { float x, y, z; };
struct D3 { double x, y, z; };

static inline F3 mk(float x, float y, float z) { F3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline F3 operator+(F3 a, F3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline F3 operator-(F3 a, F3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline F3 operator-(F3 a) { return mk(-a.x, -a.y, -a.z); }
static inline F3 operator*(F3 a, float k) { return mk(a.x * k, a.y * k, a.z * k); }
static inline F3 operator*(float k, F3 a) { return mk(k * a.x, k * a.y, k * a.z); }
static inline F3 operator/(F3 a, F3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline F3 operator/(F3 a, float k) { return mk(a.x / k, a.y / k, a.z / k); }
static inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline F3 cross(F3 a, F3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline F3 normalize(F3 v) { float inv = 1.0f / std::sqrt(dot(v, v)); return v * inv; }
static inline F3 vmin(F3 a, F3 b) { return mk(std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)); }
static inline F3 vmax(F3 a, F3 b) { return mk(std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)); }
static inline F3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }
static inline void st3(float* p, F3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

static inline D3 dsub(D3 a, D3 b) { D3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline D3 widen(F3 a) { D3 r = {(double)a.x, (double)a.y, (double)a.z}; return r; }

static const uint32_t kMiss = 0xFFFFFFFFu;

// ---------------------------------------------------------------- mesh view
// Same indexed representation as Src/mesh.h:35-63: per-vertex (position,
// texcoord, normal) indices and per-triangle vertex indices.
struct MeshView {
  uint32_t np, nt, nn, nv, nf;
  const float* pos;      // np x 3
  const float* uv;       // nt x 2
  const float* nrm;      // nn x 3
  const uint32_t* vtx;   // nv x 3 : position, texcoord, normal index
  const uint32_t* tri;   // nf x 3 : vertex indices
  const float* tan;      // nv x 3 or null
  const float* bit;      // nv x 3 or null
};

static inline F3 tri_pos(const MeshView& m, uint32_t f, int k) {
  return ld3(m.pos + 3 * (size_t)m.vtx[3 * (size_t)m.tri[3 * (size_t)f + k] + 0]);
}

// ---------------------------------------------------------------- BVH build
// Src/bvh.cpp:128-314.  Nodes hold (center, half size) like the reference's AABB
// (Src/math.h:147-154) because the flattened bounds are center -/+ size
// (Src/meshmapping.cpp:86-87) and that rounding is part of the output.
struct BNode {
  F3 c, s;
  int kid[2];
  std::vector<uint32_t> tris;
  size_t subtree;
};

struct Box { F3 lo, hi; };
static inline Box box_empty() { Box b; b.lo = mk(FLT_MAX, FLT_MAX, FLT_MAX); b.hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX); return b; }
static inline void box_add(Box& b, F3 p) { b.lo = vmin(p, b.lo); b.hi = vmax(p, b.hi); }
static inline Box box_join(const Box& a, const Box& b) { Box r = a; r.lo = vmin(b.lo, r.lo); r.hi = vmax(b.hi, r.hi); return r; }
static inline float box_cost(const Box& b, int n) {
  F3 e = b.hi - b.lo;
  // Src/bvh.cpp:66: the third product repeats x*y (the reference's formula)
  float area = 2.0f * (e.x * e.y + e.x * e.z + e.x * e.y);
  return float(n) * area;
}

struct SplitChoice { int axis; float value; };

static inline float comp(F3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Bucket sweep of Src/bvh.cpp:70-126.  The sweep's last step (all triangles on
// the left) reads one element past the right-side table in the reference; that
// step can never win there (its right side is empty), and it is skipped here.
static void sweep(const uint32_t cnt[16], const Box bb[16], uint32_t ntris, int* best_idx, float* best_cost) {
  Box right[15];
  right[14] = bb[15];
  for (int i = 13; i >= 0; --i) right[i] = box_join(right[i + 1], bb[i + 1]);
  float best = FLT_MAX;
  int bi = 0;
  Box left = box_empty();
  int nl = 0, nr = (int)ntris;
  for (int i = 0; i < 15; ++i) {
    nl += (int)cnt[i];
    nr -= (int)cnt[i];
    left = box_join(left, bb[i]);
    float cost = box_cost(left, nl) + box_cost(right[i], nr);
    if (cost < best) { best = cost; bi = i; }
  }
  *best_idx = bi;
  *best_cost = best;
}

static SplitChoice choose_split(const MeshView& m, const BNode& n) {
  Box cb = box_empty();
  for (uint32_t f : n.tris) {
    F3 cen = (tri_pos(m, f, 0) + tri_pos(m, f, 1) + tri_pos(m, f, 2)) / 3.0f;
    box_add(cb, cen);
  }
  uint32_t cnt[3][16];
  Box bb[3][16];
  std::memset(cnt, 0, sizeof(cnt));
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < 16; ++i) bb[a][i] = box_empty();
  for (uint32_t f : n.tris) {
    F3 p0 = tri_pos(m, f, 0), p1 = tri_pos(m, f, 1), p2 = tri_pos(m, f, 2);
    F3 cen = (p0 + p1 + p2) / 3.0f;
    F3 rel = ((cen - cb.lo) / (cb.hi - cb.lo)) * 15.99f;
    for (int a = 0; a < 3; ++a) {
      float r = comp(rel, a);
      size_t k = std::isnan(r) ? 0 : (size_t)r;
      cnt[a][k] += 1;
      box_add(bb[a][k], p0);
      box_add(bb[a][k], p1);
      box_add(bb[a][k], p2);
    }
  }
  int idx[3];
  float cost[3];
  for (int a = 0; a < 3; ++a) sweep(cnt[a], bb[a], (uint32_t)n.tris.size(), &idx[a], &cost[a]);
  SplitChoice sc;
  int a;
  if (cost[0] <= cost[1] && cost[0] <= cost[2]) a = 0;
  else if (cost[1] <= cost[0] && cost[1] <= cost[2]) a = 1;
  else a = 2;
  float lo = comp(cb.lo, a), hi = comp(cb.hi, a);
  sc.axis = a;
  sc.value = lo + (hi - lo) / 16.0f * float(idx[a] + 1);
  return sc;
}

struct Builder {
  const MeshView& m;
  size_t max_tris, max_depth;
  std::vector<BNode> nodes;
  Builder(const MeshView& mv, size_t mt, size_t md) : m(mv), max_tris(mt), max_depth(md) {}

  void divide(int ni, size_t depth) {
    if (nodes[ni].tris.size() <= max_tris || depth >= max_depth) {
      nodes[ni].subtree = nodes[ni].tris.size();
      return;
    }
    SplitChoice sc = choose_split(m, nodes[ni]);
    std::vector<uint32_t> lt, rt;
    Box lb = box_empty(), rb = box_empty();
    const float third = 1.0f / 3.0f;
    for (uint32_t f : nodes[ni].tris) {
      F3 p0 = tri_pos(m, f, 0), p1 = tri_pos(m, f, 1), p2 = tri_pos(m, f, 2);
      F3 cen = (p0 + p1 + p2) * third;
      F3 tlo = vmin(p0, vmin(p1, p2)), thi = vmax(p0, vmax(p1, p2));
      if (comp(cen, sc.axis) <= sc.value) {
        lt.push_back(f);
        lb.lo = vmin(lb.lo, tlo); lb.hi = vmax(lb.hi, thi);
      } else {
        rt.push_back(f);
        rb.lo = vmin(rb.lo, tlo); rb.hi = vmax(rb.hi, thi);
      }
    }
    if (lt.empty() || rt.empty()) {  // Src/bvh.cpp:248-256: give up, keep a leaf
      nodes[ni].subtree = nodes[ni].tris.size();
      return;
    }
    std::vector<uint32_t>().swap(nodes[ni].tris);
    int kids[2];
    for (int k = 0; k < 2; ++k) {
      BNode c;
      const Box& b = k == 0 ? lb : rb;
      c.c = (b.lo + b.hi) * 0.5f;
      c.s = (b.hi - b.lo) * 0.5f;
      c.kid[0] = c.kid[1] = -1;
      c.tris.swap(k == 0 ? lt : rt);
      c.subtree = 0;
      kids[k] = (int)nodes.size();
      nodes.push_back(std::move(c));
    }
    nodes[ni].kid[0] = kids[0];
    nodes[ni].kid[1] = kids[1];
    divide(kids[0], depth + 1);
    divide(kids[1], depth + 1);
    const BNode& L = nodes[kids[0]];
    const BNode& R = nodes[kids[1]];
    F3 lo = vmin(L.c - L.s, R.c - R.s);
    F3 hi = vmax(L.c + L.s, R.c + R.s);
    nodes[ni].c = (hi + lo) * 0.5f;
    nodes[ni].s = (hi - lo) * 0.5f;
    nodes[ni].subtree = L.subtree + R.subtree;
  }

  void build() {
    F3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (uint32_t i = 0; i < m.np; ++i) {
      F3 p = ld3(m.pos + 3 * (size_t)i);
      lo = vmin(lo, p);
      hi = vmax(hi, p);
    }
    BNode root;
    root.c = (hi + lo) * 0.5f;
    root.s = (hi - lo) * 0.5f;
    root.kid[0] = root.kid[1] = -1;
    root.subtree = 0;
    root.tris.resize(m.nf);
    for (uint32_t i = 0; i < m.nf; ++i) root.tris[i] = i;
    nodes.reserve(2 * (size_t)m.nf / (max_tris ? max_tris : 1) + 16);
    nodes.push_back(std::move(root));
    divide(0, 0);
  }
};

// Flattened skip-pointer node, 36 bytes: Src/meshmapping.h:33-40.
struct FlatNode { float lo[3]; float hi[3]; uint32_t start, end, jump; };

struct Scene {
  std::vector<FlatNode> nodes;
  std::vector<float> pos4;  // 4 floats per triangle corner, w = 0
  std::vector<float> nrm4;
};

// Src/meshmapping.cpp:62-125: pre-order DFS; triangles appended in leaf order.
static void flatten(const MeshView& m, const std::vector<BNode>& bn, int ni, Scene& s) {
  const BNode& n = bn[ni];
  bool has_kids = n.kid[0] >= 0;
  if (!has_kids && n.tris.empty()) return;
  if (has_kids) {
    const BNode& a = bn[n.kid[0]];
    const BNode& b = bn[n.kid[1]];
    if (a.subtree > 0 && b.subtree == 0) { flatten(m, bn, n.kid[0], s); return; }
    if (b.subtree > 0 && a.subtree == 0) { flatten(m, bn, n.kid[1], s); return; }
  }
  FlatNode fn;
  F3 lo = n.c - n.s, hi = n.c + n.s;
  fn.lo[0] = lo.x; fn.lo[1] = lo.y; fn.lo[2] = lo.z;
  fn.hi[0] = hi.x; fn.hi[1] = hi.y; fn.hi[2] = hi.z;
  fn.start = (uint32_t)(s.pos4.size() / 4);
  for (uint32_t f : n.tris) {
    for (int k = 0; k < 3; ++k) {
      const uint32_t* v = m.vtx + 3 * (size_t)m.tri[3 * (size_t)f + k];
      const float* p = m.pos + 3 * (size_t)v[0];
      const float* q = m.nrm + 3 * (size_t)v[2];
      s.pos4.insert(s.pos4.end(), {p[0], p[1], p[2], 0.0f});
      s.nrm4.insert(s.nrm4.end(), {q[0], q[1], q[2], 0.0f});
    }
  }
  fn.end = (uint32_t)(s.pos4.size() / 4);
  fn.jump = 0;
  size_t me = s.nodes.size();
  s.nodes.push_back(fn);
  if (has_kids) {
    flatten(m, bn, n.kid[0], s);
    flatten(m, bn, n.kid[1], s);
  }
  s.nodes[me].jump = (uint32_t)s.nodes.size();
}

// ---------------------------------------------------------------- mesh normals
// Src/mesh.cpp:627-648
static void face_normals(const MeshView& m, uint32_t* vtx_out, float* nrm_out) {
  std::memcpy(vtx_out, m.vtx, sizeof(uint32_t) * 3 * (size_t)m.nv);
  for (uint32_t f = 0; f < m.nf; ++f) {
    F3 p0 = tri_pos(m, f, 0), p1 = tri_pos(m, f, 1), p2 = tri_pos(m, f, 2);
    st3(nrm_out + 3 * (size_t)f, normalize(cross(p1 - p0, p2 - p0)));
    for (int k = 0; k < 3; ++k) vtx_out[3 * (size_t)m.tri[3 * (size_t)f + k] + 2] = f;
  }
}

// Src/mesh.cpp:650-678: unweighted face normals summed per position index.
static void vertex_normals(const MeshView& m, uint32_t* vtx_out, float* nrm_out) {
  std::vector<F3> acc(m.np, mk(0, 0, 0));
  for (uint32_t f = 0; f < m.nf; ++f) {
    F3 p0 = tri_pos(m, f, 0), p1 = tri_pos(m, f, 1), p2 = tri_pos(m, f, 2);
    F3 n = normalize(cross(p1 - p0, p2 - p0));
    for (int k = 0; k < 3; ++k) {
      uint32_t pi = m.vtx[3 * (size_t)m.tri[3 * (size_t)f + k] + 0];
      acc[pi] = acc[pi] + n;
    }
  }
  for (uint32_t i = 0; i < m.np; ++i) st3(nrm_out + 3 * (size_t)i, normalize(acc[i]));
  for (uint32_t v = 0; v < m.nv; ++v) {
    vtx_out[3 * (size_t)v + 0] = m.vtx[3 * (size_t)v + 0];
    vtx_out[3 * (size_t)v + 1] = m.vtx[3 * (size_t)v + 1];
    vtx_out[3 * (size_t)v + 2] = m.vtx[3 * (size_t)v + 0];
  }
}

struct KeyLess {
  bool operator()(const F3& a, const F3& b) const {
    if (a.x < b.x) return true;
    if (b.x < a.x) return false;
    if (a.y < b.y) return true;
    if (b.y < a.y) return false;
    return a.z < b.z;
  }
};

// Src/mesh.cpp:680-722: normals welded by exact position value, numbered in
// first-seen order.  Returns the number of normals written.
static uint32_t welded_normals(const MeshView& m, uint32_t* vtx_out, float* nrm_out) {
  std::memcpy(vtx_out, m.vtx, sizeof(uint32_t) * 3 * (size_t)m.nv);
  std::map<F3, uint32_t, KeyLess> slot;
  std::vector<F3> acc;
  for (uint32_t f = 0; f < m.nf; ++f) {
    F3 p[3] = {tri_pos(m, f, 0), tri_pos(m, f, 1), tri_pos(m, f, 2)};
    F3 n = normalize(cross(p[1] - p[0], p[2] - p[0]));
    for (int k = 0; k < 3; ++k) {
      auto it = slot.find(p[k]);
      uint32_t id;
      if (it != slot.end()) {
        id = it->second;
        acc[id] = acc[id] + n;
      } else {
        id = (uint32_t)acc.size();
        slot[p[k]] = id;
        acc.push_back(n);
      }
      vtx_out[3 * (size_t)m.tri[3 * (size_t)f + k] + 2] = id;
    }
  }
  for (size_t i = 0; i < acc.size(); ++i) st3(nrm_out + 3 * i, normalize(acc[i]));
  return (uint32_t)acc.size();
}

// Src/mesh.cpp:724-768: per-vertex tangent frame from UV derivatives.
static void tangent_space(const MeshView& m, float* tan_out, float* bit_out) {
  std::vector<F3> t(m.nv, mk(0, 0, 0)), b(m.nv, mk(0, 0, 0));
  for (uint32_t f = 0; f < m.nf; ++f) {
    uint32_t vi[3];
    F3 p[3];
    F2 u[3];
    for (int k = 0; k < 3; ++k) {
      vi[k] = m.tri[3 * (size_t)f + k];
      const uint32_t* v = m.vtx + 3 * (size_t)vi[k];
      p[k] = ld3(m.pos + 3 * (size_t)v[0]);
      u[k].x = m.uv[2 * (size_t)v[1]];
      u[k].y = m.uv[2 * (size_t)v[1] + 1];
    }
    F3 e0 = p[1] - p[0], e1 = p[2] - p[0];
    F2 t0 = {u[1].x - u[0].x, u[1].y - u[0].y};
    F2 t1 = {u[2].x - u[0].x, u[2].y - u[0].y};
    float r = 1.0f / (t0.x * t1.y - t1.x * t0.y);
    F3 sdir = (e0 * t1.y - e1 * t0.y) * r;
    F3 tdir = (e1 * t0.x - e0 * t1.x) * r;
    for (int k = 0; k < 3; ++k) {
      t[vi[k]] = t[vi[k]] + sdir;
      b[vi[k]] = b[vi[k]] + tdir;
    }
  }
  for (uint32_t i = 0; i < m.nv; ++i) {
    F3 n = ld3(m.nrm + 3 * (size_t)m.vtx[3 * (size_t)i + 2]);
    F3 tt = normalize(t[i] - n * dot(n, t[i]));
    st3(tan_out + 3 * (size_t)i, tt);
    st3(bit_out + 3 * (size_t)i, cross(n, tt));
  }
}

// ---------------------------------------------------------------- UV raster
// Src/math.h:250-259: 2-D barycentric in reciprocal form.
static inline F3 bary2(F2 p, F2 a, F2 b, F2 c) {
  F2 v0 = {b.x - a.x, b.y - a.y}, v1 = {c.x - a.x, c.y - a.y}, v2 = {p.x - a.x, p.y - a.y};
  float s = 1.0f / (v0.x * v1.y - v1.x * v0.y);
  float i = (v2.x * v1.y - v1.x * v2.y) * s;
  float j = (v0.x * v2.y - v2.x * v0.y) * s;
  return mk(1.0f - i - j, i, j);
}

// The reference converts a rounded float to uint32_t directly
// (Src/compute.cpp:136-139); for a negative value that conversion is undefined
// in C++.  The x86-64 code it compiles to goes through a signed 64-bit
// truncation, so -1.0f becomes 0xFFFFFFFF; that is the behaviour defined here.
static inline uint32_t to_u32(float f) {
  if (!(f > -9.2e18f && f < 9.2e18f)) return 0u;
  return (uint32_t)(uint64_t)(int64_t)f;
}

static inline float edge_dist(F3 e0, F3 e1, F3 p) {
  F3 v = p - e0, e = e1 - e0;
  float t = dot(v, e) / dot(e, e);
  F3 q = e0 + e * t;
  return std::sqrt(dot(q - p, q - p));
}

struct MapOut {
  uint32_t w, h;
  std::vector<F3> pos, dir, nrm, tan, bit;
};

enum RasterMode { kSmooth = 0, kLowPolyNormals = 1, kHybrid = 2 };

// Src/compute.cpp:75-151 (modes Smooth / LowPolyNormals) and :213-289 (Hybrid).
// dirs: per-vertex normal indices + normals of the mesh whose normals give the
// mapping direction (null: the mesh's own normals).
static bool raster_tri(const MeshView& m, const uint32_t* dvtx, const float* dnrm, uint32_t f,
                       int mode, float edge, MapOut& out) {
  const uint32_t* v[3];
  for (int k = 0; k < 3; ++k) v[k] = m.vtx + 3 * (size_t)m.tri[3 * (size_t)f + k];
  for (int k = 0; k < 3; ++k)
    if (v[k][1] == kMiss || v[k][2] == kMiss) return false;
  F3 p[3], n[3], d[3], t[3], b[3];
  F2 u[3];
  for (int k = 0; k < 3; ++k) {
    uint32_t vi = m.tri[3 * (size_t)f + k];
    p[k] = ld3(m.pos + 3 * (size_t)v[k][0]);
    u[k].x = m.uv[2 * (size_t)v[k][1]];
    u[k].y = m.uv[2 * (size_t)v[k][1] + 1];
    n[k] = ld3(m.nrm + 3 * (size_t)v[k][2]);
    d[k] = (dvtx && mode != kLowPolyNormals) ? ld3(dnrm + 3 * (size_t)dvtx[3 * (size_t)vi + 2]) : n[k];
    uint32_t ti = mode == kHybrid ? v[k][2] : vi;
    t[k] = m.tan ? ld3(m.tan + 3 * (size_t)ti) : mk(0, 0, 0);
    b[k] = m.tan ? ld3(m.bit + 3 * (size_t)ti) : mk(0, 0, 0);
  }
  const uint32_t W = out.w, H = out.h;
  F2 scale = {(float)W, (float)H};
  F2 pix = {1.0f / scale.x, 1.0f / scale.y};
  F2 half = {pix.x * 0.5f, pix.y * 0.5f};
  float sx[3], sy[3];
  for (int k = 0; k < 3; ++k) { sx[k] = (u[k].x - half.x) * scale.x; sy[k] = (u[k].y - half.y) * scale.y; }
  float fx0 = std::roundf(std::fmin(sx[0], std::fmin(sx[1], sx[2])));
  float fy0 = std::roundf(std::fmin(sy[0], std::fmin(sy[1], sy[2])));
  float fx1 = std::roundf(std::fmax(sx[0], std::fmax(sx[1], sx[2])));
  float fy1 = std::roundf(std::fmax(sy[0], std::fmax(sy[1], sy[2])));
  uint32_t x0, y0, x1, y1;
  if (mode == kHybrid) {
    x0 = to_u32(std::fmax(fx0, 0.0f)); y0 = to_u32(std::fmax(fy0, 0.0f));
    x1 = to_u32(std::fmax(fx1, 0.0f)); y1 = to_u32(std::fmax(fy1, 0.0f));
  } else {
    x0 = std::min(to_u32(fx0), W); y0 = std::min(to_u32(fy0), H);
    x1 = std::min(to_u32(fx1), W); y1 = std::min(to_u32(fy1), H);
  }
  const uint64_t total = (uint64_t)W * H;
  for (uint64_t y = y0; y <= y1; ++y) {
    for (uint64_t x = x0; x <= x1; ++x) {
      F2 q = {(float)x * pix.x + half.x, (float)y * pix.y + half.y};
      F3 w = bary2(q, u[0], u[1], u[2]);
      if (!(w.x >= -0.001f && w.x <= 1 && w.y >= -0.001f && w.y <= 1 && w.z >= -0.001f && w.z <= 1)) continue;
      // int i = y * width + x in 32-bit arithmetic; indices past the map are
      // out-of-bounds writes in the reference and are dropped here.
      uint32_t i = (uint32_t)y * W + (uint32_t)x;
      if ((uint64_t)i >= total) continue;
      F3 P = p[0] * w.x + p[1] * w.y + p[2] * w.z;
      F3 N = normalize(n[0] * w.x + n[1] * w.y + n[2] * w.z);
      F3 D;
      if (mode == kHybrid) {
        float dd = std::fmin(std::fmin(edge_dist(p[0], p[1], P), std::fmin(edge_dist(p[0], p[2], P), edge_dist(p[1], p[2], P))) / edge, 1.0f);
        F3 ds = normalize(d[0] * w.x + d[1] * w.y + d[2] * w.z);
        D = normalize(ds * (1.0f - dd) + N * dd);
      } else {
        D = normalize(d[0] * w.x + d[1] * w.y + d[2] * w.z);
      }
      out.pos[i] = P;
      out.dir[i] = D;
      out.nrm[i] = N;
      out.tan[i] = normalize(t[0] * w.x + t[1] * w.y + t[2] * w.z);
      out.bit[i] = normalize(b[0] * w.x + b[1] * w.y + b[2] * w.z);
    }
  }
  return true;
}

// ---------------------------------------------------------------- shaders
static inline float ray_box(F3 o, F3 d, const FlatNode& n) {
  F3 t1 = (ld3(n.lo) - o) / d;
  F3 t2 = (ld3(n.hi) - o) / d;
  F3 tn = vmin(t1, t2), tx = vmax(t1, t2);
  float a = std::fmax(tn.x, std::fmax(tn.y, tn.z));
  float b = std::fmin(tx.x, std::fmin(tx.y, tx.z));
  return (b >= 0 && a <= b) ? a : FLT_MAX;
}

struct Hit { float t; F3 w; };

// Shaders/meshmapping_nobackfaces.comp:48-62 (binary64)
static inline F3 bary_d(F3 p, F3 a, F3 b, F3 c) {
  D3 A = widen(a);
  D3 v0 = dsub(widen(b), A), v1 = dsub(widen(c), A), v2 = dsub(widen(p), A);
  double d00 = ddot(v0, v0), d01 = ddot(v0, v1), d11 = ddot(v1, v1);
  double d20 = ddot(v2, v0), d21 = ddot(v2, v1);
  double den = d00 * d11 - d01 * d01;
  double y = (d11 * d20 - d01 * d21) / den;
  double z = (d00 * d21 - d01 * d20) / den;
  return mk((float)(1.0 - y - z), (float)y, (float)z);
}

// Shaders/ao_step1.comp:54-68 (binary32)
static inline F3 bary_f(F3 p, F3 a, F3 b, F3 c) {
  F3 v0 = b - a, v1 = c - a, v2 = p - a;
  float d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1);
  float d20 = dot(v2, v0), d21 = dot(v2, v1);
  float den = d00 * d11 - d01 * d01;
  float y = (d11 * d20 - d01 * d21) / den;
  float z = (d00 * d21 - d01 * d20) / den;
  return mk(1.0f - y - z, y, z);
}

static inline bool bary_ok_map(F3 w) {
  return w.x >= -1e-5f && w.y >= -1e-5f && w.y <= 1.0f && w.z >= -1e-5f && w.z <= 1.0f;
}

// Shaders/meshmapping_nobackfaces.comp:64-83 (sign = +1) and :123-142 (sign = -1)
static inline Hit tri_oneside(F3 o, F3 d, F3 a, F3 b, F3 c, float lo, float hi, int sign) {
  Hit h = {FLT_MAX, mk(0, 0, 0)};
  F3 n = normalize(cross(b - a, c - a));
  float nd = dot(d, n);
  if (sign > 0 ? nd > 0 : nd < 0) {
    float pn = dot(o, n);
    float t = (dot(a, n) - pn) / nd;
    if (t >= lo && t < hi) {
      F3 w = bary_d(o + d * t, a, b, c);
      if (bary_ok_map(w)) { h.t = t; h.w = w; }
    }
  }
  return h;
}

// Shaders/meshmapping.comp:65-85
static inline Hit tri_twoside(F3 o, F3 d, F3 a, F3 b, F3 c) {
  Hit h = {FLT_MAX, mk(0, 0, 0)};
  F3 n = normalize(cross(b - a, c - a));
  float nd = dot(d, n);
  if (std::fabs(nd) > 0) {
    float pn = dot(o, n);
    float t = (dot(a, n) - pn) / nd;
    if (t >= 0) {
      F3 w = bary_d(o + d * t, a, b, c);
      if (bary_ok_map(w)) { h.t = t; h.w = w; }
    }
  }
  return h;
}

struct Counters { uint64_t box, tri; };

struct SceneView {
  const FlatNode* nodes;
  uint32_t count;
  const float* pos4;
  const float* nrm4;
};

static inline F3 corner(const float* a4, uint32_t i) { return ld3(a4 + 4 * (size_t)i); }

// Shaders/meshmapping_nobackfaces.comp:102-121 and :161-180
static void walk_oneside(const SceneView& s, F3 o, F3 d, int sign, float& cur, uint32_t& id, F3& w, Counters* ctr) {
  uint32_t i = 0;
  while (i < s.count) {
    const FlatNode& n = s.nodes[i];
    if (ctr) ctr->box++;
    if (ray_box(o, d, n) < cur) {
      for (uint32_t k = n.start; k < n.end; k += 3) {
        if (ctr) ctr->tri++;
        Hit h = tri_oneside(o, d, corner(s.pos4, k), corner(s.pos4, k + 1), corner(s.pos4, k + 2), 0.0f, cur, sign);
        if (h.t != FLT_MAX) { cur = h.t; id = k; w = h.w; }
      }
      ++i;
    } else {
      i = n.jump;
    }
  }
}

// Shaders/meshmapping.comp:87-137
static float walk_twoside(const SceneView& s, F3 o, F3 d, float mint, uint32_t& id, F3& w, Counters* ctr) {
  uint32_t i = 0;
  while (i < s.count) {
    const FlatNode& n = s.nodes[i];
    if (ctr) ctr->box++;
    if (ray_box(o, d, n) < mint) {
      float lm = FLT_MAX;
      uint32_t lid = 0;
      F3 lw = mk(0, 0, 0);
      for (uint32_t k = n.start; k < n.end; k += 3) {
        if (ctr) ctr->tri++;
        Hit h = tri_twoside(o, d, corner(s.pos4, k), corner(s.pos4, k + 1), corner(s.pos4, k + 2));
        if (h.t >= 0.0f && h.t < lm) { lm = h.t; lid = k; lw = h.w; }
      }
      if (lm < mint) { mint = lm; id = lid; w = lw; }
      ++i;
    } else {
      i = n.jump;
    }
  }
  return mint;
}

// One texel of the mesh-mapping pass: outputs vec4(t, bary) and the hit index.
// max_d is the walks' initial closest distance (FLT_MAX in the shaders:
// meshmapping_nobackfaces.comp:193, meshmapping.comp:150); a miss writes
// t = FLT_MAX whatever it is.
static void map_texel(const SceneView& s, F3 p, F3 d, int cull, float max_d, float* coord, uint32_t* tidx,
                      Counters* ctr) {
  uint32_t id = kMiss;
  F3 w = mk(0, 0, 0);
  float t = max_d;
  if (cull) {
    walk_oneside(s, p, d, +1, t, id, w, ctr);
    walk_oneside(s, p, -d, -1, t, id, w, ctr);
  } else {
    t = std::fmin(t, walk_twoside(s, p, d, t, id, w, ctr));
    t = std::fmin(t, walk_twoside(s, p, -d, t, id, w, ctr));
  }
  if (id == kMiss) t = FLT_MAX;
  coord[0] = t; coord[1] = w.x; coord[2] = w.y; coord[3] = w.z;
  *tidx = id;
}

// Shaders/ao_step1.comp:71-92
static inline float tri_sample(F3 o, F3 d, F3 a, F3 b, F3 c) {
  F3 n = normalize(cross(b - a, c - a));
  float nd = dot(d, n);
  if (std::fabs(nd) > 0) {
    float pn = dot(o, n);
    float t = (dot(a, n) - pn) / nd;
    if (t >= 0) {
      F3 w = bary_f(o + d * t, a, b, c);
      if (w.x >= 0 && w.y >= 0 && w.y <= 1 && w.z >= 0 && w.z <= 1) return t;
    }
  }
  return FLT_MAX;
}

// Shaders/ao_step1.comp:94-138 (identical in bentnormals_step1 / thick_step1)
static float walk_sample(const SceneView& s, F3 o, F3 d, float lo, float hi, Counters* ctr) {
  float mint = FLT_MAX;
  uint32_t i = 0;
  while (i < s.count) {
    const FlatNode& n = s.nodes[i];
    if (ctr) ctr->box++;
    float a = ray_box(o, d, n);
    if (a < mint && a < hi) {
      float lm = FLT_MAX;
      for (uint32_t k = n.start; k < n.end; k += 3) {
        if (ctr) ctr->tri++;
        float t = tri_sample(o, d, corner(s.pos4, k), corner(s.pos4, k + 1), corner(s.pos4, k + 2));
        if (t >= lo && t < lm) lm = t;
      }
      if (lm < mint) mint = lm;
      ++i;
    } else {
      i = n.jump;
    }
  }
  return mint;
}

struct Frame { F3 o, d, tx, ty; };

// Shaders/ao_step0.comp:22-56
static inline Frame texel_frame(const SceneView& s, const float* coord, uint32_t tidx) {
  F3 w = mk(coord[1], coord[2], coord[3]);
  Frame f;
  f.o = w.x * corner(s.pos4, tidx) + w.y * corner(s.pos4, tidx + 1) + w.z * corner(s.pos4, tidx + 2);
  f.d = normalize(w.x * corner(s.nrm4, tidx) + w.y * corner(s.nrm4, tidx + 1) + w.z * corner(s.nrm4, tidx + 2));
  F3 d = f.d;
  f.ty = normalize(std::fabs(d.x) > std::fabs(d.y) ? mk(d.z, 0, -d.x) : mk(0, d.z, -d.y));
  f.tx = cross(d, f.ty);
  return f;
}

static inline F3 sample_dir(const Frame& f, F3 d, const float* s4) {
  return normalize(f.tx * s4[0] + f.ty * s4[1] + d * s4[2]);
}

enum Kind { kAO = 0, kBN = 1, kThick = 2 };

}  // namespace orc

using namespace orc;

// ================================================================ C ABI
// Every entry point returns 0 on success and a negative value on bad input.
extern "C" {

int orc_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

static MeshView view(uint32_t np, const float* pos, uint32_t nt, const float* uv, uint32_t nn, const float* nrm,
                     uint32_t nv, const uint32_t* vtx, uint32_t nf, const uint32_t* tri, const float* tan,
                     const float* bit) {
  MeshView m = {np, nt, nn, nv, nf, pos, uv, nrm, vtx, tri, tan, bit};
  return m;
}

int orc_face_normals(uint32_t np, const float* pos, uint32_t nv, const uint32_t* vtx, uint32_t nf,
                     const uint32_t* tri, uint32_t* vtx_out, float* nrm_out) {
  MeshView m = view(np, pos, 0, nullptr, 0, nullptr, nv, vtx, nf, tri, nullptr, nullptr);
  face_normals(m, vtx_out, nrm_out);
  return 0;
}

int orc_vertex_normals(uint32_t np, const float* pos, uint32_t nv, const uint32_t* vtx, uint32_t nf,
                       const uint32_t* tri, uint32_t* vtx_out, float* nrm_out) {
  MeshView m = view(np, pos, 0, nullptr, 0, nullptr, nv, vtx, nf, tri, nullptr, nullptr);
  vertex_normals(m, vtx_out, nrm_out);
  return 0;
}

// nrm_out must hold 3 * 3 * nf floats (upper bound); returns the normal count.
int orc_welded_normals(uint32_t np, const float* pos, uint32_t nv, const uint32_t* vtx, uint32_t nf,
                       const uint32_t* tri, uint32_t* vtx_out, float* nrm_out) {
  MeshView m = view(np, pos, 0, nullptr, 0, nullptr, nv, vtx, nf, tri, nullptr, nullptr);
  return (int)welded_normals(m, vtx_out, nrm_out);
}

int orc_tangent_space(uint32_t np, const float* pos, uint32_t nt, const float* uv, uint32_t nn, const float* nrm,
                      uint32_t nv, const uint32_t* vtx, uint32_t nf, const uint32_t* tri, float* tan_out,
                      float* bit_out) {
  MeshView m = view(np, pos, nt, uv, nn, nrm, nv, vtx, nf, tri, nullptr, nullptr);
  tangent_space(m, tan_out, bit_out);
  return 0;
}

// BVH build + flatten.  Returns an opaque scene handle (null on failure).
void* orc_scene_build(uint32_t np, const float* pos, uint32_t nn, const float* nrm, uint32_t nv,
                      const uint32_t* vtx, uint32_t nf, const uint32_t* tri, uint32_t max_tris,
                      uint32_t max_depth) {
  MeshView m = view(np, pos, 0, nullptr, nn, nrm, nv, vtx, nf, tri, nullptr, nullptr);
  Builder b(m, max_tris, max_depth);
  b.build();
  Scene* s = new Scene();
  flatten(m, b.nodes, 0, *s);
  return s;
}

int orc_scene_sizes(void* h, uint32_t* nodes, uint32_t* corners) {
  Scene* s = (Scene*)h;
  *nodes = (uint32_t)s->nodes.size();
  *corners = (uint32_t)(s->pos4.size() / 4);
  return 0;
}

int orc_scene_copy(void* h, void* nodes36, float* pos4, float* nrm4) {
  Scene* s = (Scene*)h;
  if (!s->nodes.empty()) std::memcpy(nodes36, s->nodes.data(), s->nodes.size() * sizeof(FlatNode));
  if (!s->pos4.empty()) std::memcpy(pos4, s->pos4.data(), s->pos4.size() * sizeof(float));
  if (!s->nrm4.empty()) std::memcpy(nrm4, s->nrm4.data(), s->nrm4.size() * sizeof(float));
  return 0;
}

void orc_scene_free(void* h) { delete (Scene*)h; }

// UV raster + compaction.  dvtx/dnrm: mapping-direction normals (may be null).
void* orc_raster(uint32_t np, const float* pos, uint32_t nt, const float* uv, uint32_t nn, const float* nrm,
                 uint32_t nv, const uint32_t* vtx, uint32_t nf, const uint32_t* tri, const float* tan,
                 const float* bit, const uint32_t* dvtx, const float* dnrm, uint32_t w, uint32_t h, int mode,
                 float edge) {
  MeshView m = view(np, pos, nt, uv, nn, nrm, nv, vtx, nf, tri, tan, bit);
  MapOut* out = new MapOut();
  out->w = w;
  out->h = h;
  size_t n = (size_t)w * h;
  out->pos.assign(n, mk(0, 0, 0));
  out->dir.assign(n, mk(0, 0, 0));
  out->nrm.assign(n, mk(0, 0, 0));
  out->tan.assign(n, mk(0, 0, 0));
  out->bit.assign(n, mk(0, 0, 0));
  for (uint32_t f = 0; f < nf; ++f) {
    if (!raster_tri(m, dvtx, dnrm, f, mode, edge, *out)) { delete out; return nullptr; }
  }
  return out;
}

// Src/compute.cpp:372-416: texels with dot(dir, dir) > 0.5 in row-major order.
int orc_compress(void* hmap, uint32_t* count, uint32_t* idx, float* pos, float* dir, float* nrm, float* tan,
                 float* bit) {
  MapOut* m = (MapOut*)hmap;
  uint32_t c = 0;
  for (size_t i = 0; i < m->dir.size(); ++i) {
    if (dot(m->dir[i], m->dir[i]) > 0.5f) {
      if (idx) {
        idx[c] = (uint32_t)i;
        st3(pos + 3 * (size_t)c, m->pos[i]);
        st3(dir + 3 * (size_t)c, m->dir[i]);
        st3(nrm + 3 * (size_t)c, m->nrm[i]);
        st3(tan + 3 * (size_t)c, m->tan[i]);
        st3(bit + 3 * (size_t)c, m->bit[i]);
      }
      ++c;
    }
  }
  *count = c;
  return 0;
}

void orc_map_free(void* h) { delete (MapOut*)h; }

// Src/math.h:314-382 with a seeded engine in place of std::random_device.
int orc_samples(uint32_t spp, uint32_t perms, uint32_t seed, float* out4) {
  std::mt19937 eng(seed);
  std::uniform_int_distribution<uint32_t> dist;
  for (uint32_t j = 0; j < perms; ++j) {
    uint32_t rx = dist(eng);
    uint32_t ry = dist(eng);
    for (uint32_t i = 0; i < spp; ++i) {
      uint32_t r = i;
      r = (r << 16u) | (r >> 16u);
      r = ((r & 0x55555555u) << 1u) | ((r & 0xAAAAAAAAu) >> 1u);
      r = ((r & 0x33333333u) << 2u) | ((r & 0xCCCCCCCCu) >> 2u);
      r = ((r & 0x0F0F0F0Fu) << 4u) | ((r & 0xF0F0F0F0u) >> 4u);
      r = ((r & 0x00FF00FFu) << 8u) | ((r & 0xFF00FF00u) >> 8u);
      float x = float(i) / float(spp) + float(rx & 0xffffu) / float(1 << 16);
      float y = float(r ^ ry) * 2.3283064365386963e-10f;
      float ux = x - (float)(long)x;
      float rad = std::sqrt(ux);
      float phi = (float)(2.0 * 3.14159265) * y;
      float* o = out4 + 4 * ((size_t)j * spp + i);
      o[0] = rad * std::cos(phi);
      o[1] = rad * std::sin(phi);
      o[2] = std::sqrt(1.0f - ux);
      o[3] = 0.0f;
    }
  }
  return 0;
}

static SceneView sview(const void* nodes, uint32_t count, const float* pos4, const float* nrm4) {
  SceneView s = {(const FlatNode*)nodes, count, pos4, nrm4};
  return s;
}

// Mesh mapping over texels [0, count).  pix8: 8 floats per texel (p.xyz, pad,
// d.xyz, pad) = Pix_GPUData (Src/meshmapping.h:15-20).  counters (optional):
// total box / triangle tests.
int orc_meshmap(const void* nodes, uint32_t nnodes, const float* pos4, const float* pix8, uint32_t count, int cull,
                float max_d, float* coords, uint32_t* tidx, uint64_t* counters) {
  SceneView s = sview(nodes, nnodes, pos4, nullptr);
  uint64_t tb = 0, tt = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tb, tt)
  for (int64_t i = 0; i < (int64_t)count; ++i) {
    Counters c = {0, 0};
    const float* px = pix8 + 8 * (size_t)i;
    map_texel(s, ld3(px), ld3(px + 4), cull, max_d, coords + 4 * (size_t)i, tidx + i, counters ? &c : nullptr);
    tb += c.box;
    tt += c.tri;
  }
  if (counters) { counters[0] = tb; counters[1] = tt; }
  return 0;
}

// Hemisphere sampling (AO / bent normals / thickness) for the texels listed in
// `texels` (global compressed indices; null = 0..n-1), each with `spp` samples,
// sample row (texel % perms).  Writes the step2 aggregate per listed texel:
// AO 1 float, BN 3 floats, thickness 1 float, plus `hits` = number of samples
// whose closest hit is occluding (AO: t < max; BN and thickness: t != FLT_MAX).
// Texels whose mapping missed are skipped (outputs left untouched).
int orc_hemisphere(int kind, const void* nodes, uint32_t nnodes, const float* pos4, const float* nrm4,
                   const float* coords, const uint32_t* tidx, const float* samples4, uint32_t spp, uint32_t perms,
                   float min_d, float max_d, const uint32_t* texels, uint32_t n, float* out, uint32_t* hits,
                   uint64_t* counters) {
  SceneView s = sview(nodes, nnodes, pos4, nrm4);
  uint64_t tb = 0, tt = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : tb, tt)
  for (int64_t j = 0; j < (int64_t)n; ++j) {
    uint32_t g = texels ? texels[j] : (uint32_t)j;
    uint32_t id = tidx[g];
    if (id == kMiss) continue;
    Counters c = {0, 0};
    Counters* cp = counters ? &c : nullptr;
    Frame f = texel_frame(s, coords + 4 * (size_t)g, id);
    F3 d = kind == kThick ? -f.d : f.d;
    const float* row = samples4 + 4 * (size_t)(g % perms) * spp;
    float acc = 0.0f;
    F3 vacc = mk(0, 0, 0);
    uint32_t nh = 0;
    for (uint32_t k = 0; k < spp; ++k) {
      F3 dir = sample_dir(f, d, row + 4 * (size_t)k);
      float t = walk_sample(s, f.o, dir, min_d, max_d, cp);
      if (kind == kAO) {
        float v = (t != FLT_MAX && t < max_d) ? 1.0f : 0.0f;
        acc += v;
        nh += v != 0.0f;
      } else if (kind == kBN) {
        vacc = vacc + ((t != FLT_MAX) ? mk(0, 0, 0) : dir);
        nh += t != FLT_MAX;
      } else {
        acc += (t != FLT_MAX) ? t : max_d;
        nh += t != FLT_MAX;
      }
    }
    if (kind == kAO) out[j] = 1.0f - acc / float(spp);
    else if (kind == kBN) st3(out + 3 * (size_t)j, normalize(vacc));
    else out[j] = acc / float(spp);
    if (hits) hits[j] = nh;
    tb += c.box;
    tt += c.tri;
  }
  if (counters) { counters[0] = tb; counters[1] = tt; }
  return 0;
}

// Per-sample closest-hit distances of one texel (test helper for single rays).
int orc_sample_rays(int kind, const void* nodes, uint32_t nnodes, const float* pos4, const float* nrm4,
                    const float* coords, const uint32_t* tidx, const float* samples4, uint32_t spp, uint32_t perms,
                    float min_d, float max_d, uint32_t g, float* t_out) {
  SceneView s = sview(nodes, nnodes, pos4, nrm4);
  uint32_t id = tidx[g];
  if (id == kMiss) return -1;
  Frame f = texel_frame(s, coords + 4 * (size_t)g, id);
  F3 d = kind == kThick ? -f.d : f.d;
  const float* row = samples4 + 4 * (size_t)(g % perms) * spp;
  for (uint32_t k = 0; k < spp; ++k) t_out[k] = walk_sample(s, f.o, sample_dir(f, d, row + 4 * (size_t)k), min_d, max_d, nullptr);
  return 0;
}

// Shaders/heights.comp, positions.comp, normals.comp (0/1/2).  Texels with a
// missed mapping: height 0 (the shader's own rule), position / normal left 0.
int orc_gather(int what, const float* pos4, const float* nrm4, const float* coords, const uint32_t* tidx, uint32_t n,
               float* out) {
  for (uint32_t i = 0; i < n; ++i) {
    const float* c = coords + 4 * (size_t)i;
    if (what == 0) { out[i] = c[0] != FLT_MAX ? c[0] : 0.0f; continue; }
    uint32_t id = tidx[i];
    if (id == kMiss) { st3(out + 3 * (size_t)i, mk(0, 0, 0)); continue; }
    const float* src = what == 1 ? pos4 : nrm4;
    F3 v = c[1] * corner(src, id) + c[2] * corner(src, id + 1) + c[3] * corner(src, id + 2);
    st3(out + 3 * (size_t)i, what == 1 ? v : normalize(v));
  }
  return 0;
}

// Shaders/tangentspace.comp:22-41, in place on n float3 values.
int orc_tangent_transform(const float* n3, const float* t3, const float* b3, uint32_t n, float* io3) {
  for (uint32_t i = 0; i < n; ++i) {
    F3 v = ld3(io3 + 3 * (size_t)i);
    F3 N = ld3(n3 + 3 * (size_t)i), T = ld3(t3 + 3 * (size_t)i), B = ld3(b3 + 3 * (size_t)i);
    F3 d0 = mk(N.z * B.y - N.y * B.z, N.x * B.z - N.z * B.x, N.y * B.x - N.x * B.y);
    F3 d1 = mk(T.z * N.y - T.y * N.z, T.x * N.z - N.x * T.z, N.x * T.y - T.x * N.y);
    F3 d2 = mk(T.y * B.z - T.z * B.y, T.z * B.x - T.x * B.z, T.x * B.y - T.y * B.x);
    st3(io3 + 3 * (size_t)i, normalize(mk(dot(v, d0), dot(v, d1), dot(v, d2))));
  }
  return 0;
}

// ---------------------------------------------------------------- export
// Src/image.cpp:22-405: compressed texel values scattered into a W x H image
// (rows flipped: texel (x, y) lands in row h - y - 1), quantized to RGB8 or
// kept as float, and, for RGB8, dilated.  dilateRGB runs its pixels in row
// order; this restatement keeps that order, so a source centre that is itself
// an uncovered pixel gives the value it has at that point of the scan.

// (uint8_t) of a float as x86-64 code converts it: truncation to int32
// (0x80000000 for NaN and out-of-range values), low byte kept.
static inline uint8_t u8_of(float v) {
  if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
  return (uint8_t)(int32_t)v;
}

// dilateRGB (Src/image.cpp:127-182) on an RGB8 image in file row order.
static void dilate_rgb(uint8_t* data, int w, int h, const std::vector<uint8_t>& valid, int max_dist) {
  static const int off[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      if (valid[x + (size_t)y * w]) continue;
      bool filled = false;
      for (int dist = 1; dist < max_dist && !filled; ++dist)
        for (int k = 0; k < 8; ++k) {
          const int cx = x + off[k][0] * dist, cy = y + off[k][1] * dist;
          if (!(cx > 0 && cy > 0 && cx < w - 1 && cy < h - 1)) continue;
          bool ok = true;
          for (int q = 0; q < 8 && ok; ++q) ok = valid[(cx + off[q][0]) + (size_t)(cy + off[q][1]) * w] != 0;
          if (!ok) continue;
          const size_t src = ((size_t)(h - cy - 1) * w + cx) * 3, dst = ((size_t)(h - y - 1) * w + x) * 3;
          data[dst] = data[src];
          data[dst + 1] = data[src + 1];
          data[dst + 2] = data[src + 2];
          filled = true;
          break;
        }
    }
}

// exportFloatImage (Src/image.cpp:188-297).  rgb8 != 0: the PNG / TGA path
// (out w x h x 3 bytes, dilated when dilate > 0); else the EXR path (out w x h
// floats).  minmax gets the range it used.
int orc_export_float(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx, const float* data, float flo,
                     float fhi, int normalize, int dilate, int rgb8, void* out, float* minmax) {
  float mn = FLT_MAX, mx = -FLT_MAX;
  for (uint32_t i = 0; i < count; ++i) {
    mn = std::fminf(mn, data[i]);
    mx = std::fmaxf(mx, data[i]);
  }
  const bool filter = fhi > flo;
  if (filter) {
    mn = std::fmaxf(mn, flo);
    mx = std::fminf(mx, fhi);
  }
  minmax[0] = mn;
  minmax[1] = mx;
  float scale = 1.0f, bias = 0.0f;
  if (normalize && mn != FLT_MAX && mx != -FLT_MAX) {
    scale = 1.0f / (mx - mn);
    bias = -mn * scale;
  }
  if (rgb8) {
    uint8_t* rgb = (uint8_t*)out;
    std::memset(rgb, 0, (size_t)w * h * 3);
    for (uint32_t i = 0; i < count; ++i) {
      const float d = data[i];
      const float df = filter && (d < flo || d > fhi) ? 0 : d;
      const float t = df * scale + bias;
      const uint8_t c = u8_of(std::min(std::max(t, 0.0f), 1.0f) * 255.0f);
      const size_t x = idx[i] % w, y = idx[i] / w, p = ((h - y - 1) * w + x) * 3;
      rgb[p] = rgb[p + 1] = rgb[p + 2] = c;
    }
    if (dilate > 0) {
      std::vector<uint8_t> valid((size_t)w * h, 0);
      for (uint32_t i = 0; i < count; ++i) valid[idx[i]] = 1;
      dilate_rgb(rgb, (int)w, (int)h, valid, dilate);
    }
  } else {
    float* f = (float*)out;
    std::memset(f, 0, sizeof(float) * (size_t)w * h);
    for (uint32_t i = 0; i < count; ++i) {
      const float d = data[i];
      const float df = filter ? std::fminf(std::fmaxf(d, flo), fhi) : d;
      const float t = normalize ? df * scale + bias : df;
      const size_t x = idx[i] % w, y = idx[i] / w;
      f[(h - y - 1) * w + x] = t;
    }
  }
  return 0;
}

// exportNormalImage's PNG / TGA path (Src/image.cpp:358-393): n * 0.5 + 0.5
// to bytes, dilated when dilate > 0 over the pixels whose bytes are not all
// zero.  The valid table uses y = index / h as the reference does (the same as
// index / w for square maps); indices whose row would fall outside the image
// are left invalid.
int orc_export_normal(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx, const float* data3, int dilate,
                      uint8_t* rgb) {
  std::memset(rgb, 0, (size_t)w * h * 3);
  for (uint32_t i = 0; i < count; ++i) {
    const float nx = data3[3 * (size_t)i] * 0.5f + 0.5f, ny = data3[3 * (size_t)i + 1] * 0.5f + 0.5f,
                nz = data3[3 * (size_t)i + 2] * 0.5f + 0.5f;
    const size_t x = idx[i] % w, y = idx[i] / w, p = ((h - y - 1) * w + x) * 3;
    rgb[p] = u8_of(nx * 255.0f);
    rgb[p + 1] = u8_of(ny * 255.0f);
    rgb[p + 2] = u8_of(nz * 255.0f);
  }
  if (dilate > 0) {
    std::vector<uint8_t> valid((size_t)w * h, 0);
    for (uint32_t i = 0; i < count; ++i) {
      const size_t x = idx[i] % w, y = idx[i] / h;
      if (y >= h) continue;
      const size_t p = ((h - y - 1) * w + x) * 3;
      valid[idx[i]] = (rgb[p] != 0) | (rgb[p + 1] != 0) | (rgb[p + 2] != 0);
    }
    dilate_rgb(rgb, (int)w, (int)h, valid, dilate);
  }
  return 0;
}

// exportVectorImage (Src/image.cpp:299-356): three float planes in file row
// order, plane 0 = z, 1 = y, 2 = x (channels B, G, R).
int orc_export_vector(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx, const float* data3, float* planes) {
  std::memset(planes, 0, sizeof(float) * 3 * (size_t)w * h);
  for (uint32_t i = 0; i < count; ++i) {
    const size_t x = idx[i] % w, y = idx[i] / w, p = (h - y - 1) * w + x;
    planes[p] = data3[3 * (size_t)i + 2];
    planes[(size_t)w * h + p] = data3[3 * (size_t)i + 1];
    planes[2 * (size_t)w * h + p] = data3[3 * (size_t)i];
  }
  return 0;
}

}  // extern "C"
