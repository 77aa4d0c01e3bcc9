// Host mesh handling: the indexed mesh of Src/mesh.h:35-63, its normal and
// tangent generators (Src/mesh.cpp:619-768) and the cosine-weighted sample
// table (Src/math.h:314-382).  Arithmetic is binary32 in the reference's
// evaluation order (the library is built with -ffp-contract=off), so the
// results are the reference's bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <system_error>
#include <thread>
#include <unordered_map>

#include "fk_internal.h"

namespace {

struct V3 {
  float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, float k) { return v3(a.x * k, a.y * k, a.z * k); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V3 normalize(V3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline V3 get3(const std::vector<float>& a, size_t i) { return v3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
inline void put3(std::vector<float>& a, size_t i, V3 v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }

inline V3 corner_pos(const fk_mesh& m, uint32_t f, int k) {
  return get3(m.positions, m.vertices[3 * (size_t)m.triangles[3 * (size_t)f + k]]);
}

inline V3 face_normal(const fk_mesh& m, uint32_t f) {
  V3 p0 = corner_pos(m, f, 0), p1 = corner_pos(m, f, 1), p2 = corner_pos(m, f, 2);
  return normalize(cross(p1 - p0, p2 - p0));
}

bool valid(const fk_mesh& m) {
  uint32_t np = m.position_count(), nv = m.vertex_count();
  for (uint32_t t : m.triangles)
    if (t >= nv) return false;
  for (uint32_t v = 0; v < nv; ++v)
    if (m.vertices[3 * (size_t)v] >= np) return false;
  return true;
}

// Key equality of the reference's std::map<Vector3> (Src/mesh.cpp:38-41):
// float comparison, so +0 and -0 weld; the bit patterns are canonicalised.
struct PosKey {
  uint32_t b[3];
  bool operator==(const PosKey& o) const { return b[0] == o.b[0] && b[1] == o.b[1] && b[2] == o.b[2]; }
};
struct PosKeyHash {
  size_t operator()(const PosKey& k) const {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < 3; ++i) h = (h ^ k.b[i]) * 1099511628211ull;
    return (size_t)h;
  }
};
inline PosKey key_of(V3 p) {
  PosKey k;
  float c[3] = {p.x + 0.0f, p.y + 0.0f, p.z + 0.0f};
  std::memcpy(k.b, c, sizeof(c));
  return k;
}

}  // namespace

extern "C" {

int fk_mesh_create(const fk_mesh_desc* d, fk_mesh** out) {
  if (!d || !out) return FK_ERR_INVALID;
  if ((d->position_count && !d->positions) || (d->texcoord_count && !d->texcoords) ||
      (d->normal_count && !d->normals) || (d->vertex_count && !d->vertices) || (d->triangle_count && !d->triangles))
    return FK_ERR_INVALID;
  fk_mesh* m = new (std::nothrow) fk_mesh();
  if (!m) return FK_ERR_NOMEM;
  m->positions.assign(d->positions, d->positions + 3 * (size_t)d->position_count);
  m->texcoords.assign(d->texcoords, d->texcoords + 2 * (size_t)d->texcoord_count);
  m->normals.assign(d->normals, d->normals + 3 * (size_t)d->normal_count);
  m->vertices.assign(d->vertices, d->vertices + 3 * (size_t)d->vertex_count);
  m->triangles.assign(d->triangles, d->triangles + 3 * (size_t)d->triangle_count);
  if (d->tangents && d->bitangents) {
    m->tangents.assign(d->tangents, d->tangents + 3 * (size_t)d->vertex_count);
    m->bitangents.assign(d->bitangents, d->bitangents + 3 * (size_t)d->vertex_count);
  }
  if (!valid(*m)) {
    delete m;
    return FK_ERR_INVALID;
  }
  *out = m;
  return FK_OK;
}

int fk_mesh_describe(const fk_mesh* m, fk_mesh_desc* d) {
  if (!m || !d) return FK_ERR_INVALID;
  d->position_count = m->position_count();
  d->positions = m->positions.data();
  d->texcoord_count = (uint32_t)(m->texcoords.size() / 2);
  d->texcoords = m->texcoords.data();
  d->normal_count = (uint32_t)(m->normals.size() / 3);
  d->normals = m->normals.data();
  d->vertex_count = m->vertex_count();
  d->vertices = m->vertices.data();
  d->triangle_count = m->triangle_count();
  d->triangles = m->triangles.data();
  d->tangents = m->tangents.empty() ? nullptr : m->tangents.data();
  d->bitangents = m->bitangents.empty() ? nullptr : m->bitangents.data();
  return FK_OK;
}

int fk_mesh_copy(const fk_mesh* m, fk_mesh** out) {
  if (!m || !out) return FK_ERR_INVALID;
  *out = new (std::nothrow) fk_mesh(*m);
  return *out ? FK_OK : FK_ERR_NOMEM;
}

int fk_mesh_free(fk_mesh* m) {
  delete m;
  return FK_OK;
}

// Src/mesh.cpp:627-648: one normal per triangle; each corner's vertex points
// at it (a vertex shared by several triangles keeps the last one).
int fk_mesh_compute_face_normals(fk_mesh* m) {
  if (!m) return FK_ERR_INVALID;
  uint32_t nf = m->triangle_count();
  std::vector<float> n(3 * (size_t)nf);
  for (uint32_t f = 0; f < nf; ++f) {
    put3(n, f, face_normal(*m, f));
    for (int k = 0; k < 3; ++k) m->vertices[3 * (size_t)m->triangles[3 * (size_t)f + k] + 2] = f;
  }
  m->normals.swap(n);
  return FK_OK;
}

// Src/mesh.cpp:650-678: unweighted face normals summed per position, in
// triangle order; every vertex then uses its position's normal.
int fk_mesh_compute_vertex_normals(fk_mesh* m) {
  if (!m) return FK_ERR_INVALID;
  uint32_t np = m->position_count(), nf = m->triangle_count();
  std::vector<V3> acc(np, v3(0, 0, 0));
  for (uint32_t f = 0; f < nf; ++f) {
    V3 n = face_normal(*m, f);
    for (int k = 0; k < 3; ++k) {
      uint32_t p = m->vertices[3 * (size_t)m->triangles[3 * (size_t)f + k]];
      acc[p] = acc[p] + n;
    }
  }
  m->normals.assign(3 * (size_t)np, 0.0f);
  for (uint32_t i = 0; i < np; ++i) put3(m->normals, i, normalize(acc[i]));
  for (uint32_t v = 0; v < m->vertex_count(); ++v) m->vertices[3 * (size_t)v + 2] = m->vertices[3 * (size_t)v];
  return FK_OK;
}

// Src/mesh.cpp:680-722: normals welded across equal positions, numbered in
// the order positions are first met.
int fk_mesh_compute_vertex_normals_welded(fk_mesh* m) {
  if (!m) return FK_ERR_INVALID;
  uint32_t nf = m->triangle_count();
  std::unordered_map<PosKey, uint32_t, PosKeyHash> slot;
  slot.reserve(3 * (size_t)nf);
  std::vector<V3> acc;
  for (uint32_t f = 0; f < nf; ++f) {
    V3 n = face_normal(*m, f);
    for (int k = 0; k < 3; ++k) {
      V3 p = corner_pos(*m, f, k);
      auto ins = slot.emplace(key_of(p), (uint32_t)acc.size());
      uint32_t id = ins.first->second;
      if (ins.second) acc.push_back(n);
      else acc[id] = acc[id] + n;
      m->vertices[3 * (size_t)m->triangles[3 * (size_t)f + k] + 2] = id;
    }
  }
  m->normals.assign(3 * acc.size(), 0.0f);
  for (size_t i = 0; i < acc.size(); ++i) put3(m->normals, i, normalize(acc[i]));
  return FK_OK;
}

// Src/mesh.cpp:724-768: per-vertex tangent from texcoord derivatives,
// Gram-Schmidt against the vertex normal, bitangent = n x t.
int fk_mesh_compute_tangent_space(fk_mesh* m) {
  if (!m) return FK_ERR_INVALID;
  uint32_t nv = m->vertex_count(), nf = m->triangle_count();
  uint32_t nt = (uint32_t)(m->texcoords.size() / 2), nn = (uint32_t)(m->normals.size() / 3);
  for (uint32_t v = 0; v < nv; ++v)
    if (m->vertices[3 * (size_t)v + 1] >= nt || m->vertices[3 * (size_t)v + 2] >= nn) return FK_ERR_INVALID;
  std::vector<V3> t(nv, v3(0, 0, 0)), b(nv, v3(0, 0, 0));
  for (uint32_t f = 0; f < nf; ++f) {
    uint32_t vi[3];
    V3 p[3];
    float u[3][2];
    for (int k = 0; k < 3; ++k) {
      vi[k] = m->triangles[3 * (size_t)f + k];
      const uint32_t* v = &m->vertices[3 * (size_t)vi[k]];
      p[k] = get3(m->positions, v[0]);
      u[k][0] = m->texcoords[2 * (size_t)v[1]];
      u[k][1] = m->texcoords[2 * (size_t)v[1] + 1];
    }
    V3 e0 = p[1] - p[0], e1 = p[2] - p[0];
    float t0x = u[1][0] - u[0][0], t0y = u[1][1] - u[0][1];
    float t1x = u[2][0] - u[0][0], t1y = u[2][1] - u[0][1];
    float r = 1.0f / (t0x * t1y - t1x * t0y);
    V3 sdir = (e0 * t1y - e1 * t0y) * r;
    V3 tdir = (e1 * t0x - e0 * t1x) * r;
    for (int k = 0; k < 3; ++k) {
      t[vi[k]] = t[vi[k]] + sdir;
      b[vi[k]] = b[vi[k]] + tdir;
    }
  }
  m->tangents.assign(3 * (size_t)nv, 0.0f);
  m->bitangents.assign(3 * (size_t)nv, 0.0f);
  for (uint32_t i = 0; i < nv; ++i) {
    V3 n = get3(m->normals, m->vertices[3 * (size_t)i + 2]);
    V3 tt = normalize(t[i] - n * dot(n, t[i]));
    put3(m->tangents, i, tt);
    put3(m->bitangents, i, cross(n, tt));
  }
  return FK_OK;
}

// Src/math.h:339-382: Hammersley points randomised per row by (randX, randY),
// mapped to the cosine-weighted hemisphere.  The engine is std::mt19937 as in
// the reference, seeded with `seed` instead of std::random_device.
int fk_samples_cosine(uint32_t spp, uint32_t perms, uint32_t seed, float* out4) {
  if (!out4 || spp == 0 || perms == 0) return FK_ERR_INVALID;
  // The rows' random words are drawn in order from one engine; the rows are
  // then independent and are filled on several threads (the same operations
  // per sample, so the table does not depend on the thread count).
  std::mt19937 eng(seed);
  std::uniform_int_distribution<uint32_t> dist;
  std::vector<uint32_t> words(2 * (size_t)perms);
  for (uint32_t row = 0; row < perms; ++row) {
    words[2 * (size_t)row] = dist(eng);
    words[2 * (size_t)row + 1] = dist(eng);
  }
  const float two_pi = (float)(2.0 * 3.14159265);
  auto fill = [&](uint32_t row) {
    const uint32_t rx = words[2 * (size_t)row], ry = words[2 * (size_t)row + 1];
    float xoff = float(rx & 0xffffu) / float(1 << 16);
    for (uint32_t i = 0; i < spp; ++i) {
      uint32_t rev = i;
      rev = (rev << 16u) | (rev >> 16u);
      rev = ((rev & 0x55555555u) << 1u) | ((rev & 0xAAAAAAAAu) >> 1u);
      rev = ((rev & 0x33333333u) << 2u) | ((rev & 0xCCCCCCCCu) >> 2u);
      rev = ((rev & 0x0F0F0F0Fu) << 4u) | ((rev & 0xF0F0F0F0u) >> 4u);
      rev = ((rev & 0x00FF00FFu) << 8u) | ((rev & 0xFF00FF00u) >> 8u);
      float x = float(i) / float(spp) + xoff;
      float u = x - (float)(long)x;
      float v = float(rev ^ ry) * 2.3283064365386963e-10f;
      float r = std::sqrt(u);
      float phi = two_pi * v;
      float* o = out4 + 4 * ((size_t)row * spp + i);
      o[0] = r * std::cos(phi);
      o[1] = r * std::sin(phi);
      o[2] = std::sqrt(1.0f - u);
      o[3] = 0.0f;
    }
  };
  const uint64_t work = (uint64_t)spp * perms;
  const unsigned threads = work < (1u << 16) ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (threads == 1) {
    for (uint32_t row = 0; row < perms; ++row) fill(row);
    return FK_OK;
  }
  std::vector<std::thread> pool;
  pool.reserve(threads);
  unsigned t = 0;
  try {
    for (; t < threads; ++t)
      pool.emplace_back([&, t] {
        for (uint32_t row = t; row < perms; row += threads) fill(row);
      });
  } catch (const std::system_error&) {  // no more threads: the remaining rows here
  }
  for (unsigned u = t; u < threads; ++u)
    for (uint32_t row = u; row < perms; row += threads) fill(row);
  for (auto& th : pool) th.join();
  return FK_OK;
}

}  // extern "C"
