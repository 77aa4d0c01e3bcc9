// extern "C" entry points over the reference's own host code (compiled from the
// reference tree by oracle/build_ref.py).  Test infrastructure only: these pin
// the oracle restatement (oracle/oracle.cpp) to the reference's behaviour.
//
// Including Src/meshmapping.cpp here reaches fillMeshData, which sits in an
// anonymous namespace (Src/meshmapping.cpp:33-126).  The GL-facing functions it
// and Src/compute.cpp refer to are linked but never called.
#include "meshmapping.cpp"

#include "bvh.h"
#include "compute.h"
#include "image.h"
#include "mesh.h"
#include <cstring>
#include <omp.h>

static unsigned int g_seed = 0;
unsigned int std::fornos_seeded_device::operator()() { return g_seed; }

// Logging is not part of the path; silent stand-ins.  exportNormalImage is the
// name CompressedMapUV's constructor calls for a debug file
// (Src/compute.cpp:413-415): a no-op here; the reference's function itself is
// compiled as ref_exportNormalImage (oracle/build_ref.py).
void logDebug(const std::string&, const std::string&) {}
void logWarning(const std::string&, const std::string&) {}
void logError(const std::string&, const std::string&) {}
void exportNormalImage(const Vector3*, const CompressedMapUV*, const char*, int) {}
void ref_exportNormalImage(const Vector3* data, const CompressedMapUV* map, const char* path, int dilate);
void exportVectorImage(const Vector3* data, const CompressedMapUV* map, const char* path);
GLuint LoadComputeShader_MeshMapping() { return 0; }
GLuint LoadComputeShader_MeshMappingCullBackfaces() { return 0; }

static Mesh* make_mesh(uint32_t np, const float* pos, uint32_t nt, const float* uv, uint32_t nn, const float* nrm,
                       uint32_t nv, const uint32_t* vtx, uint32_t nf, const uint32_t* tri) {
  Mesh* m = new Mesh();
  m->positions.resize(np);
  for (uint32_t i = 0; i < np; ++i) m->positions[i] = Vector3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  m->texcoords.resize(nt);
  for (uint32_t i = 0; i < nt; ++i) m->texcoords[i] = Vector2(uv[2 * i], uv[2 * i + 1]);
  m->normals.resize(nn);
  for (uint32_t i = 0; i < nn; ++i) m->normals[i] = Vector3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
  m->vertices.resize(nv);
  for (uint32_t i = 0; i < nv; ++i) m->vertices[i] = Mesh::Vertex{vtx[3 * i], vtx[3 * i + 1], vtx[3 * i + 2]};
  m->triangles.resize(nf);
  for (uint32_t i = 0; i < nf; ++i) m->triangles[i] = Mesh::Triangle{tri[3 * i], tri[3 * i + 1], tri[3 * i + 2]};
  return m;
}

static void copy_normals(const Mesh* m, uint32_t* vtx_out, float* nrm_out) {
  for (size_t i = 0; i < m->vertices.size(); ++i) {
    vtx_out[3 * i] = m->vertices[i].positionIndex;
    vtx_out[3 * i + 1] = m->vertices[i].texcoordIndex;
    vtx_out[3 * i + 2] = m->vertices[i].normalIndex;
  }
  for (size_t i = 0; i < m->normals.size(); ++i) {
    nrm_out[3 * i] = m->normals[i].x;
    nrm_out[3 * i + 1] = m->normals[i].y;
    nrm_out[3 * i + 2] = m->normals[i].z;
  }
}

extern "C" {

// which: 0 face, 1 vertex, 2 welded (aggressive).  Returns the normal count.
int ref_normals(int which, uint32_t np, const float* pos, uint32_t nv, const uint32_t* vtx, uint32_t nf,
                const uint32_t* tri, uint32_t* vtx_out, float* nrm_out) {
  Mesh* m = make_mesh(np, pos, 0, nullptr, 0, nullptr, nv, vtx, nf, tri);
  if (which == 0) m->computeFaceNormals();
  else if (which == 1) m->computeVertexNormals();
  else m->computeVertexNormalsAggressive();
  copy_normals(m, vtx_out, nrm_out);
  int n = (int)m->normals.size();
  delete m;
  return n;
}

int ref_tangent_space(uint32_t np, const float* pos, uint32_t nt, const float* uv, uint32_t nn, const float* nrm,
                      uint32_t nv, const uint32_t* vtx, uint32_t nf, const uint32_t* tri, float* tan_out,
                      float* bit_out) {
  Mesh* m = make_mesh(np, pos, nt, uv, nn, nrm, nv, vtx, nf, tri);
  m->computeTangentSpace();
  for (uint32_t i = 0; i < nv; ++i) {
    tan_out[3 * i] = m->tangents[i].x; tan_out[3 * i + 1] = m->tangents[i].y; tan_out[3 * i + 2] = m->tangents[i].z;
    bit_out[3 * i] = m->bitangents[i].x; bit_out[3 * i + 1] = m->bitangents[i].y; bit_out[3 * i + 2] = m->bitangents[i].z;
  }
  delete m;
  return 0;
}

struct RefScene {
  std::vector<BVHGPUData> nodes;
  std::vector<Vector4> pos, nrm;
};

void* ref_scene_build(uint32_t np, const float* pos, uint32_t nn, const float* nrm, uint32_t nv, const uint32_t* vtx,
                      uint32_t nf, const uint32_t* tri, uint32_t max_tris, uint32_t max_depth) {
  Mesh* m = make_mesh(np, pos, 0, nullptr, nn, nrm, nv, vtx, nf, tri);
  BVH* root = BVH::createBinary(m, max_tris, max_depth);
  RefScene* s = new RefScene();
  fillMeshData(m, *root, s->nodes, s->pos, s->nrm);
  delete root;
  delete m;
  return s;
}

int ref_scene_sizes(void* h, uint32_t* nodes, uint32_t* corners) {
  RefScene* s = (RefScene*)h;
  *nodes = (uint32_t)s->nodes.size();
  *corners = (uint32_t)s->pos.size();
  return 0;
}

int ref_scene_copy(void* h, void* nodes36, float* pos4, float* nrm4) {
  RefScene* s = (RefScene*)h;
  static_assert(sizeof(BVHGPUData) == 36, "node layout");
  if (!s->nodes.empty()) std::memcpy(nodes36, s->nodes.data(), s->nodes.size() * 36);
  for (size_t i = 0; i < s->pos.size(); ++i) {
    pos4[4 * i] = s->pos[i].x; pos4[4 * i + 1] = s->pos[i].y; pos4[4 * i + 2] = s->pos[i].z; pos4[4 * i + 3] = s->pos[i].w;
    nrm4[4 * i] = s->nrm[i].x; nrm4[4 * i + 1] = s->nrm[i].y; nrm4[4 * i + 2] = s->nrm[i].z; nrm4[4 * i + 3] = s->nrm[i].w;
  }
  return 0;
}

void ref_scene_free(void* h) { delete (RefScene*)h; }

// mode: 0 Smooth (fromMeshes), 1 LowPolyNormals (fromMesh), 2 Hybrid.
// tan/bit: per-vertex tangent frame or null.  dvtx/dnrm: the direction mesh's
// vertex normal indices and normals (modes 0 and 2).
void* ref_raster(uint32_t np, const float* pos, uint32_t nt, const float* uv, uint32_t nn, const float* nrm,
                 uint32_t nv, const uint32_t* vtx, uint32_t nf, const uint32_t* tri, const float* tan,
                 const float* bit, const uint32_t* dvtx, uint32_t dnn, const float* dnrm, uint32_t w, uint32_t h,
                 int mode, float edge) {
  Mesh* m = make_mesh(np, pos, nt, uv, nn, nrm, nv, vtx, nf, tri);
  if (tan) {
    m->tangents.resize(nv);
    m->bitangents.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) {
      m->tangents[i] = Vector3(tan[3 * i], tan[3 * i + 1], tan[3 * i + 2]);
      m->bitangents[i] = Vector3(bit[3 * i], bit[3 * i + 1], bit[3 * i + 2]);
    }
  }
  Mesh* d = nullptr;
  if (mode != 1) {
    d = Mesh::createCopy(m);
    d->normals.resize(dnn);
    for (uint32_t i = 0; i < dnn; ++i) d->normals[i] = Vector3(dnrm[3 * i], dnrm[3 * i + 1], dnrm[3 * i + 2]);
    for (uint32_t i = 0; i < nv; ++i) d->vertices[i].normalIndex = dvtx[3 * i + 2];
  }
  MapUV* map = nullptr;
  if (mode == 0) map = MapUV::fromMeshes(m, d, w, h);
  else if (mode == 1) map = MapUV::fromMesh(m, w, h);
  else map = MapUV::fromMeshes_Hybrid(m, d, w, h, edge);
  CompressedMapUV* c = map ? new CompressedMapUV(map) : nullptr;
  delete map;
  delete d;
  delete m;
  return c;
}

int ref_cmap_copy(void* h, uint32_t* count, uint32_t* idx, float* pos, float* dir, float* nrm, float* tan,
                  float* bit) {
  CompressedMapUV* c = (CompressedMapUV*)h;
  *count = (uint32_t)c->indices.size();
  if (!idx) return 0;
  for (size_t i = 0; i < c->indices.size(); ++i) {
    idx[i] = c->indices[i];
    const Vector3* src[5] = {&c->positions[i], &c->directions[i], &c->normals[i], &c->tangents[i], &c->bitangents[i]};
    float* dst[5] = {pos, dir, nrm, tan, bit};
    for (int k = 0; k < 5; ++k) {
      dst[k][3 * i] = src[k]->x; dst[k][3 * i + 1] = src[k]->y; dst[k][3 * i + 2] = src[k]->z;
    }
  }
  return 0;
}

void ref_cmap_free(void* h) { delete (CompressedMapUV*)h; }

// Src/math.h:363-382, engine seeded with `seed` through the shim.
int ref_samples(uint32_t spp, uint32_t perms, uint32_t seed, float* out4) {
  g_seed = seed;
  std::vector<Vector3> v((size_t)spp * perms);
  computeSamplesImportanceCosDir(spp, perms, v.data());
  for (size_t i = 0; i < v.size(); ++i) {
    out4[4 * i] = v[i].x; out4[4 * i + 1] = v[i].y; out4[4 * i + 2] = v[i].z; out4[4 * i + 3] = 0.0f;
  }
  return 0;
}

// A compressed map holding exactly the texels `idx` (ascending) of a w x h
// map: CompressedMapUV keeps the texels whose direction has length > 0.5.
static CompressedMapUV* make_cmap(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx) {
  MapUV m(w, h);
  for (uint32_t i = 0; i < count; ++i) m.directions[idx[i]] = Vector3(1.0f, 0.0f, 0.0f);
  return new CompressedMapUV(&m);
}

// The export functions of Src/image.cpp:188-405, writing `path` (the
// extension picks the format); dilation runs on one OpenMP thread, in row
// order.
int ref_export_float(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx, const float* data,
                     const char* path, float flo, float fhi, int normalize, int dilate, float* minmax) {
  CompressedMapUV* c = make_cmap(w, h, count, idx);
  if (c->indices.size() != count) { delete c; return -1; }
  const int threads = omp_get_max_threads();
  omp_set_num_threads(1);
  Vector2 mm;
  exportFloatImage(data, c, path, Vector2(flo, fhi), normalize != 0, dilate, &mm);
  omp_set_num_threads(threads);
  minmax[0] = mm.x;
  minmax[1] = mm.y;
  delete c;
  return 0;
}

int ref_export_normal(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx, const float* data3,
                      const char* path, int dilate) {
  CompressedMapUV* c = make_cmap(w, h, count, idx);
  if (c->indices.size() != count) { delete c; return -1; }
  std::vector<Vector3> v(count);
  for (uint32_t i = 0; i < count; ++i) v[i] = Vector3(data3[3 * i], data3[3 * i + 1], data3[3 * i + 2]);
  const int threads = omp_get_max_threads();
  omp_set_num_threads(1);
  ref_exportNormalImage(v.data(), c, path, dilate);
  omp_set_num_threads(threads);
  delete c;
  return 0;
}

int ref_export_vector(uint32_t w, uint32_t h, uint32_t count, const uint32_t* idx, const float* data3,
                      const char* path) {
  CompressedMapUV* c = make_cmap(w, h, count, idx);
  if (c->indices.size() != count) { delete c; return -1; }
  std::vector<Vector3> v(count);
  for (uint32_t i = 0; i < count; ++i) v[i] = Vector3(data3[3 * i], data3[3 * i + 1], data3[3 * i + 2]);
  exportVectorImage(v.data(), c, path);
  delete c;
  return 0;
}

// Mesh::loadFile (Src/mesh.cpp:612-617).  ref_mesh_load returns the mesh or
// null; ref_mesh_sizes gives position, texcoord, normal, vertex and triangle
// counts; ref_mesh_arrays copies the arrays out (positions / normals 3
// floats, texcoords 2, vertices and triangles 3 u32 each).
void* ref_mesh_load(const char* path) { return Mesh::loadFile(path); }

void ref_mesh_sizes(const void* h, uint64_t* n) {
  const Mesh* m = static_cast<const Mesh*>(h);
  n[0] = m->positions.size();
  n[1] = m->texcoords.size();
  n[2] = m->normals.size();
  n[3] = m->vertices.size();
  n[4] = m->triangles.size();
}

void ref_mesh_arrays(const void* h, float* pos, float* uv, float* nrm, uint32_t* vtx, uint32_t* tri) {
  const Mesh* m = static_cast<const Mesh*>(h);
  for (size_t i = 0; i < m->positions.size(); ++i) {
    pos[3 * i] = m->positions[i].x; pos[3 * i + 1] = m->positions[i].y; pos[3 * i + 2] = m->positions[i].z;
  }
  for (size_t i = 0; i < m->texcoords.size(); ++i) { uv[2 * i] = m->texcoords[i].x; uv[2 * i + 1] = m->texcoords[i].y; }
  for (size_t i = 0; i < m->normals.size(); ++i) {
    nrm[3 * i] = m->normals[i].x; nrm[3 * i + 1] = m->normals[i].y; nrm[3 * i + 2] = m->normals[i].z;
  }
  for (size_t i = 0; i < m->vertices.size(); ++i) {
    vtx[3 * i] = m->vertices[i].positionIndex;
    vtx[3 * i + 1] = m->vertices[i].texcoordIndex;
    vtx[3 * i + 2] = m->vertices[i].normalIndex;
  }
  for (size_t i = 0; i < m->triangles.size(); ++i) {
    tri[3 * i] = m->triangles[i].vertexIndex0;
    tri[3 * i + 1] = m->triangles[i].vertexIndex1;
    tri[3 * i + 2] = m->triangles[i].vertexIndex2;
  }
}

void ref_mesh_free(void* h) { delete static_cast<Mesh*>(h); }

}  // extern "C"
