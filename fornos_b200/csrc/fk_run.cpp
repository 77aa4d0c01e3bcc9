// fk_run: FornosRunner::start followed by FornosRunner::run until every task
// has finished (Src/fornos.cpp:53-251), from mesh files to image files.  The
// steps are the reference's, each through this library's entry points:
//   * Mesh::loadFile for both meshes (the high-poly one may be the low-poly
//     one), normals per NormalImport, tangent space when the normals or bent
//     normals are wanted in tangent space -- on the device;
//   * the texel map of the mapping method (Smooth and Hybrid take a copy of
//     the low-poly mesh with welded normals unless its normals were computed
//     per vertex) -- fk_raster_uv;
//   * BVH::createBinary of the high-poly mesh with bvhTrisPerNode and depth
//     8192, flattened and resident -- fk_scene_build;
//   * mesh mapping, then every enabled solver, each result exported with the
//     arguments its task's finish() passes (Src/solver_*.cpp) and written by
//     the output path's extension (.png / .tga / .exr; any other extension
//     writes nothing, as in the reference).
// Sample tables come from `seed` (the reference draws them from
// std::random_device); AO and bent normals with equal sample parameters
// share one traversal.
#include <cfloat>
#include <cstring>
#include <future>
#include <memory>
#include <string>
#include <system_error>
#include <vector>

#include "fk_internal.h"

namespace {

struct Owned {
  fk_ctx* ctx;
  std::vector<fk_mesh*> meshes;
  std::vector<fk_buf*> bufs;
  fk_scene* scene = nullptr;
  fk_texel_map* map = nullptr;
  ~Owned() {
    for (fk_buf* b : bufs) fk_buf_release(ctx, b);
    if (scene) fk_scene_free(ctx, scene);
    if (map) fk_texel_map_free(ctx, map);
    for (fk_mesh* m : meshes) fk_mesh_free(m);
  }
  fk_mesh* keep(fk_mesh* m) {
    meshes.push_back(m);
    return m;
  }
  int alloc(size_t bytes, fk_buf** out) {
    int rc = fk_buf_alloc(ctx, bytes ? bytes : 16, out);
    if (rc == FK_OK) bufs.push_back(*out);
    return rc;
  }
};

enum Format { kNone, kRgb8, kExr };

Format format_of(const char* path) {
  if (!path) return kNone;
  const size_t n = std::strlen(path);
  auto ends = [&](const char* t) { return n >= 4 && std::strcmp(path + n - 4, t) == 0; };
  if (ends(".png") || ends(".tga")) return kRgb8;
  if (ends(".exr")) return kExr;
  return kNone;
}

// NormalImport (Src/fornos.h:35).
int import_normals(fk_ctx* ctx, fk_mesh* m, int how) {
  if (how == FK_NORMAL_COMPUTE_PER_FACE) return fk_mesh_compute_normals_device(ctx, m, FK_NORMALS_FACE);
  if (how == FK_NORMAL_COMPUTE_PER_VERTEX) return fk_mesh_compute_normals_device(ctx, m, FK_NORMALS_VERTEX);
  return FK_OK;
}

}  // namespace

extern "C" {

void fk_run_params_default(fk_run_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->lo_poly_mesh_normal = FK_NORMAL_IMPORT;
  p->hi_poly_mesh_normal = FK_NORMAL_IMPORT;
  p->bvh_tris_per_node = 8;
  p->tex_width = 2048;
  p->tex_height = 2048;
  p->tex_dilation = 16;
  p->ignore_backfaces = 1;
  p->mapping = FK_MAP_SMOOTH;
  p->mapping_edge = 0.05f;
  p->height.normalize_output = 1;
  p->normals.tangent_space = 1;
  p->bent_normals.tangent_space = 1;
  fk_run_solver* s[3] = {&p->ao, &p->bent_normals, &p->thickness};
  for (fk_run_solver* q : s) {
    q->sample_count = 256;
    q->min_distance = 0.01f;
    q->max_distance = 10.0f;
  }
  p->traverse = FK_TRAVERSE_AUTO;
}

int fk_run(fk_ctx* ctx, const fk_run_params* p) {
  if (!ctx || !p) return fk_fail(ctx, FK_ERR_INVALID, "fk_run: null argument");
  if (p->mapping < FK_MAP_SMOOTH || p->mapping > FK_MAP_HYBRID || p->bvh_tris_per_node == 0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_run: bad parameters");
  Owned o{ctx};
  int rc;
  fk_mesh* lo = nullptr;
  if (!p->lo_poly_mesh_path || fk_mesh_load(p->lo_poly_mesh_path, &lo) != FK_OK)
    return fk_fail(ctx, FK_ERR_INVALID, "Missing low poly mesh");
  o.keep(lo);
  if ((rc = import_normals(ctx, lo, p->lo_poly_mesh_normal)) != FK_OK) return rc;
  fk_mesh* hi = lo;
  if (p->hi_poly_mesh_path && p->hi_poly_mesh_path[0]) {
    if (fk_mesh_load(p->hi_poly_mesh_path, &hi) != FK_OK) return fk_fail(ctx, FK_ERR_INVALID, "Missing high poly mesh");
    o.keep(hi);
    if ((rc = import_normals(ctx, hi, p->hi_poly_mesh_normal)) != FK_OK) return rc;
  }
  const bool tangents = (p->normals.enabled && p->normals.tangent_space) ||
                        (p->bent_normals.enabled && p->bent_normals.tangent_space);
  if (tangents && (rc = fk_mesh_compute_tangent_space_device(ctx, lo)) != FK_OK) return rc;

  // texel map of the mapping method
  const fk_mesh* dirs = nullptr;
  if (p->mapping != FK_MAP_LOWPOLY_NORMALS) {
    if (p->lo_poly_mesh_normal != FK_NORMAL_COMPUTE_PER_VERTEX) {
      fk_mesh* copy = nullptr;
      if ((rc = fk_mesh_copy(lo, &copy)) != FK_OK) return fk_fail(ctx, rc, "fk_run: mesh copy");
      o.keep(copy);
      if ((rc = fk_mesh_compute_normals_device(ctx, copy, FK_NORMALS_WELDED)) != FK_OK) return rc;
      dirs = copy;
    } else {
      dirs = lo;
    }
  }
  if (fk_raster_uv(ctx, lo, dirs, p->tex_width, p->tex_height, p->mapping, p->mapping_edge, &o.map) != FK_OK)
    return fk_fail(ctx, FK_ERR_INVALID, "Low poly mesh is missing texture coordinates or normals information");
  if ((rc = fk_scene_build(ctx, hi, p->bvh_tris_per_node, 8192, &o.scene)) != FK_OK) return rc;

  uint32_t w = 0, h = 0, n = 0;
  fk_texel_map_info(o.map, &w, &h, &n);
  const size_t nn = n ? n : 1;
  fk_buf *coords, *tidx;
  if ((rc = o.alloc(16 * nn, &coords)) != FK_OK || (rc = o.alloc(4 * nn, &tidx)) != FK_OK) return rc;
  if ((rc = fk_meshmap(ctx, o.scene, o.map, p->ignore_backfaces, FLT_MAX, 0, n, coords, tidx)) != FK_OK) return rc;

  // exports: one device image buffer, reused; each downloaded image is encoded
  // and written on a thread of its own while the device runs the next
  // solvers (the futures are waited for before any return)
  fk_buf* image = nullptr;
  if ((rc = o.alloc(12 * (size_t)w * h, &image)) != FK_OK) return rc;
  std::vector<std::pair<std::string, std::future<int>>> writes;
  auto export_map = [&](const fk_buf* data, const char* path, bool vec3, bool vector_only, float lo_f, float hi_f,
                        int normalize, int dilate) -> int {
    const Format f = format_of(path);
    if (f == kNone || (vector_only && f != kExr)) return FK_OK;  // the reference writes nothing
    fk_export_params ep{};
    ep.filter_lo = lo_f;
    ep.filter_hi = hi_f;
    ep.normalize = normalize;
    ep.dilate = f == kRgb8 ? dilate : 0;  // the EXR branches of the exporters do not dilate
    if (vec3) ep.mode = f == kExr ? FK_EXPORT_VECTOR_F32 : FK_EXPORT_NORMAL_RGB8;
    else ep.mode = f == kExr ? FK_EXPORT_FLOAT_F32 : FK_EXPORT_FLOAT_RGB8;
    float minmax[2];
    int r = fk_export_image(ctx, o.map, data, &ep, image, minmax);
    const size_t bytes = f == kRgb8 ? 3 * (size_t)w * h : (vec3 ? 12 : 4) * (size_t)w * h;
    std::vector<float> host((bytes + 3) / 4);
    if (r == FK_OK) r = fk_buf_download(ctx, image, 0, host.data(), bytes);
    if (r != FK_OK) return r;
    const uint32_t planes = vec3 ? 3 : 1;
    std::string file(path);
    auto pixels = std::make_shared<std::vector<float>>(std::move(host));
    auto job = [pixels, file, f, w, h, planes]() {
      return f == kRgb8 ? fk_image_write_rgb8(file.c_str(), w, h, reinterpret_cast<const uint8_t*>(pixels->data()))
                        : fk_image_write_exr(file.c_str(), w, h, planes, pixels->data());
    };
    std::future<int> done;
    try {
      done = std::async(std::launch::async, job);
    } catch (const std::system_error&) {  // no thread to be had: written here
      std::promise<int> now;
      now.set_value(job());
      done = now.get_future();
    }
    writes.emplace_back(file, std::move(done));
    return FK_OK;
  };
  auto gather = [&](int kind, size_t width, int tangent, fk_buf** out) -> int {
    int r = o.alloc(4 * width * nn, out);
    if (r == FK_OK) r = fk_gather(ctx, o.scene, kind, coords, tidx, 0, n, *out);
    if (r == FK_OK && tangent) r = fk_tangent_space(ctx, o.map, 0, n, *out);
    return r;
  };
  std::vector<std::pair<uint32_t, fk_buf*>> tables;
  auto table = [&](uint32_t spp, fk_buf** tb) -> int {
    for (auto& t : tables)
      if (t.first == spp) {
        *tb = t.second;
        return FK_OK;
      }
    std::vector<float> samples(4 * (size_t)spp * 4096);
    int r = fk_samples_cosine(spp, 4096, p->seed, samples.data());
    if (r == FK_OK) r = o.alloc(4 * samples.size(), tb);
    if (r == FK_OK) r = fk_buf_upload(ctx, *tb, 0, samples.data(), 4 * samples.size());
    if (r == FK_OK) tables.push_back({spp, *tb});
    return r;
  };
  auto sampled = [&](const fk_run_solver& s, int kind, fk_buf* out0, fk_buf* out1) -> int {
    if (s.sample_count == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_run: sample count 0");
    fk_buf* tb;
    int r = table(s.sample_count, &tb);
    fk_sample_params sp{s.sample_count, 4096, s.min_distance, s.max_distance};
    if (r == FK_OK) r = fk_hemisphere(ctx, o.scene, coords, tidx, kind, &sp, tb, 0, n, p->traverse, out0, out1, nullptr,
                                      nullptr);
    return r;
  };

  // the tasks in the order run() takes them (the reverse of start()'s pushes)
  fk_buf* b;
  if (p->height.enabled) {  // HeightTask::finish, Src/solver_height.cpp:103-118
    if ((rc = gather(FK_GATHER_HEIGHT, 1, 0, &b)) != FK_OK ||
        (rc = export_map(b, p->height.output_path, false, false, 0.0f, p->height.max_distance,
                         p->height.normalize_output, p->tex_dilation)) != FK_OK)
      return rc;
  }
  if (p->positions.enabled) {  // PositionTask::finish, Src/solver_position.cpp:104-111 (EXR only)
    if ((rc = gather(FK_GATHER_POSITION, 3, 0, &b)) != FK_OK ||
        (rc = export_map(b, p->positions.output_path, true, true, 0.0f, 0.0f, 0, 0)) != FK_OK)
      return rc;
  }
  if (p->normals.enabled) {  // NormalsTask::finish, Src/solver_normals.cpp:116-123
    if ((rc = gather(FK_GATHER_NORMAL, 3, p->normals.tangent_space, &b)) != FK_OK ||
        (rc = export_map(b, p->normals.output_path, true, false, 0.0f, 0.0f, 0, p->tex_dilation)) != FK_OK)
      return rc;
  }
  const fk_run_solver &ao = p->ao, &bn = p->bent_normals, &th = p->thickness;
  const bool fuse = ao.enabled && bn.enabled && ao.sample_count == bn.sample_count &&
                    ao.min_distance == bn.min_distance && ao.max_distance == bn.max_distance;
  fk_buf *ao_out = nullptr, *bn_out = nullptr;
  if (ao.enabled && (rc = o.alloc(4 * nn, &ao_out)) != FK_OK) return rc;
  if (bn.enabled && (rc = o.alloc(12 * nn, &bn_out)) != FK_OK) return rc;
  if (fuse) {
    if ((rc = sampled(ao, FK_AO_BN, ao_out, bn_out)) != FK_OK) return rc;
  } else {
    if (ao.enabled && (rc = sampled(ao, FK_AO, ao_out, nullptr)) != FK_OK) return rc;
    if (bn.enabled && (rc = sampled(bn, FK_BN, bn_out, nullptr)) != FK_OK) return rc;
  }
  if (ao.enabled &&  // AmbientOcclusionTask::finish, Src/solver_ao.cpp:157-163
      (rc = export_map(ao_out, ao.output_path, false, false, 0.0f, 0.0f, 1, p->tex_dilation)) != FK_OK)
    return rc;
  if (bn.enabled) {  // BentNormalsTask::finish, Src/solver_bentnormals.cpp:168-174
    if (bn.tangent_space && (rc = fk_tangent_space(ctx, o.map, 0, n, bn_out)) != FK_OK) return rc;
    if ((rc = export_map(bn_out, bn.output_path, true, false, 0.0f, 0.0f, 0, p->tex_dilation)) != FK_OK) return rc;
  }
  if (th.enabled) {  // ThicknessTask::finish, Src/solver_thickness.cpp:157-164
    fk_buf* th_out;
    if ((rc = o.alloc(4 * nn, &th_out)) != FK_OK || (rc = sampled(th, FK_THICK, th_out, nullptr)) != FK_OK ||
        (rc = export_map(th_out, th.output_path, false, false, 0.0f, 0.0f, 1, p->tex_dilation)) != FK_OK)
      return rc;
  }
  rc = FK_OK;
  for (auto& wr : writes)
    if (wr.second.get() != FK_OK) rc = fk_fail(ctx, FK_ERR_INVALID, "fk_run: cannot write " + wr.first);
  if (rc != FK_OK) return rc;
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  int st = 0;
  FK_CUDA(ctx, cudaMemcpy(&st, ctx->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemset(ctx->status, 0, sizeof(int));
    return fk_fail(ctx, FK_ERR_DEVICE, "fk_run: a traversal exceeded its stack");
  }
  return FK_OK;
}

}  // extern "C"
