// fk_bake: the runner of Src/fornos.cpp:53-251 from host arrays, in one call.
// Scene and texel rows go up, mesh mapping and the enabled solvers run on the
// context's stream, results come back.  Built only from the public entry
// points of include/fornos_gpu.h.
#include <cfloat>
#include <cstring>
#include <vector>

#include "fk_internal.h"

namespace {

struct Scoped {
  fk_ctx* ctx;
  std::vector<fk_buf*> bufs;
  fk_scene* scene = nullptr;
  fk_texel_map* map = nullptr;
  ~Scoped() {
    // result copies on the copy stream read these buffers: they finish first
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    for (fk_buf* b : bufs) fk_buf_release(ctx, b);  // used on the context's stream only
    if (scene) fk_scene_free(ctx, scene);
    if (map) fk_texel_map_free(ctx, map);
  }
  int alloc(size_t bytes, fk_buf** out) {
    int rc = fk_buf_alloc(ctx, bytes ? bytes : 16, out);
    if (rc == FK_OK) bufs.push_back(*out);
    return rc;
  }
};

bool same_params(const fk_bake_sampler& a, const fk_bake_sampler& b) {
  return a.sample_count == b.sample_count && a.min_distance == b.min_distance && a.max_distance == b.max_distance &&
         a.seed == b.seed;
}

// Copies a finished result to the host on the copy stream, once the work
// queued so far on the context's stream is done, so that the copy overlaps
// the passes queued after it.
int download(fk_ctx* ctx, const fk_buf* b, void* dst, size_t bytes) {
  if (!dst || !bytes) return FK_OK;
  cudaEvent_t ev;
  FK_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, ev, 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst, b->ptr, bytes, cudaMemcpyDeviceToHost, ctx->copy_stream);
  cudaEventDestroy(ev);
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "fk_bake: result copy");
  return FK_OK;
}

}  // namespace

extern "C" int fk_bake(fk_ctx* ctx, const fk_bake_desc* d, fk_bake_out* out) {
  if (!ctx || !d || !out) return fk_fail(ctx, FK_ERR_INVALID, "fk_bake: null argument");
  const uint32_t perms = 4096;
  if (!ctx->copy_stream && cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    ctx->copy_stream = nullptr;
    return fk_fail(ctx, FK_ERR_CUDA, "fk_bake: copy stream");
  }
  Scoped s{ctx};
  // the texel rows go up while the host checks and lays out the scene (the
  // scene upload waits for the stream before it returns)
  int rc = fk::texel_map_upload_async(ctx, d->width, d->height, d->texel_count, d->pix8, d->pixt12, d->indices,
                                      &s.map);
  if (rc != FK_OK) return rc;
  rc = fk_scene_upload(ctx, d->nodes, d->node_count, d->positions4, d->normals4, d->corner_count, &s.scene);
  if (rc != FK_OK) return rc;
  const uint32_t n = d->texel_count;
  const size_t nn = n ? n : 1;
  fk_buf *coords, *tidx;
  if ((rc = s.alloc(16 * nn, &coords)) != FK_OK || (rc = s.alloc(4 * nn, &tidx)) != FK_OK) return rc;
  if ((rc = fk_meshmap(ctx, s.scene, s.map, d->cull_backfaces,
                       d->mapping_max_distance > 0.0f ? d->mapping_max_distance : FLT_MAX, 0, n, coords, tidx)) != FK_OK) return rc;
  if ((rc = download(ctx, coords, out->coords4, 16 * (size_t)n)) != FK_OK) return rc;
  if ((rc = download(ctx, tidx, out->tidx, 4 * (size_t)n)) != FK_OK) return rc;

  auto gather = [&](int enabled, int kind, float* host, size_t width, int tangent) -> int {
    if (!enabled) return FK_OK;
    fk_buf* o;
    int r = s.alloc(4 * width * nn, &o);
    if (r == FK_OK) r = fk_gather(ctx, s.scene, kind, coords, tidx, 0, n, o);
    if (r == FK_OK && tangent) r = fk_tangent_space(ctx, s.map, 0, n, o);
    if (r == FK_OK) r = download(ctx, o, host, 4 * width * n);
    return r;
  };
  if ((rc = gather(d->height_enabled, FK_GATHER_HEIGHT, out->height, 1, 0)) != FK_OK) return rc;
  if ((rc = gather(d->position_enabled, FK_GATHER_POSITION, out->position3, 3, 0)) != FK_OK) return rc;
  if ((rc = gather(d->normals_enabled, FK_GATHER_NORMAL, out->normals3, 3, d->normals_tangent_space)) != FK_OK) return rc;

  // Sample tables, one per distinct (spp, seed), generated on the host as the
  // solvers' init does (Src/solver_ao.cpp:36-68).
  std::vector<std::pair<std::pair<uint32_t, uint32_t>, fk_buf*>> tables;
  auto table = [&](const fk_bake_sampler& p, fk_buf** tb) -> int {
    for (auto& t : tables)
      if (t.first.first == p.sample_count && t.first.second == p.seed) { *tb = t.second; return FK_OK; }
    std::vector<float> host(4 * (size_t)p.sample_count * perms);
    int r = fk_samples_cosine(p.sample_count, perms, p.seed, host.data());
    if (r == FK_OK) r = s.alloc(4 * host.size(), tb);
    if (r == FK_OK) r = fk_buf_upload(ctx, *tb, 0, host.data(), 4 * host.size());
    if (r == FK_OK) tables.push_back({{p.sample_count, p.seed}, *tb});
    return r;
  };
  const fk_bake_sampler& ao = d->ao;
  const fk_bake_sampler& bn = d->bent_normals;
  const fk_bake_sampler& th = d->thickness;
  bool fuse = ao.enabled && bn.enabled && same_params(ao, bn);
  fk_buf *ao_out = nullptr, *bn_out = nullptr;
  if (ao.enabled || bn.enabled) {
    if (ao.enabled && (rc = s.alloc(4 * nn, &ao_out)) != FK_OK) return rc;
    if (bn.enabled && (rc = s.alloc(12 * nn, &bn_out)) != FK_OK) return rc;
    if (fuse) {
      fk_buf* tb;
      if ((rc = table(ao, &tb)) != FK_OK) return rc;
      fk_sample_params sp{ao.sample_count, perms, ao.min_distance, ao.max_distance};
      rc = fk_hemisphere(ctx, s.scene, coords, tidx, FK_AO_BN, &sp, tb, 0, n, d->traverse, ao_out, bn_out, nullptr, nullptr);
      if (rc != FK_OK) return rc;
    } else {
      if (ao.enabled) {
        fk_buf* tb;
        if ((rc = table(ao, &tb)) != FK_OK) return rc;
        fk_sample_params sp{ao.sample_count, perms, ao.min_distance, ao.max_distance};
        if ((rc = fk_hemisphere(ctx, s.scene, coords, tidx, FK_AO, &sp, tb, 0, n, d->traverse, ao_out, nullptr, nullptr,
                                nullptr)) != FK_OK)
          return rc;
      }
      if (bn.enabled) {
        fk_buf* tb;
        if ((rc = table(bn, &tb)) != FK_OK) return rc;
        fk_sample_params sp{bn.sample_count, perms, bn.min_distance, bn.max_distance};
        if ((rc = fk_hemisphere(ctx, s.scene, coords, tidx, FK_BN, &sp, tb, 0, n, d->traverse, bn_out, nullptr, nullptr,
                                nullptr)) != FK_OK)
          return rc;
      }
    }
    if (bn.enabled && bn.tangent_space && (rc = fk_tangent_space(ctx, s.map, 0, n, bn_out)) != FK_OK) return rc;
    if (ao.enabled && (rc = download(ctx, ao_out, out->ao, 4 * (size_t)n)) != FK_OK) return rc;
    if (bn.enabled && (rc = download(ctx, bn_out, out->bent_normals3, 12 * (size_t)n)) != FK_OK) return rc;
  }
  if (th.enabled) {
    fk_buf *tb, *th_out;
    if ((rc = table(th, &tb)) != FK_OK || (rc = s.alloc(4 * nn, &th_out)) != FK_OK) return rc;
    fk_sample_params sp{th.sample_count, perms, th.min_distance, th.max_distance};
    if ((rc = fk_hemisphere(ctx, s.scene, coords, tidx, FK_THICK, &sp, tb, 0, n, d->traverse, th_out, nullptr, nullptr,
                            nullptr)) != FK_OK)
      return rc;
    if ((rc = download(ctx, th_out, out->thickness, 4 * (size_t)n)) != FK_OK) return rc;
  }
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->copy_stream));
  int st = 0;
  FK_CUDA(ctx, cudaMemcpy(&st, ctx->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemset(ctx->status, 0, sizeof(int));
    return fk_fail(ctx, FK_ERR_DEVICE, "fk_bake: a traversal exceeded its stack");
  }
  return FK_OK;
}
