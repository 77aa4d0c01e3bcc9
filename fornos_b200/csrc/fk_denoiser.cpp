// Learned denoiser: the C ABI (fk_denoiser_*, fk_denoise_*) over the kernels
// of fk_denoise.cu, and the verified denoised bake.  No counterpart in the
// reference; the plain AO / bent-normal bake it shortcuts is
// Src/solver_ao.cpp + Src/solver_bentnormals.cpp (Shaders/ao_step1.comp,
// Shaders/bentnormals_step1.comp), here fk_hemisphere with FK_AO_BN.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fk_internal.h"

using fk::DnWeights;
namespace dn = fk::dn;

struct fk_denoiser {
  fk_ctx* ctx = nullptr;
  float* params = nullptr;  // fp32 master weights
  float* m = nullptr;       // Adam moments
  float* v = nullptr;
  void *w1 = nullptr, *w2 = nullptr, *w2t = nullptr, *w3 = nullptr, *w3t = nullptr;  // bf16 copies
  float* grad = nullptr;    // reduced gradient (fk_denoiser_gradient)
  float* partials = nullptr;
  float* loss = nullptr;    // per-tile squared-error sums of the last step
  uint32_t tile_capacity = 0, last_tiles = 0, last_batch = 0;
  uint32_t step = 0;
  int engine = FK_DN_ENGINE_TCGEN05;  // inference kernel
  // denoised-bake scratch
  void* scratch[6] = {};
  size_t scratch_bytes[6] = {};
};

namespace {

bool fits(const fk_buf* b, uint64_t bytes) { return b && b->bytes >= bytes; }

DnWeights weights(const fk_denoiser* d) { return DnWeights{d->params, d->w1, d->w2, d->w2t, d->w3, d->w3t}; }

int launched(fk_ctx* ctx, cudaError_t e, const char* what, int kernels = 1) {
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, what);
  ctx->launches += kernels;
  return FK_OK;
}

// Inference through the denoiser's engine (the two kernels compute the same
// network; see fk_denoiser_set_engine).
cudaError_t apply(const fk_denoiser* d, const float4* image, uint32_t w, uint32_t h, const uint32_t* indices,
                  const uint32_t* tidx, const float* ao_in, const float* bn_in, uint32_t offset, uint32_t count,
                  float* ao_out, float* bn_out, const uint32_t* rows, float4* y_out) {
  fk_ctx* ctx = d->ctx;
  if (d->engine == FK_DN_ENGINE_TCGEN05)
    return dn::launch_apply_tc(ctx->stream, ctx->sm_count, image, w, h, indices, tidx, ao_in, bn_in, offset, count,
                               weights(d), ao_out, bn_out, rows, y_out, ctx->status);
  return dn::launch_apply(ctx->stream, ctx->sm_count, image, w, h, indices, tidx, ao_in, bn_in, offset, count,
                          weights(d), ao_out, bn_out, rows, y_out);
}

int ensure_tiles(fk_denoiser* d, uint32_t tiles) {
  if (tiles <= d->tile_capacity) return FK_OK;
  fk_dev_free(d->ctx, d->partials);
  fk_dev_free(d->ctx, d->loss);
  d->partials = nullptr;
  d->loss = nullptr;
  d->tile_capacity = 0;
  int rc = fk_dev_alloc(d->ctx, (void**)&d->partials, (size_t)tiles * dn::kParams * sizeof(float));
  if (rc == FK_OK) rc = fk_dev_alloc(d->ctx, (void**)&d->loss, (size_t)tiles * sizeof(float));
  if (rc == FK_OK) d->tile_capacity = tiles;
  return rc;
}

// Denoised-bake scratch slot k of at least `bytes` (kept between calls).
void* scratch(fk_denoiser* d, int k, size_t bytes) {
  if (d->scratch_bytes[k] >= bytes) return d->scratch[k];
  if (cudaStreamSynchronize(d->ctx->stream) != cudaSuccess) return nullptr;
  fk_dev_free(d->ctx, d->scratch[k]);
  d->scratch[k] = nullptr;
  d->scratch_bytes[k] = 0;
  if (fk_dev_alloc(d->ctx, &d->scratch[k], std::max<size_t>(bytes, 16)) != FK_OK) return nullptr;
  d->scratch_bytes[k] = bytes;
  return d->scratch[k];
}

int check_batch(fk_denoiser* d, const fk_buf* rows, const fk_buf* targets, uint32_t n_rows, const fk_buf* row_ids,
                uint32_t offset, uint32_t batch, const char* who) {
  fk_ctx* ctx = d->ctx;
  if (!rows || !targets) return fk_fail(ctx, FK_ERR_INVALID, std::string(who) + ": null argument");
  if (batch == 0 || batch % dn::kRows)
    return fk_fail(ctx, FK_ERR_INVALID, std::string(who) + ": batch must be a positive multiple of 128");
  if (!fits(rows, (uint64_t)n_rows * FK_DN_ROW_BYTES) || !fits(targets, (uint64_t)n_rows * 16))
    return fk_fail(ctx, FK_ERR_INVALID, std::string(who) + ": rows / targets smaller than n_rows");
  if (row_ids ? !fits(row_ids, 4 * ((uint64_t)offset + batch)) : (uint64_t)offset + batch > n_rows)
    return fk_fail(ctx, FK_ERR_INVALID, std::string(who) + ": batch outside the row list");
  return ensure_tiles(d, batch / dn::kRows);
}

int run_train(fk_denoiser* d, const fk_buf* rows, const fk_buf* targets, uint32_t n_rows, const fk_buf* row_ids,
              uint32_t offset, uint32_t batch, int update, const fk_adam* adam) {
  fk_ctx* ctx = d->ctx;
  const uint32_t tiles = batch / dn::kRows;
  int rc = launched(ctx,
                    dn::launch_train(ctx->stream, (const uint32_t*)rows->ptr, (const float4*)targets->ptr,
                                     row_ids ? (const uint32_t*)row_ids->ptr : nullptr, n_rows, offset, batch,
                                     weights(d), d->partials, d->loss, ctx->status),
                    "dn_train_kernel");
  if (rc != FK_OK) return rc;
  float lr = 0, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f, c1 = 1, c2 = 1;
  if (update) {
    lr = adam->learning_rate;
    b1 = adam->beta1;
    b2 = adam->beta2;
    eps = adam->eps;
    const double t = (double)(d->step + 1);
    c1 = (float)(1.0 / (1.0 - std::pow((double)b1, t)));
    c2 = (float)(1.0 / (1.0 - std::pow((double)b2, t)));
  }
  rc = launched(ctx,
                dn::launch_adam(ctx->stream, d->partials, tiles, d->params, d->m, d->v, update ? nullptr : d->grad,
                                update, lr, b1, b2, eps, c1, c2, weights(d)),
                "dn_adam_kernel");
  if (rc != FK_OK) return rc;
  if (update) ++d->step;
  d->last_tiles = tiles;
  d->last_batch = batch;
  return FK_OK;
}

int read_loss(fk_denoiser* d, double* loss) {
  fk_ctx* ctx = d->ctx;
  if (!d->last_tiles) return fk_fail(ctx, FK_ERR_STATE, "fk_denoiser_last_loss: no step has run");
  std::vector<float> l(d->last_tiles);
  FK_CUDA(ctx, cudaMemcpyAsync(l.data(), d->loss, l.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double s = 0;
  for (float x : l) s += x;
  *loss = s / (4.0 * d->last_batch);
  return FK_OK;
}

}  // namespace

extern "C" {

int fk_denoiser_create(fk_ctx* ctx, fk_denoiser** out) {
  if (!ctx || !out) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoiser_create: null argument");
  static_assert(dn::kParams == FK_DN_PARAMS, "parameter count");
  auto* d = new fk_denoiser();
  d->ctx = ctx;
  const size_t pb = (size_t)dn::kParams * sizeof(float);
  int rc = fk_dev_alloc(ctx, (void**)&d->params, pb);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&d->m, pb);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&d->v, pb);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&d->grad, pb);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, &d->w1, (size_t)dn::kHidden * dn::kK1 * 2);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, &d->w2, (size_t)dn::kHidden * dn::kHidden * 2);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, &d->w2t, (size_t)dn::kHidden * dn::kHidden * 2);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, &d->w3, (size_t)8 * dn::kHidden * 2);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, &d->w3t, (size_t)8 * dn::kHidden * 2);
  if (rc == FK_OK) {
    for (void* p : {(void*)d->params, (void*)d->m, (void*)d->v})
      if (cudaMemsetAsync(p, 0, pb, ctx->stream) != cudaSuccess) rc = fk_fail(ctx, FK_ERR_CUDA, "memset");
  }
  if (rc == FK_OK) rc = launched(ctx, dn::launch_refresh(ctx->stream, weights(d)), "dn_refresh_kernel");
  if (rc != FK_OK) {
    fk_denoiser_free(d);
    return rc;
  }
  *out = d;
  return FK_OK;
}

int fk_denoiser_free(fk_denoiser* d) {
  if (!d) return FK_ERR_INVALID;
  if (d->ctx) cudaStreamSynchronize(d->ctx->stream);
  for (void* p : {(void*)d->params, (void*)d->m, (void*)d->v, (void*)d->grad, d->w1, d->w2, d->w2t, d->w3, d->w3t,
                  (void*)d->partials, (void*)d->loss})
    fk_dev_free(d->ctx, p);
  for (void* p : d->scratch) fk_dev_free(d->ctx, p);
  delete d;
  return FK_OK;
}

int fk_denoiser_set_params(fk_denoiser* d, const float* params, uint32_t count) {
  if (!d || !params) return FK_ERR_INVALID;
  fk_ctx* ctx = d->ctx;
  if (count != (uint32_t)dn::kParams) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoiser_set_params: count must be FK_DN_PARAMS");
  std::vector<float> h(params, params + count);
  for (int r = 0; r < dn::kHidden; ++r)
    for (int c = dn::kInputs; c < dn::kK1; ++c) h[dn::kW1 + r * dn::kK1 + c] = 0.0f;
  const size_t pb = (size_t)dn::kParams * sizeof(float);
  FK_CUDA(ctx, cudaMemcpyAsync(d->params, h.data(), pb, cudaMemcpyHostToDevice, ctx->stream));
  FK_CUDA(ctx, cudaMemsetAsync(d->m, 0, pb, ctx->stream));
  FK_CUDA(ctx, cudaMemsetAsync(d->v, 0, pb, ctx->stream));
  d->step = 0;
  int rc = launched(ctx, dn::launch_refresh(ctx->stream, weights(d)), "dn_refresh_kernel");
  if (rc != FK_OK) return rc;
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // `h` goes out of scope
  return FK_OK;
}

int fk_denoiser_set_engine(fk_denoiser* d, int engine) {
  if (!d) return FK_ERR_INVALID;
  if (engine != FK_DN_ENGINE_MMA_SYNC && engine != FK_DN_ENGINE_TCGEN05)
    return fk_fail(d->ctx, FK_ERR_INVALID, "fk_denoiser_set_engine: unknown engine");
  d->engine = engine;
  return FK_OK;
}

int fk_denoiser_get_params(fk_denoiser* d, float* params, uint32_t count) {
  if (!d || !params) return FK_ERR_INVALID;
  fk_ctx* ctx = d->ctx;
  if (count != (uint32_t)dn::kParams) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoiser_get_params: count must be FK_DN_PARAMS");
  FK_CUDA(ctx, cudaMemcpyAsync(params, d->params, (size_t)count * 4, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return FK_OK;
}

int fk_denoise_features(fk_ctx* ctx, const fk_texel_map* map, const fk_buf* coords, const fk_buf* tidx,
                        const fk_buf* ao, const fk_buf* bn3, const fk_buf* pos3, const fk_buf* nrm3,
                        float max_distance, fk_buf* image) {
  if (!ctx || !map || !coords || !tidx || !ao || !bn3 || !pos3 || !nrm3 || !image)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_features: null argument");
  const uint64_t n = map->count, px = (uint64_t)map->width * map->height;
  if (!(max_distance > 0.0f)) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_features: max_distance must be > 0");
  if (!fits(coords, 16 * n) || !fits(tidx, 4 * n) || !fits(ao, 4 * n) || !fits(bn3, 12 * n) || !fits(pos3, 12 * n) ||
      !fits(nrm3, 12 * n))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_features: per-texel buffers smaller than the map");
  if (!fits(image, 48 * px)) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_features: image smaller than 48 x W x H bytes");
  return launched(ctx,
                  dn::launch_features(ctx->stream, map->count, map->width, map->height, map->indices,
                                      (const uint32_t*)tidx->ptr, (const float4*)coords->ptr, (const float*)ao->ptr,
                                      (const float*)bn3->ptr, (const float*)pos3->ptr, (const float*)nrm3->ptr,
                                      max_distance, (float4*)image->ptr),
                  "dn_features_kernel", 2);
}

int fk_denoise_rows(fk_ctx* ctx, const fk_buf* image, uint32_t width, uint32_t height, const fk_buf* pixels,
                    uint32_t count, fk_buf* rows) {
  if (!ctx || !image || !pixels || !rows) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_rows: null argument");
  if (!fits(image, 48ull * width * height) || !fits(pixels, 4ull * count) || !fits(rows, (uint64_t)count * FK_DN_ROW_BYTES))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_rows: buffers too small");
  return launched(ctx,
                  dn::launch_rows(ctx->stream, (const float4*)image->ptr, width, height,
                                  (const uint32_t*)pixels->ptr, count, (uint32_t*)rows->ptr),
                  "dn_rows_kernel");
}

int fk_denoiser_train_step(fk_denoiser* d, const fk_buf* rows, const fk_buf* targets4, uint32_t n_rows,
                           const fk_buf* row_ids, uint32_t offset, uint32_t batch, const fk_adam* adam) {
  if (!d || !adam) return FK_ERR_INVALID;
  if (!(adam->learning_rate >= 0.0f) || !(adam->beta1 >= 0.0f && adam->beta1 < 1.0f) ||
      !(adam->beta2 >= 0.0f && adam->beta2 < 1.0f) || !(adam->eps > 0.0f))
    return fk_fail(d->ctx, FK_ERR_INVALID, "fk_denoiser_train_step: Adam needs lr >= 0, betas in [0, 1), eps > 0");
  int rc = check_batch(d, rows, targets4, n_rows, row_ids, offset, batch, "fk_denoiser_train_step");
  if (rc != FK_OK) return rc;
  return run_train(d, rows, targets4, n_rows, row_ids, offset, batch, 1, adam);
}

int fk_denoiser_last_loss(fk_denoiser* d, double* loss) {
  if (!d || !loss) return FK_ERR_INVALID;
  return read_loss(d, loss);
}

int fk_denoiser_gradient(fk_denoiser* d, const fk_buf* rows, const fk_buf* targets4, uint32_t n_rows,
                         const fk_buf* row_ids, uint32_t offset, uint32_t batch, float* grad, double* loss) {
  if (!d || !grad) return FK_ERR_INVALID;
  int rc = check_batch(d, rows, targets4, n_rows, row_ids, offset, batch, "fk_denoiser_gradient");
  if (rc == FK_OK) rc = run_train(d, rows, targets4, n_rows, row_ids, offset, batch, 0, nullptr);
  if (rc != FK_OK) return rc;
  fk_ctx* ctx = d->ctx;
  FK_CUDA(ctx, cudaMemcpyAsync(grad, d->grad, (size_t)dn::kParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (loss) return read_loss(d, loss);
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return FK_OK;
}

int fk_denoiser_forward(fk_denoiser* d, const fk_buf* rows, uint32_t count, fk_buf* y4) {
  if (!d || !rows || !y4) return FK_ERR_INVALID;
  fk_ctx* ctx = d->ctx;
  if (!fits(rows, (uint64_t)count * FK_DN_ROW_BYTES) || !fits(y4, 16ull * count))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoiser_forward: buffers too small");
  return launched(ctx,
                  apply(d, nullptr, 0, 0, nullptr, nullptr, nullptr, nullptr, 0,
                                   count, nullptr, nullptr, (const uint32_t*)rows->ptr,
                                   (float4*)y4->ptr),
                  "dn_apply_kernel", count ? 1 : 0);
}

int fk_denoise_apply(fk_denoiser* d, const fk_texel_map* map, const fk_buf* image, const fk_buf* tidx,
                     const fk_buf* ao_in, const fk_buf* bn_in, uint32_t offset, uint32_t count, fk_buf* ao_out,
                     fk_buf* bn_out) {
  if (!d || !map || !image || !tidx || !ao_in || !bn_in || !ao_out || !bn_out) return FK_ERR_INVALID;
  fk_ctx* ctx = d->ctx;
  const uint64_t end = (uint64_t)offset + count, n = map->count;
  if (end > n) return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_apply: texel range outside the map");
  if (!fits(image, 48ull * map->width * map->height) || !fits(tidx, 4 * n) || !fits(ao_in, 4 * n) ||
      !fits(bn_in, 12 * n) || !fits(ao_out, 4 * n) || !fits(bn_out, 12 * n))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_apply: buffers smaller than the map");
  return launched(ctx,
                  apply(d, (const float4*)image->ptr, map->width, map->height,
                                   map->indices, (const uint32_t*)tidx->ptr, (const float*)ao_in->ptr,
                                   (const float*)bn_in->ptr, offset, count, (float*)ao_out->ptr,
                                   (float*)bn_out->ptr, nullptr, nullptr),
                  "dn_apply_kernel", count ? 1 : 0);
}

int fk_denoise_bake(fk_denoiser* d, const fk_scene* scene, const fk_texel_map* map, const fk_buf* coords,
                    const fk_buf* tidx, const fk_denoise_params* prm, const fk_buf* samples_low,
                    const fk_buf* samples_full, fk_buf* ao_out, fk_buf* bn_out, fk_denoise_stats* stats) {
  if (!d || !scene || !map || !coords || !tidx || !prm || !samples_low || !samples_full || !ao_out || !bn_out)
    return FK_ERR_INVALID;
  fk_ctx* ctx = d->ctx;
  const uint32_t n = map->count, w = map->width, h = map->height;
  if (prm->low_samples == 0 || prm->full_samples == 0 || prm->perm_count == 0 || prm->tile == 0 ||
      prm->verify_cells == 0 || prm->verify_cells > prm->tile || !(prm->max_distance > 0.0f))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_bake: bad parameters");
  if (!fits(coords, 16ull * n) || !fits(tidx, 4ull * n) || !fits(ao_out, 4ull * n) || !fits(bn_out, 12ull * n))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_bake: per-texel buffers smaller than the map");
  if (!fits(samples_low, 16ull * prm->low_samples * prm->perm_count) ||
      !fits(samples_full, 16ull * prm->full_samples * prm->perm_count))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_denoise_bake: sample tables smaller than samples x perm_count");
  fk_denoise_stats st{};
  if (n == 0) {
    if (stats) *stats = st;
    return FK_OK;
  }
  const uint64_t px = (uint64_t)w * h;
  const uint32_t tiles_x = (w + prm->tile - 1) / prm->tile, tiles_y = (h + prm->tile - 1) / prm->tile;
  const uint32_t tiles = tiles_x * tiles_y, per = prm->verify_cells * prm->verify_cells;
  float* pos3 = (float*)scratch(d, 0, 12ull * n);
  float* nrm3 = (float*)scratch(d, 1, 12ull * n);
  float4* image = (float4*)scratch(d, 2, 48 * px);
  uint32_t* inv = (uint32_t*)scratch(d, 3, 4 * px);
  uint32_t* slots = (uint32_t*)scratch(d, 4, 4ull * tiles * per + 4ull * n + 16);
  float* err = (float*)scratch(d, 5, 4ull * tiles + tiles + 16);
  if (!pos3 || !nrm3 || !image || !inv || !slots || !err)
    return fk_fail(ctx, FK_ERR_NOMEM, "fk_denoise_bake: scratch allocation failed");
  uint32_t* list = slots + (size_t)tiles * per;  // spot-check list, later the fallback list
  uint8_t* failed = (uint8_t*)(err + tiles);
  const float4* c4 = (const float4*)coords->ptr;
  const uint32_t* ti = (const uint32_t*)tidx->ptr;
  float* ao = (float*)ao_out->ptr;
  float* bn = (float*)bn_out->ptr;

  fk::HemiLaunch hl;
  hl.kind = FK_AO_BN;
  hl.perms = prm->perm_count;
  hl.min_d = prm->min_distance;
  hl.max_d = prm->max_distance;
  hl.coords = c4;
  hl.tidx = ti;
  hl.traverse = prm->traverse;
  hl.out0 = ao;
  hl.out1 = bn;
  hl.hits0 = hl.hits1 = nullptr;
  // 1. low-sample bake of every texel
  hl.spp = prm->low_samples;
  hl.samples = (const float4*)samples_low->ptr;
  hl.offset = 0;
  hl.count = n;
  int rc = fk::launch_hemisphere(ctx, scene, hl);
  if (rc != FK_OK) return rc;
  st.rays += (uint64_t)n * prm->low_samples;
  // 2. features and network (in place over the low-sample values)
  rc = fk::launch_gather(ctx, scene, FK_GATHER_POSITION, c4, ti, 0, n, pos3);
  if (rc == FK_OK) rc = fk::launch_gather(ctx, scene, FK_GATHER_NORMAL, c4, ti, 0, n, nrm3);
  if (rc != FK_OK) return rc;
  rc = launched(ctx,
                dn::launch_features(ctx->stream, n, w, h, map->indices, ti, c4, ao, bn, pos3, nrm3,
                                    prm->max_distance, image),
                "dn_features_kernel", 2);
  if (rc == FK_OK)
    rc = launched(ctx,
                  apply(d, image, w, h, map->indices, ti, ao, bn, 0, n,
                                   ao, bn, nullptr, nullptr),
                  "dn_apply_kernel");
  if (rc != FK_OK) return rc;
  // 3. spot checks at full sample count (into the position / normal scratch)
  rc = launched(ctx, dn::launch_inverse(ctx->stream, n, map->indices, (uint32_t)px, inv), "dn_inverse_kernel");
  if (rc == FK_OK)
    rc = launched(ctx, dn::launch_verify_slots(ctx->stream, w, h, prm->tile, prm->verify_cells, inv, ti, slots),
                  "dn_verify_slots_kernel");
  if (rc != FK_OK) return rc;
  std::vector<uint32_t> hs((size_t)tiles * per);
  FK_CUDA(ctx, cudaMemcpyAsync(hs.data(), slots, hs.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<uint32_t> checks;
  checks.reserve(hs.size());
  for (uint32_t s : hs)
    if (s != 0xFFFFFFFFu) checks.push_back(s);
  st.spot_checks = (uint32_t)checks.size();
  float* ao_v = pos3;
  float* bn_v = nrm3;
  if (!checks.empty()) {
    FK_CUDA(ctx, cudaMemcpyAsync(list, checks.data(), checks.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    hl.spp = prm->full_samples;
    hl.samples = (const float4*)samples_full->ptr;
    hl.offset = 0;
    hl.count = (uint32_t)checks.size();
    hl.ids = list;
    hl.texel_limit = n;
    hl.out0 = ao_v;
    hl.out1 = bn_v;
    rc = fk::launch_hemisphere(ctx, scene, hl);
    if (rc != FK_OK) return rc;
    st.rays += (uint64_t)checks.size() * prm->full_samples;
  }
  // 4. per-tile errors; re-bake the tiles that fail
  rc = launched(ctx, dn::launch_tile_error(ctx->stream, tiles, per, slots, ao, bn, ao_v, bn_v, err),
                "dn_tile_error_kernel");
  if (rc != FK_OK) return rc;
  std::vector<float> he(tiles);
  FK_CUDA(ctx, cudaMemcpyAsync(he.data(), err, (size_t)tiles * 4, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<uint8_t> hf(tiles, 0);
  for (uint32_t t = 0; t < tiles; ++t) {
    if (he[t] < 0.0f) continue;
    ++st.tiles;
    st.worst_tile_error = std::max(st.worst_tile_error, he[t]);
    if (!(he[t] <= prm->max_tile_error)) {
      hf[t] = 1;
      ++st.tiles_failed;
    }
  }
  if (st.tiles_failed) {
    FK_CUDA(ctx, cudaMemcpyAsync(failed, hf.data(), tiles, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t* counter = fk_take_counter(ctx);
    rc = launched(ctx, dn::launch_fallback_list(ctx->stream, n, w, prm->tile, map->indices, ti, failed, list, counter),
                  "dn_fallback_list_kernel");
    if (rc != FK_OK) return rc;
    uint32_t m = 0;
    FK_CUDA(ctx, cudaMemcpyAsync(&m, counter, 4, cudaMemcpyDeviceToHost, ctx->stream));
    FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    st.texels_rebaked = m;
    if (m) {
      hl.spp = prm->full_samples;
      hl.samples = (const float4*)samples_full->ptr;
      hl.offset = 0;
      hl.count = m;
      hl.ids = list;
      hl.texel_limit = n;
      hl.out0 = ao;
      hl.out1 = bn;
      rc = fk::launch_hemisphere(ctx, scene, hl);
      if (rc != FK_OK) return rc;
      st.rays += (uint64_t)m * prm->full_samples;
    }
  }
  if (stats) *stats = st;
  return FK_OK;
}

}  // extern "C"
