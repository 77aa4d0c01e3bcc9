// Context, device buffers, device scene and texel-map handles of the C ABI
// (include/fornos_gpu.h).  Replaces the GL buffer layer: ComputeBuffer<T>
// (Src/compute.h:37-87) and the uploads of MeshMapping::init
// (Src/meshmapping.cpp:128-184).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fk_internal.h"
#include "fk_layout.h"
#include "fk_sah_rules.h"

int fk_fail(fk_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int fk_cuda_fail(fk_ctx* ctx, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return fk_fail(ctx, e == cudaErrorMemoryAllocation ? FK_ERR_NOMEM : FK_ERR_CUDA, m);
}

int fk_after_launch(fk_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, what);
  ctx->launches++;
  return FK_OK;
}

int fk_dev_alloc(fk_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return FK_OK;
  if (ctx->pool) FK_CUDA(ctx, cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream));
  else FK_CUDA(ctx, cudaMalloc(p, bytes));
  return FK_OK;
}

void fk_dev_free(fk_ctx* ctx, void* p) {
  if (!p) return;
  if (ctx->pool) cudaFreeAsync(p, ctx->stream);
  else cudaFree(p);
}

uint32_t* fk_take_counter(fk_ctx* ctx) {
  uint32_t* c = ctx->counters + (ctx->next_counter++ % ctx->counter_slots);
  cudaMemsetAsync(c, 0, sizeof(uint32_t), ctx->stream);
  return c;
}

void* fk_scratch(fk_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->scratch_bytes) return ctx->scratch;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->scratch) cudaFree(ctx->scratch);
  ctx->scratch = nullptr;
  ctx->scratch_bytes = 0;
  if (cudaMalloc(&ctx->scratch, bytes) != cudaSuccess) {
    ctx->scratch = nullptr;
    return nullptr;
  }
  ctx->scratch_bytes = bytes;
  return ctx->scratch;
}

namespace fk {
// Builds the collapsed 4-wide layout of the scene's active inner tree on first
// use (from the 2-wide records on the device) and points the scene at it.
int raise_l2(fk_ctx* ctx, size_t bytes, float* hit_ratio) {
  int max_persist = 0;
  FK_CUDA(ctx, cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device));
  if (max_persist <= 0) return fk_fail(ctx, FK_ERR_UNSUPPORTED, "no persisting L2 on this device");
  const size_t want = std::min(bytes, (size_t)max_persist);
  if (!ctx->l2_raised) {
    FK_CUDA(ctx, cudaDeviceGetLimit(&ctx->l2_prev_limit, cudaLimitPersistingL2CacheSize));
    FK_CUDA(ctx, cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)max_persist));
    ctx->l2_raised = true;
  }
  *hit_ratio = bytes ? std::min(1.0f, (float)((double)want / (double)bytes)) : 0.0f;
  return FK_OK;
}

void restore_l2(fk_ctx* ctx) {
  if (!ctx->l2_raised) return;
  cudaCtxResetPersistingL2Cache();
  cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, ctx->l2_prev_limit);
  ctx->l2_raised = false;
}

int ensure_wide4(fk_ctx* ctx, fk_scene* s) {
  const int t = s->tree;
  if (!s->tree_wide4[t] && s->tree_wide[t] && s->tree_count[t] > 0) {
    std::vector<float4> wide(4 * (size_t)s->tree_count[t]), wide4;
    FK_CUDA(ctx, cudaMemcpyAsync(wide.data(), s->tree_wide[t], sizeof(float4) * wide.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    uint32_t n4 = 0, d4 = 0;
    collapse_wide4(wide, wide4, n4, d4);
    float4* dw4 = nullptr;
    int rc = fk_dev_alloc(ctx, (void**)&dw4, sizeof(float4) * wide4.size());
    if (rc != FK_OK) return rc;
    if (cudaMemcpyAsync(dw4, wide4.data(), sizeof(float4) * wide4.size(), cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      fk_dev_free(ctx, dw4);
      return fk_fail(ctx, FK_ERR_CUDA, "4-wide layout upload");
    }
    s->tree_wide4[t] = dw4;
    s->tree_count4[t] = n4;
    s->tree_depth4[t] = d4;
    s->bytes += sizeof(float4) * wide4.size();
  }
  s->wide4 = s->tree_wide4[t];
  s->wide4_count = s->tree_count4[t];
  s->depth4 = s->tree_depth4[t];
  return FK_OK;
}
}  // namespace fk

extern "C" {

int fk_ctx_create(int device, fk_ctx** out) {
  if (!out) return FK_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return FK_ERR_UNSUPPORTED;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return FK_ERR_CUDA;
  if (prop.major != 10) return FK_ERR_UNSUPPORTED;  // kernels are built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return FK_ERR_CUDA;
  fk_ctx* c = new (std::nothrow) fk_ctx();
  if (!c) return FK_ERR_NOMEM;
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return FK_ERR_CUDA;
  }
  c->stream = c->own_stream;
  c->counter_slots = 1024;
  if (cudaMalloc(&c->counters, c->counter_slots * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->status, sizeof(int)) != cudaSuccess) {
    cudaFree(c->counters);
    cudaStreamDestroy(c->own_stream);
    delete c;
    return FK_ERR_NOMEM;
  }
  cudaMemset(c->counters, 0, c->counter_slots * sizeof(uint32_t));
  cudaMemset(c->status, 0, sizeof(int));
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&c->pool, &props) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  } else {
    c->pool = nullptr;  // plain cudaMalloc / cudaFree
    cudaGetLastError();
  }
  *out = c;
  return FK_OK;
}

int fk_ctx_destroy(fk_ctx* ctx) {
  if (!ctx) return FK_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (fk_buf* b : ctx->bufs) { fk_dev_free(ctx, b->ptr); delete b; }
  for (fk_scene* s : std::set<fk_scene*>(ctx->scenes)) fk_scene_free(ctx, s);
  for (fk_texel_map* m : std::set<fk_texel_map*>(ctx->maps)) fk_texel_map_free(ctx, m);
  cudaStreamSynchronize(ctx->stream);
  fk::restore_l2(ctx);
  cudaFree(ctx->counters);
  cudaFree(ctx->status);
  cudaFree(ctx->scratch);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->stage_done) cudaEventDestroy(ctx->stage_done);
  if (ctx->stage) cudaFreeHost(ctx->stage);
  cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return FK_OK;
}

int fk_ctx_trim(fk_ctx* ctx) {
  if (!ctx) return FK_ERR_INVALID;
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->pool) FK_CUDA(ctx, cudaMemPoolTrimTo(ctx->pool, 0));
  if (ctx->stage) FK_CUDA(ctx, cudaFreeHost(ctx->stage));  // its copies were on the stream
  ctx->stage = nullptr;
  ctx->stage_bytes = 0;
  return FK_OK;
}

const char* fk_last_error(const fk_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fk_ctx_set_stream(fk_ctx* ctx, void* s) {
  if (!ctx) return FK_ERR_INVALID;
  // work queued on the old stream (and memory it gives back) is done before
  // the new stream orders anything
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->stream = s ? (cudaStream_t)s : ctx->own_stream;
  return FK_OK;
}

void* fk_ctx_stream(const fk_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int fk_sync(fk_ctx* ctx) {
  if (!ctx) return FK_ERR_INVALID;
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return FK_OK;
}

uint64_t fk_launch_count(const fk_ctx* ctx) { return ctx ? ctx->launches : 0; }

int fk_ctx_set_tuning(fk_ctx* ctx, const fk_tuning* t) {
  if (!ctx || !t) return FK_ERR_INVALID;
  if (t->refill < 1 || t->refill > 32 || t->leaf_batch < 1 || t->leaf_batch > 32 || t->speculate > 1 ||
      t->ray_order > FK_RAY_ORDER_SECTOR || t->top_records > FK_MAX_TOP_RECORDS || t->l2_persist > FK_L2_TRIANGLES ||
      (t->block_threads != 128 && t->block_threads != 256 && t->block_threads != 512) ||
      (t->stack_depth != 32 && t->stack_depth != 64))
    return fk_fail(ctx, FK_ERR_INVALID,
                   "fk_ctx_set_tuning: refill and leaf_batch in 1..32, speculate 0 or 1, ray_order 0 or 1, "
                   "top_records at most 1024, l2_persist 0..2, block_threads 128 / 256 / 512, stack_depth 32 / 64");
  if (t->l2_persist == FK_L2_NONE && ctx->l2_raised) {
    FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // windows already queued finish first
    fk::restore_l2(ctx);
  }
  ctx->tuning = *t;
  return FK_OK;
}

int fk_ctx_get_tuning(const fk_ctx* ctx, fk_tuning* t) {
  if (!ctx || !t) return FK_ERR_INVALID;
  *t = ctx->tuning;
  return FK_OK;
}

// ------------------------------------------------------------------ buffers
int fk_buf_alloc(fk_ctx* ctx, size_t bytes, fk_buf** out) {
  if (!ctx || !out || bytes == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_buf_alloc: zero size or null");
  fk_buf* b = new (std::nothrow) fk_buf();
  if (!b) return FK_ERR_NOMEM;
  int rc = fk_dev_alloc(ctx, &b->ptr, bytes);
  if (rc != FK_OK) {
    delete b;
    return rc;
  }
  cudaError_t e = cudaMemsetAsync(b->ptr, 0, bytes, ctx->stream);
  if (e != cudaSuccess) {
    fk_dev_free(ctx, b->ptr);
    delete b;
    return fk_cuda_fail(ctx, e, "cudaMemsetAsync");
  }
  b->ctx = ctx;
  b->bytes = bytes;
  ctx->bufs.insert(b);
  *out = b;
  return FK_OK;
}

int fk_buf_upload(fk_ctx* ctx, fk_buf* b, size_t off, const void* src, size_t bytes) {
  if (!ctx || !b || (!src && bytes) || off > b->bytes || bytes > b->bytes - off)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_buf_upload: range outside the buffer");
  if (!bytes) return FK_OK;
  FK_CUDA(ctx, cudaMemcpyAsync((char*)b->ptr + off, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return FK_OK;
}

int fk_buf_download(fk_ctx* ctx, const fk_buf* b, size_t off, void* dst, size_t bytes) {
  if (!ctx || !b || (!dst && bytes) || off > b->bytes || bytes > b->bytes - off)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_buf_download: range outside the buffer");
  if (!bytes) return FK_OK;
  FK_CUDA(ctx, cudaMemcpyAsync(dst, (const char*)b->ptr + off, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return FK_OK;
}

int fk_buf_free(fk_ctx* ctx, fk_buf* b) {
  if (!ctx || !b || !ctx->bufs.count(b)) return fk_fail(ctx, FK_ERR_INVALID, "fk_buf_free: unknown buffer");
  // the caller may have used the buffer on any stream: wait for the device
  // before the pool can hand the memory out again
  cudaDeviceSynchronize();
  return fk_buf_release(ctx, b);
}

int fk_buf_release(fk_ctx* ctx, fk_buf* b) {
  if (!ctx || !b || !ctx->bufs.count(b)) return fk_fail(ctx, FK_ERR_INVALID, "fk_buf_free: unknown buffer");
  fk_dev_free(ctx, b->ptr);
  ctx->bufs.erase(b);
  delete b;
  return FK_OK;
}

size_t fk_buf_size(const fk_buf* b) { return b ? b->bytes : 0; }
void* fk_buf_device_ptr(const fk_buf* b) { return b ? b->ptr : nullptr; }

// ------------------------------------------------------------------ scene
}  // extern "C"

// Scene from a flattened node array: host corner arrays (fk_scene_upload), or
// the device build's arrays, which the scene adopts (`dev`: nodes, corners).
static int scene_create(fk_ctx* ctx, const fk_bvh_node* nodes, uint32_t nn, const float* pos4, const float* nrm4,
                        uint32_t nc, fk::DevBvh* dev, fk_scene** out) {
  if (!ctx || !out || !nodes || (!dev && (!pos4 || !nrm4)) || nn == 0 || nc == 0 || nc % 3 != 0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_scene_upload: empty or malformed scene");
  // Check the skip-pointer structure so no kernel can walk outside it, and
  // lay out the device arrays (fk_layout.cpp, over host threads) in the
  // context's pinned staging, once the previous upload's copies from it are
  // done.
  const size_t stage_need = fk::layout_bytes(nn);
  if (ctx->stage_done) FK_CUDA(ctx, cudaEventSynchronize(ctx->stage_done));
  if (ctx->stage_bytes < stage_need) {
    if (ctx->stage) FK_CUDA(ctx, cudaFreeHost(ctx->stage));
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    if (cudaMallocHost(&ctx->stage, stage_need) != cudaSuccess) {
      cudaGetLastError();
      ctx->stage = nullptr;
      return fk_fail(ctx, FK_ERR_NOMEM, "fk_scene_upload: pinned staging of " + std::to_string(stage_need) + " bytes");
    }
    ctx->stage_bytes = stage_need;
  }
  fk::NodeLayout lay;
  const std::string bad = fk::layout_nodes(nodes, nn, nc, ctx->stage, lay);
  if (!bad.empty()) return fk_fail(ctx, FK_ERR_INVALID, bad);
  const uint32_t leaves = lay.leaves, nw = lay.wide_count, maxd = lay.depth;
  const bool sah_ok = lay.sah_ok;  // leaf boxes within the rebuilt tree's coordinate range
  const std::vector<uint32_t>& leaf_ids = lay.leaf_ids;
  fk_scene* s = new (std::nothrow) fk_scene();
  if (!s) return FK_ERR_NOMEM;
  s->ctx = ctx;
  s->node_count = nn;
  s->corner_count = nc;
  s->depth = maxd;
  s->odepth = maxd;
  s->leaf_count = leaves;
  s->wide_count = nw;
  s->wide4_count = 0;  // the 4-wide layout is built on first use (fk::ensure_wide4)
  s->depth4 = 0;
  s->root_is_leaf = nodes[0].jump == 1;
  // The filtered box tests assume |box - origin| < 2^26; ray origins lie on
  // the scene's triangles, so box and corner coordinates below 2^24 suffice.
  // The conservative inner test also takes each box's faces in order.
  {
    const float lim = 16777216.0f;
    bool ok = lay.coords_ok;
    if (!dev) {
      // the corners are checked on the device once uploaded (below)
    } else if (ok) {
      bool below = false;
      const int rc = fk::corners_below(ctx, dev->pos4, nc, lim, &below);
      if (rc != FK_OK) {
        delete s;
        return rc;
      }
      ok = below;
    }
    s->filter_ok = ok ? 1 : 0;
  }
  size_t nb = sizeof(float4) * nn, cb = sizeof(float4) * (size_t)nc;
  int rc = FK_OK;
  auto up = [&](void** dst, const void* src, size_t bytes) {
    if (rc != FK_OK || bytes == 0) return;
    rc = fk_dev_alloc(ctx, dst, bytes);
    if (rc == FK_OK) {
      cudaError_t e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
      if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "scene upload");
    }
    s->bytes += bytes;
  };
  if (dev) {  // adopted: the scene frees them
    s->node_lo = dev->lo;
    s->node_hi = dev->hi;
    s->node_jump = dev->jump;
    s->pos4 = dev->pos4;
    s->nrm4 = dev->nrm4;
    *dev = fk::DevBvh{};
    s->bytes += 2 * nb + sizeof(uint32_t) * nn + 2 * cb;
  } else {
    up((void**)&s->node_lo, lay.lo, nb);
    up((void**)&s->node_hi, lay.hi, nb);
    up((void**)&s->node_jump, lay.jump, sizeof(uint32_t) * nn);
    up((void**)&s->pos4, pos4, cb);
    up((void**)&s->nrm4, nrm4, cb);
  }
  up((void**)&s->wide, lay.wide, sizeof(float4) * 4 * (size_t)nw);
  {  // the copies above read the staging: the next upload waits for them
    cudaError_t e = cudaSuccess;
    if (!ctx->stage_done) e = cudaEventCreateWithFlags(&ctx->stage_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->stage_done, ctx->stream);
    if (e != cudaSuccess) {
      cudaStreamSynchronize(ctx->stream);
      if (rc == FK_OK) rc = fk_cuda_fail(ctx, e, "scene upload staging");
    }
  }
  if (rc == FK_OK && !dev && s->filter_ok) {  // the uploaded corners, on the device: 100 MB take ~20 us there
    bool below = false;
    rc = fk::corners_below(ctx, s->pos4, nc, 16777216.0f, &below);
    s->filter_ok = below ? 1 : 0;
  }
  s->tree_wide[FK_TREE_REFERENCE] = s->wide;
  s->tree_count[FK_TREE_REFERENCE] = nw;
  s->tree_depth[FK_TREE_REFERENCE] = maxd;
  // The inner tree the ordered traversals walk by default: rebuilt on the
  // device over the same leaves with a surface-area split on all three face
  // pairs (fk_sah.cu); the reference's records above stay available
  // (fk_scene_set_tree).  Too deep for the ordered traversals: not kept.
  if (rc == FK_OK && nw > 0 && sah_ok) {
    float4* sw = nullptr;
    uint32_t sdepth = 0;
    rc = fk::build_sah_device(ctx, s->node_lo, s->node_hi, leaf_ids, &sw, &sdepth);
    if (rc == FK_OK && sw) {
      s->tree_wide[FK_TREE_SAH] = sw;
      s->tree_count[FK_TREE_SAH] = leaves - 1;
      s->tree_depth[FK_TREE_SAH] = sdepth;
      s->bytes += sizeof(float4) * 4 * (size_t)(leaves - 1);
    }
  }
  if (rc == FK_OK) {
    rc = fk_dev_alloc(ctx, (void**)&s->tri_rec, 4 * sizeof(float4) * (size_t)(nc / 3));
    s->bytes += 4 * sizeof(float4) * (size_t)(nc / 3);
  }
  if (rc == FK_OK) rc = fk::launch_tri_records(ctx, s);
  if (rc == FK_OK) {
    rc = fk_dev_alloc(ctx, (void**)&s->node_box, 2 * sizeof(float4) * (size_t)nn);
    s->bytes += 2 * sizeof(float4) * (size_t)nn;
  }
  if (rc == FK_OK) {
    const cudaError_t e = fk::pair_node_boxes(ctx->stream, s->node_lo, s->node_hi, nn, s->node_box);
    if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "pair_boxes_kernel");
    else ++ctx->launches;
  }
  if (rc == FK_OK) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "scene upload sync");
  }
  if (rc != FK_OK) {
    ctx->scenes.insert(s);
    fk_scene_free(ctx, s);
    return rc;
  }
  ctx->scenes.insert(s);
  if (s->tree_wide[FK_TREE_SAH]) {
    rc = fk_scene_set_tree(s, FK_TREE_SAH);
    if (rc != FK_OK) {
      fk_scene_free(ctx, s);
      return rc;
    }
  }
  *out = s;
  return FK_OK;
}

// Flattened nodes of a device build, downloaded into the ABI's node layout.
static int dev_nodes(fk_ctx* ctx, const fk::DevBvh& d, std::vector<fk_bvh_node>& nodes) {
  const uint32_t nn = d.node_count;
  std::vector<float4> lo(nn), hi(nn);
  std::vector<uint32_t> jump(nn);
  FK_CUDA(ctx, cudaMemcpyAsync(lo.data(), d.lo, sizeof(float4) * nn, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaMemcpyAsync(hi.data(), d.hi, sizeof(float4) * nn, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaMemcpyAsync(jump.data(), d.jump, sizeof(uint32_t) * nn, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  nodes.resize(nn);
  for (uint32_t i = 0; i < nn; ++i) {
    fk_bvh_node& n = nodes[i];
    n.aabb_min[0] = lo[i].x;
    n.aabb_min[1] = lo[i].y;
    n.aabb_min[2] = lo[i].z;
    n.aabb_max[0] = hi[i].x;
    n.aabb_max[1] = hi[i].y;
    n.aabb_max[2] = hi[i].z;
    std::memcpy(&n.start, &lo[i].w, 4);
    std::memcpy(&n.end, &hi[i].w, 4);
    n.jump = jump[i];
  }
  return FK_OK;
}

static void dev_free(fk_ctx* ctx, fk::DevBvh& d) {
  for (void* p : {(void*)d.lo, (void*)d.hi, (void*)d.jump, (void*)d.pos4, (void*)d.nrm4}) fk_dev_free(ctx, p);
  d = fk::DevBvh{};
}

extern "C" {

int fk_scene_upload(fk_ctx* ctx, const fk_bvh_node* nodes, uint32_t nn, const float* pos4, const float* nrm4,
                    uint32_t nc, fk_scene** out) {
  return scene_create(ctx, nodes, nn, pos4, nrm4, nc, nullptr, out);
}

int fk_bvh_build_flat(fk_ctx* ctx, const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, fk_bvh_node* nodes,
                      uint32_t node_capacity, uint32_t* node_count, float* positions4, float* normals4) {
  if (!ctx || !mesh || max_tris == 0 || !node_count)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_bvh_build_flat: bad arguments");
  fk::DevBvh d;
  int rc = fk::build_bvh_device(ctx, mesh, max_tris, max_depth, &d);
  if (rc != FK_OK) return rc;
  *node_count = d.node_count;
  std::vector<fk_bvh_node> v;
  if (nodes || positions4 || normals4) {
    if (nodes && node_capacity < d.node_count) {
      dev_free(ctx, d);
      return fk_fail(ctx, FK_ERR_INVALID, "fk_bvh_build_flat: node capacity below the node count");
    }
    if (nodes && (rc = dev_nodes(ctx, d, v)) == FK_OK) std::memcpy(nodes, v.data(), sizeof(fk_bvh_node) * v.size());
    const size_t cb = sizeof(float4) * (size_t)d.corner_count;
    if (rc == FK_OK && positions4 && cb &&
        cudaMemcpyAsync(positions4, d.pos4, cb, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
      rc = fk_fail(ctx, FK_ERR_CUDA, "fk_bvh_build_flat: corner copy");
    if (rc == FK_OK && normals4 && cb &&
        cudaMemcpyAsync(normals4, d.nrm4, cb, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
      rc = fk_fail(ctx, FK_ERR_CUDA, "fk_bvh_build_flat: corner copy");
    if (rc == FK_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = fk_fail(ctx, FK_ERR_CUDA, "fk_bvh_build_flat: sync");
  }
  dev_free(ctx, d);
  return rc;
}

int fk_scene_build(fk_ctx* ctx, const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, fk_scene** out) {
  if (!ctx || !mesh || !out || max_tris == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_scene_build: bad arguments");
  fk::DevBvh d;
  int rc = fk::build_bvh_device(ctx, mesh, max_tris, max_depth, &d);
  if (rc != FK_OK) return rc;
  if (d.node_count == 0) {
    dev_free(ctx, d);
    return fk_fail(ctx, FK_ERR_INVALID, "fk_scene_build: the mesh has no triangles");
  }
  std::vector<fk_bvh_node> v;
  rc = dev_nodes(ctx, d, v);
  if (rc == FK_OK) rc = scene_create(ctx, v.data(), d.node_count, nullptr, nullptr, d.corner_count, &d, out);
  dev_free(ctx, d);  // nothing left after a successful adoption
  return rc;
}

int fk_scene_free(fk_ctx* ctx, fk_scene* s) {
  if (!ctx || !s || !ctx->scenes.count(s)) return fk_fail(ctx, FK_ERR_INVALID, "fk_scene_free: unknown scene");
  cudaStreamSynchronize(ctx->stream);
  void* ps[] = {s->node_lo,         s->node_hi,         s->node_jump, s->pos4,    s->nrm4,  s->tree_wide[0],
                s->tree_wide[1],   s->tree_wide4[0],   s->tree_wide4[1], s->tri_rec, s->top, s->node_box};
  for (void* p : ps) fk_dev_free(ctx, p);
  ctx->scenes.erase(s);
  delete s;
  return FK_OK;
}

int fk_scene_set_tree(fk_scene* s, int tree) {
  if (!s) return FK_ERR_INVALID;
  fk_ctx* ctx = s->ctx;
  if (tree != FK_TREE_REFERENCE && tree != FK_TREE_SAH)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_scene_set_tree: unknown tree");
  if (tree == FK_TREE_SAH && !s->tree_wide[FK_TREE_SAH] && !s->root_is_leaf)
    return fk_fail(ctx, FK_ERR_UNSUPPORTED, "fk_scene_set_tree: the rebuilt tree is deeper than the ordered traversal's 48");
  if (s->root_is_leaf) tree = FK_TREE_REFERENCE;  // a single leaf has no inner tree to rebuild
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // work queued on the previous tree is done
  s->tree = tree;
  s->wide = s->tree_wide[tree];
  s->wide4 = s->tree_wide4[tree];
  s->wide_count = s->tree_count[tree];
  s->wide4_count = s->tree_count4[tree];
  s->odepth = s->tree_depth[tree];
  s->depth4 = s->tree_depth4[tree];
  return FK_OK;
}

int fk_diag_scene_tree(fk_ctx* ctx, const fk_scene* s, int tree, float* records, uint32_t capacity, uint32_t* count,
                       uint32_t* depth) {
  if (!ctx || !s || !ctx->scenes.count(const_cast<fk_scene*>(s)) || (tree != FK_TREE_REFERENCE && tree != FK_TREE_SAH))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_diag_scene_tree: bad arguments");
  const uint32_t n = s->tree_wide[tree] ? s->tree_count[tree] : 0;
  if (count) *count = n;
  if (depth) *depth = s->tree_depth[tree];
  if (records && n) {
    if (capacity < n) return fk_fail(ctx, FK_ERR_INVALID, "fk_diag_scene_tree: capacity below the record count");
    FK_CUDA(ctx, cudaMemcpyAsync(records, s->tree_wide[tree], sizeof(float4) * 4 * (size_t)n, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return FK_OK;
}

int fk_scene_get_info(const fk_scene* s, fk_scene_info* o) {
  if (!s || !o) return FK_ERR_INVALID;
  o->node_count = s->node_count;
  o->corner_count = s->corner_count;
  o->depth = s->depth;
  o->leaf_count = s->leaf_count;
  o->device_bytes = s->bytes;
  return FK_OK;
}

// ------------------------------------------------------------------ texel map
int fk_texel_map_from_host(fk_ctx* ctx, uint32_t w, uint32_t h, uint32_t count, const float* pix8,
                           const float* pixt12, const uint32_t* idx, fk_texel_map** out) {
  int rc = fk::texel_map_upload_async(ctx, w, h, count, pix8, pixt12, idx, out);
  if (rc == FK_OK && count) {
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      fk_texel_map_free(ctx, *out);
      *out = nullptr;
      return fk_cuda_fail(ctx, e, "fk_texel_map_from_host");
    }
  }
  return rc;
}

}  // extern "C"

namespace fk {

// fk_texel_map_from_host without the final wait: the copies are queued on the
// context's stream, so the host rows must stay unchanged until that stream
// has passed them.
int texel_map_upload_async(fk_ctx* ctx, uint32_t w, uint32_t h, uint32_t count, const float* pix8,
                           const float* pixt12, const uint32_t* idx, fk_texel_map** out) {
  if (!ctx || !out || (count && (!pix8 || !pixt12 || !idx)) || (uint64_t)count > (uint64_t)w * h)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_texel_map_from_host: bad arguments");
  fk_texel_map* m = new (std::nothrow) fk_texel_map();
  if (!m) return FK_ERR_NOMEM;
  m->ctx = ctx;
  m->width = w;
  m->height = h;
  m->count = count;
  int rc = fk_dev_alloc(ctx, (void**)&m->pix, 32 * (size_t)count);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&m->pixt, 48 * (size_t)count);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&m->indices, 4 * (size_t)count);
  ctx->maps.insert(m);
  if (rc != FK_OK) {
    fk_texel_map_free(ctx, m);
    return rc;
  }
  if (count) {
    FK_CUDA(ctx, cudaMemcpyAsync(m->pix, pix8, 32 * (size_t)count, cudaMemcpyHostToDevice, ctx->stream));
    FK_CUDA(ctx, cudaMemcpyAsync(m->pixt, pixt12, 48 * (size_t)count, cudaMemcpyHostToDevice, ctx->stream));
    FK_CUDA(ctx, cudaMemcpyAsync(m->indices, idx, 4 * (size_t)count, cudaMemcpyHostToDevice, ctx->stream));
  }
  *out = m;
  return FK_OK;
}

}  // namespace fk

extern "C" {

int fk_texel_map_info(const fk_texel_map* m, uint32_t* w, uint32_t* h, uint32_t* count) {
  if (!m) return FK_ERR_INVALID;
  if (w) *w = m->width;
  if (h) *h = m->height;
  if (count) *count = m->count;
  return FK_OK;
}

int fk_texel_map_download(fk_ctx* ctx, const fk_texel_map* m, float* pix8, float* pixt12, uint32_t* idx) {
  if (!ctx || !m) return fk_fail(ctx, FK_ERR_INVALID, "fk_texel_map_download: null");
  if (!m->count) return FK_OK;
  if (pix8) FK_CUDA(ctx, cudaMemcpyAsync(pix8, m->pix, 32 * (size_t)m->count, cudaMemcpyDeviceToHost, ctx->stream));
  if (pixt12) FK_CUDA(ctx, cudaMemcpyAsync(pixt12, m->pixt, 48 * (size_t)m->count, cudaMemcpyDeviceToHost, ctx->stream));
  if (idx) FK_CUDA(ctx, cudaMemcpyAsync(idx, m->indices, 4 * (size_t)m->count, cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return FK_OK;
}

int fk_texel_map_free(fk_ctx* ctx, fk_texel_map* m) {
  if (!ctx || !m || !ctx->maps.count(m)) return fk_fail(ctx, FK_ERR_INVALID, "fk_texel_map_free: unknown map");
  cudaStreamSynchronize(ctx->stream);
  fk_dev_free(ctx, m->pix);
  fk_dev_free(ctx, m->pixt);
  fk_dev_free(ctx, m->indices);
  ctx->maps.erase(m);
  delete m;
  return FK_OK;
}

}  // extern "C"
