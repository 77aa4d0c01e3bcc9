// Batched bakes and the traversal autotuner.
//
// A batch is a set of hemisphere-sampling jobs, each with its own scene,
// mapped texels, sample table, parameters and output buffers.  Jobs of fewer
// than 2^21 rays share persistent launches: their rays are laid end to end in
// one 64-bit ray space (chunked at texel boundaries to fit the scratch), and
// every lane maps its ray back to its job, so small jobs fill the GPU together
// instead of each paying a launch and its tail.  A larger job gains nothing
// from sharing (its launches' tails are a small part of its time, and the
// shared kernel carries each lane's job beside the traversal) and runs alone
// through the single-job path, on the batch's scratch, in the same run and the
// same graph.  The launches of a run can be recorded once into a
// CUDA graph and replayed.  The autotuner times a strided sample of the
// batch's rays (every job represented) for each candidate schedule and keeps
// the fastest: ordered vs skip-pointer traversal, filtered vs divided box
// tests, the refill threshold and the postponed-leaf batch.
#include <algorithm>
#include <cstring>
#include <vector>

#include "fk_internal.h"

namespace {

struct Chunk {
  unsigned long long r0, r1;
  uint32_t t0, t1;
};

constexpr unsigned long long kMaxChunkRays = 1ull << 27;  // 512 MB of distances
// Jobs of at least this many rays run alone through the single-job path.
#ifndef FK_BATCH_SOLO_RAYS
#define FK_BATCH_SOLO_RAYS (1ull << 21)
#endif
constexpr unsigned long long kSoloRays = FK_BATCH_SOLO_RAYS;

// A job run alone (fk_batch's `solo`): its scene and its launch.
struct Solo {
  const fk_scene* scene;
  fk::HemiLaunch h;
};

}  // namespace

struct fk_batch {
  fk_ctx* ctx = nullptr;
  int kind = FK_AO;
  uint32_t njobs = 0;
  unsigned long long total_rays = 0;
  uint32_t total_texels = 0;
  fk::BatchJobDev* jobs = nullptr;        // device job table
  unsigned long long* queues = nullptr;   // one counter per chunk (and one for calibration)
  float* scratch = nullptr;
  unsigned long long scratch_rays = 0;
  std::vector<Chunk> chunks;
  std::vector<Solo> solo;                 // jobs of at least kSoloRays rays, run alone
  uint64_t solo_launches = 0;             // kernel launches of the solo jobs in one run
  int traverse = FK_TRAVERSE_ORDERED;     // tuned choice
  bool ordered_ok = true;                 // every tree fits the 2-wide ordered traversal's stack
  bool ordered4_ok = true;                // every collapsed tree fits the 4-wide traversal's stack
  bool filter = true;
  bool filter_ok = true;                  // every scene's coordinates admit the filtered box tests
  fk_tuning tuning = {8, 8, 0, 0, 0, FK_L2_NONE, 256, 64};
  // the jobs' scenes laid end to end (fk::BatchArgs::cat) and its allocations
  fk::SceneDev cat = {};
  void* cat_mem[8] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static bool fits(const fk_buf* b, uint64_t bytes) { return b && b->bytes >= bytes; }

static int batch_run_chunks(fk_batch* b, int trav, bool filter, const fk_tuning& tun) {
  fk_ctx* ctx = b->ctx;
  if (!b->solo.empty()) {
    // the solo jobs take the batch's schedule: the context's tuning for the duration of their launches
    const fk_tuning saved = ctx->tuning;
    const uint64_t before = ctx->launches;
    ctx->tuning = tun;
    int rc = FK_OK;
    for (Solo& j : b->solo) {
      if (rc != FK_OK) break;
      j.h.traverse = trav | FK_SCHEDULE_DYNAMIC | (filter && b->filter_ok ? 0 : FK_EXACT_BOX_TESTS);
      rc = fk::launch_hemisphere(ctx, j.scene, j.h);
    }
    ctx->tuning = saved;
    if (rc != FK_OK) return rc;
    b->solo_launches = ctx->launches - before;
  }
  for (size_t c = 0; c < b->chunks.size(); ++c) {
    const Chunk& ch = b->chunks[c];
    FK_CUDA(ctx, cudaMemsetAsync(b->queues + c, 0, sizeof(unsigned long long), ctx->stream));
    fk::BatchArgs a;
    a.cat = b->cat;
    a.jobs = b->jobs;
    a.njobs = b->njobs;
    a.r0 = ch.r0;
    a.r1 = ch.r1;
    a.t0 = ch.t0;
    a.t1 = ch.t1;
    a.stride = 1;
    a.scratch = b->scratch;
    a.queue = b->queues + c;
    a.status = ctx->status;
    a.refill = tun.refill;
    a.leaf_batch = tun.leaf_batch;
    a.ray_order = tun.ray_order;
    a.speculate = tun.speculate;
    cudaError_t e = fk::launch_batch(a, b->kind, trav, filter && b->filter_ok, ctx->stream, ctx->sm_count, true);
    if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "batch launch");
    ctx->launches += 2;
  }
  return FK_OK;
}

static void batch_drop_graph(fk_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// Times the trace of every `stride`-th ray of the batch under one schedule.
static int batch_time(fk_batch* b, unsigned long long stride, int trav, bool filter, const fk_tuning& tun,
                      float* ms) {
  fk_ctx* ctx = b->ctx;
  unsigned long long* q = b->queues + b->chunks.size();
  fk::BatchArgs a;
  a.cat = b->cat;
  a.jobs = b->jobs;
  a.njobs = b->njobs;
  a.r0 = 0;
  a.r1 = b->total_rays;
  a.t0 = a.t1 = 0;
  a.stride = stride;
  a.scratch = b->scratch;
  a.queue = q;
  a.status = ctx->status;
  a.refill = tun.refill;
  a.leaf_batch = tun.leaf_batch;
  a.ray_order = FK_RAY_ORDER_SAMPLE;  // calibration samples every stride-th ray
  a.speculate = tun.speculate;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int rc = FK_OK;
  for (int rep = 0; rep < 2 && rc == FK_OK; ++rep) {
    cudaMemsetAsync(q, 0, sizeof(unsigned long long), ctx->stream);
    cudaEventRecord(e0, ctx->stream);
    cudaError_t e = fk::launch_batch(a, b->kind, trav, filter && b->filter_ok, ctx->stream, ctx->sm_count, false);
    cudaEventRecord(e1, ctx->stream);
    if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "batch calibration");
    else if ((e = cudaEventSynchronize(e1)) != cudaSuccess) rc = fk_cuda_fail(ctx, e, "batch calibration sync");
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    best = std::min(best, t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

extern "C" {

int fk_batch_create(fk_ctx* ctx, const fk_batch_job* jobs, uint32_t njobs, int kind, fk_batch** out) {
  if (!ctx || !jobs || !out || njobs == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_batch_create: no jobs");
  if (njobs > fk::kMaxBatchJobs)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_batch_create: at most " + std::to_string(fk::kMaxBatchJobs) + " jobs");
  if (kind < FK_AO || kind > FK_AO_BN) return fk_fail(ctx, FK_ERR_INVALID, "fk_batch_create: unknown kind");
  std::vector<fk::BatchJobDev> table(njobs);
  unsigned long long rays = 0;
  uint64_t texels = 0, nodes = 0, corners = 0, recs2 = 0, recs4 = 0;
  for (uint32_t i = 0; i < njobs; ++i) {
    const fk_batch_job& J = jobs[i];
    const uint64_t n = J.texel_count;
    const std::string who = "fk_batch_create: job " + std::to_string(i);
    if (!J.scene || !ctx->scenes.count(const_cast<fk_scene*>(J.scene)))
      return fk_fail(ctx, FK_ERR_INVALID, who + " has no scene of this context");
    if (J.params.sample_count == 0 || J.params.perm_count == 0)
      return fk_fail(ctx, FK_ERR_INVALID, who + " has zero samples");
    if (!fits(J.coords, 16 * n) || !fits(J.tidx, 4 * n) ||
        !fits(J.samples, 16ull * J.params.sample_count * J.params.perm_count) ||
        !fits(J.out0, (kind == FK_BN ? 12 : 4) * n) || (kind == FK_AO_BN && !fits(J.out1, 12 * n)) ||
        (J.hits0 && !fits(J.hits0, 4 * n)) || (J.hits1 && !fits(J.hits1, 4 * n)))
      return fk_fail(ctx, FK_ERR_INVALID, who + " has a buffer too small for its texels");
    if ((unsigned long long)J.params.sample_count > kMaxChunkRays)
      return fk_fail(ctx, FK_ERR_INVALID, who + " has too many samples per texel");
    // the tuner may pick the 4-wide traversal: its layout must exist before the table is copied
    const int rc = fk::ensure_wide4(ctx, const_cast<fk_scene*>(J.scene));
    if (rc != FK_OK) return rc;
    fk::BatchJobDev& d = table[i];
    std::memset(&d, 0, sizeof(d));
    d.s = fk::scene_dev(J.scene);
    d.samples = (const float4*)J.samples->ptr;
    d.coords = (const float4*)J.coords->ptr;
    d.tidx = (const uint32_t*)J.tidx->ptr;
    d.out0 = (float*)J.out0->ptr;
    d.out1 = kind == FK_AO_BN ? (float*)J.out1->ptr : nullptr;
    d.hits0 = J.hits0 ? (uint32_t*)J.hits0->ptr : nullptr;
    d.hits1 = (kind == FK_AO_BN && J.hits1) ? (uint32_t*)J.hits1->ptr : nullptr;
    d.ray_base = rays;
    d.texel_base = (uint32_t)texels;
    d.texels = J.texel_count;
    d.spp = J.params.sample_count;
    d.perms = J.params.perm_count;
    d.lo = J.params.min_distance;
    d.hi = J.params.max_distance;
    d.node_base = (uint32_t)nodes;
    d.corner_base = (uint32_t)corners;
    d.root2 = J.scene->wide_count ? (int32_t)recs2 : -1;
    d.root4 = J.scene->wide4_count ? (int32_t)recs4 : -1;
    nodes += J.scene->node_count;
    corners += J.scene->corner_count;
    recs2 += J.scene->wide_count;
    recs4 += J.scene->wide4_count;
    if (nodes > 0x7FFFFFFFull || corners > 0xFFFFFFFFull || recs2 > 0x7FFFFFFFull || recs4 > 0x7FFFFFFFull)
      return fk_fail(ctx, FK_ERR_INVALID, "fk_batch_create: the jobs' scenes exceed 2^31 nodes or records");
    rays += n * J.params.sample_count;
    texels += n;
    if (texels > 0xFFFFFFFFull) return fk_fail(ctx, FK_ERR_INVALID, "fk_batch_create: more than 2^32 texels");
  }
  fk_batch* b = new (std::nothrow) fk_batch();
  if (!b) return FK_ERR_NOMEM;
  b->ctx = ctx;
  b->kind = kind;
  b->njobs = njobs;
  b->total_rays = rays;
  b->total_texels = (uint32_t)texels;
  // chunks at texel boundaries, at most kMaxChunkRays rays each, over the
  // jobs that share launches; a solo job's rays and texels are stepped over
  Chunk cur = {0, 0, 0, 0};
  for (uint32_t i = 0; i < njobs; ++i) {
    const fk::BatchJobDev& d = table[i];
    const unsigned long long job_rays = (unsigned long long)d.texels * d.spp;
    if (job_rays >= kSoloRays) {
      if (cur.t1 > cur.t0) b->chunks.push_back(cur);
      cur = {cur.r1 + job_rays, cur.r1 + job_rays, cur.t1 + d.texels, cur.t1 + d.texels};
      const fk_batch_job& J = jobs[i];
      Solo so;
      so.scene = J.scene;
      so.h.kind = kind;
      so.h.spp = J.params.sample_count;
      so.h.perms = J.params.perm_count;
      so.h.min_d = J.params.min_distance;
      so.h.max_d = J.params.max_distance;
      so.h.samples = d.samples;
      so.h.coords = d.coords;
      so.h.tidx = d.tidx;
      so.h.offset = 0;
      so.h.count = d.texels;
      so.h.traverse = 0;
      so.h.out0 = d.out0;
      so.h.out1 = d.out1;
      so.h.hits0 = d.hits0;
      so.h.hits1 = d.hits1;
      b->solo.push_back(so);
      continue;
    }
    uint32_t t = 0;
    while (t < d.texels) {
      unsigned long long room = (kMaxChunkRays - (cur.r1 - cur.r0)) / d.spp;
      if (room == 0) {
        b->chunks.push_back(cur);
        cur = {cur.r1, cur.r1, cur.t1, cur.t1};
        continue;
      }
      uint32_t take = (uint32_t)std::min<unsigned long long>(room, d.texels - t);
      cur.r1 += (unsigned long long)take * d.spp;
      cur.t1 += take;
      t += take;
    }
  }
  if (cur.t1 > cur.t0) b->chunks.push_back(cur);
  b->scratch_rays = std::min<unsigned long long>(std::max<unsigned long long>(rays, 1), kMaxChunkRays);
  for (Solo& j : b->solo) {
    j.h.scratch = nullptr;  // set once the scratch exists (below)
    j.h.scratch_rays = b->scratch_rays;
  }
  int rc = fk_dev_alloc(ctx, (void**)&b->jobs, sizeof(fk::BatchJobDev) * njobs);
  // the concatenated scene: nodes (lo, hi, jump), corners (positions, normals), triangle records, both layouts,
  // node boxes side by side
  const size_t cat_bytes[8] = {16 * (size_t)nodes,   16 * (size_t)nodes,   4 * (size_t)nodes,
                               16 * (size_t)corners, 16 * (size_t)corners, 64 * (size_t)(corners / 3),
                               64 * (size_t)recs2,   32 * (size_t)nodes};
  for (int k = 0; k < 8 && rc == FK_OK; ++k) rc = fk_dev_alloc(ctx, &b->cat_mem[k], std::max<size_t>(cat_bytes[k], 16));
  if (rc == FK_OK && recs4) rc = fk_dev_alloc(ctx, (void**)&b->cat.wide4, 128 * (size_t)recs4);
  if (rc == FK_OK) {
    b->cat.node_lo = (const float4*)b->cat_mem[0];
    b->cat.node_hi = (const float4*)b->cat_mem[1];
    b->cat.node_jump = (const uint32_t*)b->cat_mem[2];
    b->cat.pos4 = (const float4*)b->cat_mem[3];
    b->cat.nrm4 = (const float4*)b->cat_mem[4];
    b->cat.rec = (const float4*)b->cat_mem[5];
    b->cat.rec_bary = b->cat.rec + corners / 3;  // the planes of every job's triangles, then their barycentric terms
    b->cat.wide = (const float4*)b->cat_mem[6];
    b->cat.node_box = (const float4*)b->cat_mem[7];
    b->cat.node_count = (uint32_t)nodes;
    b->cat.corner_count = (uint32_t)corners;
    b->cat.filter_ok = 1;
    for (uint32_t i = 0; i < njobs && rc == FK_OK; ++i)
      if (fk::concat_batch_scene(ctx->stream, jobs[i].scene, table[i].node_base, table[i].corner_base,
                                 table[i].root2 < 0 ? 0 : (uint32_t)table[i].root2,
                                 table[i].root4 < 0 ? 0 : (uint32_t)table[i].root4, b->cat) != FK_OK)
        rc = fk_fail(ctx, FK_ERR_CUDA, "fk_batch_create: scene concatenation");
    if (rc == FK_OK &&
        fk::pair_node_boxes(ctx->stream, b->cat.node_lo, b->cat.node_hi, (uint32_t)nodes,
                            const_cast<float4*>(b->cat.node_box)) != cudaSuccess)
      rc = fk_fail(ctx, FK_ERR_CUDA, "fk_batch_create: node boxes");
  }
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&b->queues, sizeof(unsigned long long) * (b->chunks.size() + 1));
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&b->scratch, sizeof(float) * b->scratch_rays);
  for (Solo& j : b->solo) j.h.scratch = b->scratch;
  if (rc == FK_OK) {
    cudaError_t e = cudaMemcpyAsync(b->jobs, table.data(), sizeof(fk::BatchJobDev) * njobs, cudaMemcpyHostToDevice,
                                    ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "fk_batch_create upload");
  }
  if (rc != FK_OK) {
    fk_batch_free(b);
    return rc;
  }
  // default schedule: ordered when every scene's tree is shallow enough
  for (uint32_t i = 0; i < njobs; ++i) {
    if (jobs[i].scene->odepth > fk::kMaxOrderedDepth) b->ordered_ok = false;
    if (jobs[i].scene->depth4 > fk::kMaxOrdered4Depth) b->ordered4_ok = false;
    if (!jobs[i].scene->filter_ok) b->filter_ok = false;
  }
  b->traverse = b->ordered_ok ? FK_TRAVERSE_ORDERED : FK_TRAVERSE_SKIP;
  b->tuning = ctx->tuning;
  *out = b;
  return FK_OK;
}

int fk_batch_info(const fk_batch* b, uint64_t* rays, uint32_t* texels, uint32_t* launches_per_run) {
  if (!b) return FK_ERR_INVALID;
  if (rays) *rays = b->total_rays;
  if (texels) *texels = b->total_texels;
  // a solo job launches its trace and fold per chunk of its texels
  uint64_t solo = 0;
  for (const Solo& j : b->solo) {
    const uint64_t per = std::max<uint64_t>(1, std::min<uint64_t>(1ull << 27, b->scratch_rays) / j.h.spp);
    solo += 2 * ((j.h.count + per - 1) / per);
  }
  if (launches_per_run) *launches_per_run = (uint32_t)(2 * b->chunks.size() + solo);
  return FK_OK;
}

int fk_batch_tune(fk_batch* b, uint64_t sample_rays, fk_tuning* best_tuning, int* best_traverse) {
  if (!b) return FK_ERR_INVALID;
  fk_ctx* ctx = b->ctx;
  if (sample_rays == 0) sample_rays = 1ull << 22;
  sample_rays = std::min<uint64_t>(sample_rays, b->scratch_rays);
  unsigned long long stride = std::max<unsigned long long>(1, (b->total_rays + sample_rays - 1) / sample_rays);
  struct Cand {
    int trav;
    bool filter;
    fk_tuning t;
  };
  std::vector<Cand> cands;
  const bool ordered_ok = b->ordered_ok;
  const fk_tuning ct = ctx->tuning;  // the context's ray order, block and stack carry over
  auto knobs = [&](uint32_t refill, uint32_t lb, uint32_t spec) {
    fk_tuning t = ct;
    t.refill = refill;
    t.leaf_batch = lb;
    t.speculate = spec;
    t.top_records = 0;
    t.l2_persist = FK_L2_NONE;
    return t;
  };
  // the incumbent first: the batch's current schedule
  cands.push_back({b->traverse, b->filter, b->tuning});
  for (uint32_t refill : {8u, 16u, 20u, 24u}) {
    if (ordered_ok)
      for (uint32_t lb : {4u, 8u, 16u}) cands.push_back({FK_TRAVERSE_ORDERED, true, knobs(refill, lb, 1)});
    if (b->ordered4_ok)
      for (uint32_t lb : {4u, 8u, 16u}) cands.push_back({FK_TRAVERSE_ORDERED4, true, knobs(refill, lb, 1)});
    cands.push_back({FK_TRAVERSE_SKIP, true, knobs(refill, 8, 0)});
  }
  if (ordered_ok) {
    cands.push_back({FK_TRAVERSE_ORDERED, true, knobs(16, 8, 0)});
    cands.push_back({FK_TRAVERSE_ORDERED, false, knobs(16, 8, 1)});
  }
  cands.push_back({FK_TRAVERSE_SKIP, false, knobs(16, 8, 0)});
  float best_ms = 1e30f;
  Cand best = cands[0];
  float warm = 0.0f;
  int rc = batch_time(b, stride, cands[0].trav, cands[0].filter, cands[0].t, &warm);  // warms caches and code
  // A strided sample traces rays of scattered texels, unlike a whole run whose
  // lanes share texels, so small differences on it do not carry over: a
  // candidate replaces the incumbent only when at least 2 % faster.
  for (size_t i = 0; i < cands.size(); ++i) {
    if (rc != FK_OK) break;
    const Cand& c = cands[i];
    float ms = 0.0f;
    rc = batch_time(b, stride, c.trav, c.filter, c.t, &ms);
    if (rc == FK_OK && (i == 0 || ms < 0.98f * best_ms)) {
      best_ms = ms;
      best = c;
    }
  }
  if (rc != FK_OK) return rc;
  b->traverse = best.trav;
  b->filter = best.filter;
  b->tuning = best.t;
  batch_drop_graph(b);
  if (best_tuning) *best_tuning = best.t;
  if (best_traverse) *best_traverse = best.trav | FK_SCHEDULE_DYNAMIC | (best.filter ? 0 : FK_EXACT_BOX_TESTS);
  return FK_OK;
}

int fk_batch_run(fk_batch* b, int traverse) {
  if (!b) return FK_ERR_INVALID;
  int trav = traverse & FK_TRAVERSE_MASK;
  bool filter = b->filter && !(traverse & FK_EXACT_BOX_TESTS);
  if (trav == FK_TRAVERSE_AUTO) trav = b->traverse;
  if (trav == FK_TRAVERSE_ORDERED && b->traverse == FK_TRAVERSE_SKIP && !(traverse & FK_TRAVERSE_MASK))
    trav = FK_TRAVERSE_SKIP;
  if (trav > FK_TRAVERSE_ORDERED4)
    return fk_fail(b->ctx, FK_ERR_INVALID, "fk_batch_run: unknown traversal");
  if (trav == FK_TRAVERSE_ORDERED4 && !b->ordered4_ok)
    return fk_fail(b->ctx, FK_ERR_INVALID, "fk_batch_run: a job's tree is too deep for the 4-wide traversal");
  return batch_run_chunks(b, trav, filter, b->tuning);
}

int fk_batch_capture(fk_batch* b, int traverse) {
  if (!b) return FK_ERR_INVALID;
  fk_ctx* ctx = b->ctx;
  batch_drop_graph(b);
  FK_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = fk_batch_run(b, traverse);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc != FK_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "cudaStreamEndCapture");
  b->graph = g;
  e = cudaGraphInstantiate(&b->exec, g, 0);
  if (e != cudaSuccess) {
    batch_drop_graph(b);
    return fk_cuda_fail(ctx, e, "cudaGraphInstantiate");
  }
  return FK_OK;
}

int fk_batch_replay(fk_batch* b) {
  if (!b) return FK_ERR_INVALID;
  if (!b->exec) return fk_fail(b->ctx, FK_ERR_STATE, "fk_batch_replay: nothing captured");
  FK_CUDA(b->ctx, cudaGraphLaunch(b->exec, b->ctx->stream));
  b->ctx->launches += 2 * b->chunks.size() + b->solo_launches;
  return FK_OK;
}

int fk_batch_free(fk_batch* b) {
  if (!b) return FK_ERR_INVALID;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  batch_drop_graph(b);
  fk_dev_free(b->ctx, b->jobs);
  fk_dev_free(b->ctx, b->queues);
  fk_dev_free(b->ctx, b->scratch);
  for (void* p : b->cat_mem) fk_dev_free(b->ctx, p);
  fk_dev_free(b->ctx, const_cast<float4*>(b->cat.wide4));
  delete b;
  return FK_OK;
}

// Tuner for a single fk_hemisphere call.  It times the call's own trace
// kernel on a sample that keeps the coherence of a whole-map pass: eight
// windows of consecutive texels spread over [offset, offset + count), about
// sample_rays rays in all, traced through the texel-list path (which traces
// each listed texel exactly as the whole-map pass does).  The knobs are
// searched one group at a time from the context's current tuning, each group
// keeping its fastest value: traversal layout, refill x leaf batch,
// speculation, ray order, block shape x stack depth, staged top records, L2
// window.  The context's tuning is left as it was.
int fk_tune_hemisphere(fk_ctx* ctx, const fk_scene* scene, const fk_buf* coords, const fk_buf* tidx, int kind,
                       const fk_sample_params* params, const fk_buf* samples, uint32_t offset, uint32_t count,
                       uint64_t sample_rays, fk_tuning* best_tuning, int* best_traverse) {
  if (!ctx || !scene || !coords || !tidx || !params || !samples || !best_tuning || !best_traverse)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_tune_hemisphere: null argument");
  const uint64_t end = (uint64_t)offset + count;
  if (!fits(coords, 16 * end) || !fits(tidx, 4 * end))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_tune_hemisphere: mapping buffers too small");
  if (count == 0 || params->sample_count == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_tune_hemisphere: no work");
  if (kind < FK_AO || kind > FK_AO_BN) return fk_fail(ctx, FK_ERR_INVALID, "fk_tune_hemisphere: unknown kind");
  if (sample_rays == 0) sample_rays = 1ull << 24;
  // the sample: eight windows of consecutive texels (or every texel)
  const uint64_t want = std::max<uint64_t>(256, sample_rays / params->sample_count);
  std::vector<uint32_t> ids;
  if (want >= count) {
    for (uint32_t t = 0; t < count; ++t) ids.push_back(offset + t);
  } else {
    const uint32_t per = (uint32_t)(want / 8), span = count - per;
    for (uint32_t w = 0; w < 8; ++w) {
      const uint32_t start = offset + (uint32_t)((uint64_t)span * w / 7);
      for (uint32_t t = 0; t < per; ++t) ids.push_back(start + t);
    }
  }
  fk_buf *idb = nullptr, *o0 = nullptr, *o1 = nullptr;
  int rc = fk_buf_alloc(ctx, 4 * ids.size(), &idb);
  if (rc == FK_OK) rc = fk_buf_upload(ctx, idb, 0, ids.data(), 4 * ids.size());
  if (rc == FK_OK) rc = fk_buf_alloc(ctx, 12 * (size_t)end, &o0);
  if (rc == FK_OK) rc = fk_buf_alloc(ctx, 12 * (size_t)end, &o1);
  const fk_tuning saved = ctx->tuning;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rc == FK_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    rc = fk_fail(ctx, FK_ERR_CUDA, "fk_tune_hemisphere: events");
  // one candidate: best of two timed launches
  auto time_one = [&](const fk_tuning& t, int trav, float* ms) -> int {
    ctx->tuning = t;
    float best = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(e0, ctx->stream);
      int r = fk_hemisphere_texels(ctx, scene, coords, tidx, (uint32_t)end, kind, params, samples, idb, 0,
                                   (uint32_t)ids.size(), trav | FK_SCHEDULE_DYNAMIC, o0, kind == FK_AO_BN ? o1 : nullptr,
                                   nullptr, nullptr);
      if (r != FK_OK) return r;
      cudaEventRecord(e1, ctx->stream);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "fk_tune_hemisphere: timing");
      float x = 0.0f;
      cudaEventElapsedTime(&x, e0, e1);
      best = std::min(best, x);
    }
    *ms = best;
    return FK_OK;
  };
  fk_tuning cur = saved;
  int trav = scene->odepth <= fk::kMaxOrderedDepth ? FK_TRAVERSE_ORDERED : FK_TRAVERSE_SKIP;
  float cur_ms = 0.0f;
  if (rc == FK_OK) rc = time_one(cur, trav, &cur_ms);  // warms code and caches
  if (rc == FK_OK) rc = time_one(cur, trav, &cur_ms);
  // tries `t` with traversal `tv`; keeps it when faster
  auto consider = [&](const fk_tuning& t, int tv) {
    float ms = 0.0f;
    if (rc == FK_OK) rc = time_one(t, tv, &ms);
    if (rc == FK_OK && ms < cur_ms) {
      cur_ms = ms;
      cur = t;
      trav = tv;
    }
  };
  if (rc == FK_OK) {
    const fk_tuning base = cur;
    const int base_trav = trav;
    if (base_trav != FK_TRAVERSE_SKIP) consider(base, FK_TRAVERSE_SKIP);
    // the 4-wide layout: built on first use; skipped when its tree is too deep
    if (base_trav == FK_TRAVERSE_ORDERED && fk::ensure_wide4(ctx, const_cast<fk_scene*>(scene)) == FK_OK &&
        scene->depth4 <= fk::kMaxOrdered4Depth)
      consider(base, FK_TRAVERSE_ORDERED4);
  }
  if (rc == FK_OK && trav != FK_TRAVERSE_SKIP) {
    const fk_tuning base = cur;
    for (uint32_t refill : {8u, 16u, 24u, 32u})
      for (uint32_t lb : {4u, 8u, 16u}) {
        fk_tuning t = base;
        t.refill = refill;
        t.leaf_batch = lb;
        if (t.refill != base.refill || t.leaf_batch != base.leaf_batch) consider(t, trav);
      }
    fk_tuning t = cur;
    t.speculate = 1 - t.speculate;
    consider(t, trav);
  }
  if (rc == FK_OK) {
    fk_tuning t = cur;
    t.ray_order = cur.ray_order == FK_RAY_ORDER_SECTOR ? FK_RAY_ORDER_SAMPLE : FK_RAY_ORDER_SECTOR;
    consider(t, trav);
  }
  if (rc == FK_OK && trav == FK_TRAVERSE_ORDERED) {
    const fk_tuning base = cur;
    for (uint32_t block : {128u, 256u, 512u})
      for (uint32_t stack : {32u, 64u}) {
        if (stack == 32 && scene->odepth > 24) continue;
        fk_tuning t = base;
        t.block_threads = block;
        t.stack_depth = stack;
        if (block != base.block_threads || stack != base.stack_depth) consider(t, trav);
      }
    const fk_tuning base2 = cur;
    for (uint32_t top : {0u, 64u, 256u}) {
      fk_tuning t = base2;
      t.top_records = top;
      if (top != base2.top_records) consider(t, trav);
    }
  }
  if (rc == FK_OK) {
    const fk_tuning base = cur;
    for (uint32_t l2 : {(uint32_t)FK_L2_NONE, (uint32_t)FK_L2_TREE, (uint32_t)FK_L2_TRIANGLES}) {
      fk_tuning t = base;
      t.l2_persist = l2;
      if (l2 != base.l2_persist) consider(t, trav);
    }
  }
  ctx->tuning = saved;
  if (saved.l2_persist == FK_L2_NONE && ctx->l2_raised) {
    cudaStreamSynchronize(ctx->stream);
    fk::restore_l2(ctx);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (idb) fk_buf_free(ctx, idb);
  if (o0) fk_buf_free(ctx, o0);
  if (o1) fk_buf_free(ctx, o1);
  if (rc != FK_OK) return rc;
  *best_tuning = cur;
  *best_traverse = trav | FK_SCHEDULE_DYNAMIC;
  return FK_OK;
}

}  // extern "C"
