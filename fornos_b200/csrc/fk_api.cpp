// Dispatch entry points of the C ABI (the replacement for LoadComputeShader_*
// + glDispatchCompute) and the host solver layer above them: MeshMapping
// (Src/meshmapping.cpp:128-218) and the six solvers (Src/solver_*.cpp), with
// the reference's init / runStep / getResults / progress contract.
#include <cfloat>
#include <cstring>
#include <vector>

#include "fk_internal.h"

namespace {

constexpr uint32_t kGroup = 64;  // k_groupSize: result buffers are rounded up to it

inline uint32_t round_up(uint32_t n) { return (n + kGroup - 1) / kGroup * kGroup; }

bool fits(const fk_buf* b, uint64_t bytes) { return b && b->bytes >= bytes; }

}  // namespace

extern "C" {

int fk_meshmap(fk_ctx* ctx, const fk_scene* s, const fk_texel_map* m, int cull, float max_dist, uint32_t offset,
               uint32_t count, fk_buf* coords, fk_buf* tidx) {
  if (!ctx || !s || !m) return fk_fail(ctx, FK_ERR_INVALID, "fk_meshmap: null handle");
  if (!(max_dist > 0.0f)) return fk_fail(ctx, FK_ERR_INVALID, "fk_meshmap: max_dist must be positive");
  if ((uint64_t)offset + count > m->count) return fk_fail(ctx, FK_ERR_INVALID, "fk_meshmap: texel range outside the map");
  uint64_t end = (uint64_t)offset + count;
  if (!fits(coords, 16 * end) || !fits(tidx, 4 * end))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_meshmap: output buffers too small");
  return fk::launch_meshmap(ctx, s, m, cull, max_dist, offset, count, (float4*)coords->ptr, (uint32_t*)tidx->ptr);
}

int fk_hemisphere(fk_ctx* ctx, const fk_scene* s, const fk_buf* coords, const fk_buf* tidx, int kind,
                  const fk_sample_params* prm, const fk_buf* samples, uint32_t offset, uint32_t count, int traverse,
                  fk_buf* out0, fk_buf* out1, fk_buf* hits0, fk_buf* hits1) {
  if (!ctx || !s || !coords || !tidx || !prm || !samples || !out0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: null argument");
  if (kind < FK_AO || kind > FK_AO_BN) return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: unknown kind");
  if (prm->sample_count == 0 || prm->perm_count == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: zero samples");
  if ((traverse & ~(FK_TRAVERSE_MASK | FK_SCHEDULE_MASK | FK_EXACT_BOX_TESTS)) ||
      (traverse & FK_TRAVERSE_MASK) > FK_TRAVERSE_ORDERED4 ||
      (traverse & FK_SCHEDULE_MASK) > FK_SCHEDULE_DYNAMIC)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: unknown traversal or schedule");
  uint64_t end = (uint64_t)offset + count;
  if (!fits(coords, 16 * end) || !fits(tidx, 4 * end)) return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: mapping buffers too small");
  if (!fits(samples, 16ull * prm->sample_count * prm->perm_count))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: sample table smaller than perm_count x sample_count");
  uint64_t w0 = (kind == FK_BN ? 12 : 4) * end;
  if (!fits(out0, w0) || (kind == FK_AO_BN && !fits(out1, 12 * end)))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: output buffers too small");
  if ((hits0 && !fits(hits0, 4 * end)) || (hits1 && !fits(hits1, 4 * end)))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: hit buffers too small");
  if (count == 0) return FK_OK;
  fk::HemiLaunch h;
  h.kind = kind;
  h.spp = prm->sample_count;
  h.perms = prm->perm_count;
  h.min_d = prm->min_distance;
  h.max_d = prm->max_distance;
  h.samples = (const float4*)samples->ptr;
  h.coords = (const float4*)coords->ptr;
  h.tidx = (const uint32_t*)tidx->ptr;
  h.offset = offset;
  h.count = count;
  h.traverse = traverse;
  h.out0 = (float*)out0->ptr;
  h.out1 = kind == FK_AO_BN ? (float*)out1->ptr : nullptr;
  h.hits0 = hits0 ? (uint32_t*)hits0->ptr : nullptr;
  h.hits1 = (kind == FK_AO_BN && hits1) ? (uint32_t*)hits1->ptr : nullptr;
  return fk::launch_hemisphere(ctx, s, h);
}

int fk_hemisphere_texels(fk_ctx* ctx, const fk_scene* s, const fk_buf* coords, const fk_buf* tidx,
                         uint32_t texel_count, int kind, const fk_sample_params* prm, const fk_buf* samples,
                         const fk_buf* ids, uint32_t offset, uint32_t count, int traverse, fk_buf* out0, fk_buf* out1,
                         fk_buf* hits0, fk_buf* hits1) {
  if (!ctx || !s || !coords || !tidx || !prm || !samples || !ids || !out0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: null argument");
  if (kind < FK_AO || kind > FK_AO_BN) return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: unknown kind");
  if (prm->sample_count == 0 || prm->perm_count == 0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: zero samples");
  if ((traverse & ~(FK_TRAVERSE_MASK | FK_SCHEDULE_MASK | FK_EXACT_BOX_TESTS)) ||
      (traverse & FK_TRAVERSE_MASK) > FK_TRAVERSE_ORDERED4 || (traverse & FK_SCHEDULE_MASK) > FK_SCHEDULE_DYNAMIC)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: unknown traversal or schedule");
  if ((traverse & FK_SCHEDULE_MASK) == FK_SCHEDULE_STATIC)
    return fk_fail(ctx, FK_ERR_UNSUPPORTED, "fk_hemisphere_texels: texel lists run on the dynamic schedule only");
  const uint64_t n = texel_count;
  if (!fits(ids, 4 * ((uint64_t)offset + count))) return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: id list too small");
  if (!fits(coords, 16 * n) || !fits(tidx, 4 * n))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: mapping buffers smaller than texel_count");
  if (!fits(samples, 16ull * prm->sample_count * prm->perm_count))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: sample table smaller than perm_count x sample_count");
  if (!fits(out0, (kind == FK_BN ? 12 : 4) * n) || (kind == FK_AO_BN && !fits(out1, 12 * n)))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: output buffers smaller than texel_count");
  if ((hits0 && !fits(hits0, 4 * n)) || (kind == FK_AO_BN && hits1 && !fits(hits1, 4 * n)))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_texels: hit buffers smaller than texel_count");
  if (count == 0) return FK_OK;
  fk::HemiLaunch h;
  h.kind = kind;
  h.spp = prm->sample_count;
  h.perms = prm->perm_count;
  h.min_d = prm->min_distance;
  h.max_d = prm->max_distance;
  h.samples = (const float4*)samples->ptr;
  h.coords = (const float4*)coords->ptr;
  h.tidx = (const uint32_t*)tidx->ptr;
  h.offset = offset;
  h.count = count;
  h.traverse = traverse;
  h.out0 = (float*)out0->ptr;
  h.out1 = kind == FK_AO_BN ? (float*)out1->ptr : nullptr;
  h.hits0 = hits0 ? (uint32_t*)hits0->ptr : nullptr;
  h.hits1 = (kind == FK_AO_BN && hits1) ? (uint32_t*)hits1->ptr : nullptr;
  h.ids = (const uint32_t*)ids->ptr;
  h.texel_limit = texel_count;
  return fk::launch_hemisphere(ctx, s, h);
}

// Runs the counting variant and returns its first `n` counters (at most 8):
// box tests, triangle tests, then for the dynamic schedule the per-warp
// iteration profile (see fk_diag_traversal_profile).
static int diag_counts(fk_ctx* ctx, const fk_scene* s, const fk_buf* coords, const fk_buf* tidx, int kind,
                       const fk_sample_params* prm, const fk_buf* samples, uint32_t offset, uint32_t count,
                       int traverse, uint64_t* tests, int n) {
  if (!ctx || !s || !coords || !tidx || !prm || !samples || !tests)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_diag_traversal_counts: null argument");
  if (kind < FK_AO || kind > FK_AO_BN || prm->sample_count == 0 || prm->perm_count == 0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_diag_traversal_counts: bad kind or params");
  uint64_t end = (uint64_t)offset + count;
  if (!fits(coords, 16 * end) || !fits(tidx, 4 * end) || !fits(samples, 16ull * prm->sample_count * prm->perm_count))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_diag_traversal_counts: buffers too small");
  fk_buf *o0 = nullptr, *o1 = nullptr;
  unsigned long long* tally = nullptr;
  int rc = fk_buf_alloc(ctx, 12 * (end ? end : 1), &o0);
  if (rc == FK_OK) rc = fk_buf_alloc(ctx, 12 * (end ? end : 1), &o1);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&tally, 8 * sizeof(unsigned long long));
  if (rc == FK_OK && cudaMemsetAsync(tally, 0, 8 * sizeof(unsigned long long), ctx->stream) != cudaSuccess)
    rc = fk_fail(ctx, FK_ERR_CUDA, "fk_diag_traversal_counts: memset");
  if (rc == FK_OK && count) {
    fk::HemiLaunch h;
    h.kind = kind;
    h.spp = prm->sample_count;
    h.perms = prm->perm_count;
    h.min_d = prm->min_distance;
    h.max_d = prm->max_distance;
    h.samples = (const float4*)samples->ptr;
    h.coords = (const float4*)coords->ptr;
    h.tidx = (const uint32_t*)tidx->ptr;
    h.offset = offset;
    h.count = count;
    h.traverse = traverse;
    h.out0 = (float*)o0->ptr;
    h.out1 = (float*)o1->ptr;
    h.hits0 = h.hits1 = nullptr;
    h.tally = tally;
    rc = fk::launch_hemisphere(ctx, s, h);
  }
  unsigned long long host[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (rc == FK_OK && cudaMemcpyAsync(host, tally, sizeof(host), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
    rc = fk_fail(ctx, FK_ERR_CUDA, "fk_diag_traversal_counts: copy");
  if (rc == FK_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    rc = fk_fail(ctx, FK_ERR_CUDA, "fk_diag_traversal_counts: sync");
  for (int k = 0; k < n; ++k) tests[k] = host[k];
  if (o0) fk_buf_free(ctx, o0);
  if (o1) fk_buf_free(ctx, o1);
  fk_dev_free(ctx, tally);
  return rc;
}

int fk_diag_traversal_counts(fk_ctx* ctx, const fk_scene* s, const fk_buf* coords, const fk_buf* tidx, int kind,
                             const fk_sample_params* prm, const fk_buf* samples, uint32_t offset, uint32_t count,
                             int traverse, uint64_t* tests) {
  return diag_counts(ctx, s, coords, tidx, kind, prm, samples, offset, count, traverse, tests, 2);
}

int fk_diag_traversal_profile(fk_ctx* ctx, const fk_scene* s, const fk_buf* coords, const fk_buf* tidx, int kind,
                              const fk_sample_params* prm, const fk_buf* samples, uint32_t offset, uint32_t count,
                              int traverse, uint64_t* counters) {
  if ((traverse & FK_SCHEDULE_MASK) == FK_SCHEDULE_STATIC)
    return fk_fail(ctx, FK_ERR_UNSUPPORTED, "fk_diag_traversal_profile: dynamic schedule only");
  return diag_counts(ctx, s, coords, tidx, kind, prm, samples, offset, count, traverse, counters, 8);
}

int fk_gather(fk_ctx* ctx, const fk_scene* s, int kind, const fk_buf* coords, const fk_buf* tidx, uint32_t offset,
              uint32_t count, fk_buf* out) {
  if (!ctx || !s || !coords || !tidx || !out) return fk_fail(ctx, FK_ERR_INVALID, "fk_gather: null argument");
  uint64_t end = (uint64_t)offset + count;
  if (!fits(coords, 16 * end) || !fits(tidx, 4 * end) || !fits(out, (kind == FK_GATHER_HEIGHT ? 4 : 12) * end))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_gather: buffers too small");
  return fk::launch_gather(ctx, s, kind, (const float4*)coords->ptr, (const uint32_t*)tidx->ptr, offset, count,
                           (float*)out->ptr);
}

int fk_tangent_space(fk_ctx* ctx, const fk_texel_map* m, uint32_t offset, uint32_t count, fk_buf* io3) {
  if (!ctx || !m || !io3) return fk_fail(ctx, FK_ERR_INVALID, "fk_tangent_space: null argument");
  uint64_t end = (uint64_t)offset + count;
  if (end > m->count || !fits(io3, 12 * end)) return fk_fail(ctx, FK_ERR_INVALID, "fk_tangent_space: range outside the map");
  return fk::launch_tangent_space(ctx, m, offset, count, (float*)io3->ptr);
}

}  // extern "C"

// ==================================================================== MeshMapping
struct fk_meshmapping {
  fk_ctx* ctx = nullptr;
  const fk_texel_map* map = nullptr;
  fk_scene* scene = nullptr;
  bool owns_scene = false;
  fk_buf* coords = nullptr;
  fk_buf* tidx = nullptr;
  int cull = 1;
  uint32_t count = 0, work_count = 0, done = 0, per_step = 0;
  bool ready = false;
};

static void mm_release(fk_meshmapping* mm) {
  if (mm->coords) fk_buf_free(mm->ctx, mm->coords);
  if (mm->tidx) fk_buf_free(mm->ctx, mm->tidx);
  if (mm->owns_scene && mm->scene) fk_scene_free(mm->ctx, mm->scene);
  mm->coords = mm->tidx = nullptr;
  mm->scene = nullptr;
  mm->ready = false;
}

extern "C" {

int fk_meshmapping_create(fk_ctx* ctx, fk_meshmapping** out) {
  if (!ctx || !out) return FK_ERR_INVALID;
  *out = new (std::nothrow) fk_meshmapping();
  if (!*out) return FK_ERR_NOMEM;
  (*out)->ctx = ctx;
  return FK_OK;
}

static int mm_buffers(fk_meshmapping* mm) {
  fk_ctx* ctx = mm->ctx;
  mm->count = mm->map->count;
  mm->work_count = round_up(mm->count);
  size_t n = mm->work_count ? mm->work_count : kGroup;
  int rc = fk_buf_alloc(ctx, 16 * n, &mm->coords);
  if (rc == FK_OK) rc = fk_buf_alloc(ctx, 4 * n, &mm->tidx);
  if (rc != FK_OK) return rc;
  // Padding texels read as misses.
  FK_CUDA(ctx, cudaMemsetAsync(mm->tidx->ptr, 0xFF, 4 * n, ctx->stream));
  mm->done = 0;
  mm->ready = true;
  return FK_OK;
}

int fk_meshmapping_init_scene(fk_meshmapping* mm, const fk_texel_map* map, const fk_scene* scene, int cull) {
  if (!mm || !map || !scene) return fk_fail(mm ? mm->ctx : nullptr, FK_ERR_INVALID, "fk_meshmapping_init: null");
  mm_release(mm);
  mm->map = map;
  mm->scene = const_cast<fk_scene*>(scene);
  mm->owns_scene = false;
  mm->cull = cull ? 1 : 0;
  return mm_buffers(mm);
}

// MeshMapping::init (Src/meshmapping.cpp:128-184): fillMeshData, then upload.
int fk_meshmapping_init(fk_meshmapping* mm, const fk_texel_map* map, const fk_mesh* hipoly, const fk_bvh* bvh,
                        int cull) {
  if (!mm || !map || !hipoly || !bvh) return fk_fail(mm ? mm->ctx : nullptr, FK_ERR_INVALID, "fk_meshmapping_init: null");
  mm_release(mm);
  uint32_t nn = 0, nc = 0;
  int rc = fk_bvh_flatten_sizes(bvh, &nn, &nc);
  if (rc != FK_OK) return fk_fail(mm->ctx, rc, "fk_meshmapping_init: flatten");
  if (nn == 0 || nc == 0) return fk_fail(mm->ctx, FK_ERR_INVALID, "fk_meshmapping_init: high-poly mesh has no triangles");
  std::vector<fk_bvh_node> nodes(nn);
  std::vector<float> pos(4 * (size_t)nc), nrm(4 * (size_t)nc);
  rc = fk_bvh_flatten(bvh, hipoly, nodes.data(), pos.data(), nrm.data());
  if (rc != FK_OK) return fk_fail(mm->ctx, rc, "fk_meshmapping_init: flatten (mesh and BVH disagree)");
  rc = fk_scene_upload(mm->ctx, nodes.data(), nn, pos.data(), nrm.data(), nc, &mm->scene);
  if (rc != FK_OK) return rc;
  mm->owns_scene = true;
  mm->map = map;
  mm->cull = cull ? 1 : 0;
  return mm_buffers(mm);
}

int fk_meshmapping_set_work_per_step(fk_meshmapping* mm, uint32_t texels) {
  if (!mm) return FK_ERR_INVALID;
  mm->per_step = texels;
  return FK_OK;
}

// MeshMapping::runStep (Src/meshmapping.cpp:186-218).
int fk_meshmapping_run_step(fk_meshmapping* mm, int* done) {
  if (!mm) return FK_ERR_INVALID;
  if (!mm->ready) return fk_fail(mm->ctx, FK_ERR_STATE, "fk_meshmapping_run_step: not initialised");
  uint32_t left = mm->count - mm->done;
  uint32_t n = (mm->per_step && mm->per_step < left) ? mm->per_step : left;
  int rc = fk_meshmap(mm->ctx, mm->scene, mm->map, mm->cull, FLT_MAX, mm->done, n, mm->coords, mm->tidx);
  if (rc != FK_OK) return rc;
  mm->done += n;
  if (done) *done = mm->done >= mm->count;
  return FK_OK;
}

float fk_meshmapping_progress(const fk_meshmapping* mm) {
  if (!mm || !mm->ready) return 0.0f;
  return mm->count ? (float)mm->done / (float)mm->count : 1.0f;
}

int fk_meshmapping_results(fk_meshmapping* mm, float* coords4, uint32_t* tidx) {
  if (!mm || !mm->ready) return fk_fail(mm ? mm->ctx : nullptr, FK_ERR_STATE, "fk_meshmapping_results: not initialised");
  int rc = FK_OK;
  if (coords4) rc = fk_buf_download(mm->ctx, mm->coords, 0, coords4, 16 * (size_t)mm->work_count);
  if (rc == FK_OK && tidx) rc = fk_buf_download(mm->ctx, mm->tidx, 0, tidx, 4 * (size_t)mm->work_count);
  return rc;
}

const fk_buf* fk_meshmapping_coords(const fk_meshmapping* mm) { return mm ? mm->coords : nullptr; }
const fk_buf* fk_meshmapping_tidx(const fk_meshmapping* mm) { return mm ? mm->tidx : nullptr; }
const fk_scene* fk_meshmapping_scene(const fk_meshmapping* mm) { return mm ? mm->scene : nullptr; }

int fk_meshmapping_free(fk_meshmapping* mm) {
  if (!mm) return FK_ERR_INVALID;
  mm_release(mm);
  delete mm;
  return FK_OK;
}

}  // extern "C"

// ==================================================================== solvers
struct fk_solver {
  fk_ctx* ctx = nullptr;
  fk_solver_params p{};
  const fk_texel_map* map = nullptr;
  fk_meshmapping* mm = nullptr;
  fk_buf* result = nullptr;
  fk_buf* hits = nullptr;
  fk_buf* samples = nullptr;
  uint32_t count = 0, work_count = 0, done = 0, per_step = 0;
  bool ready = false;
};

static const uint32_t kPerms = 4096;  // k_samplePermCount (Src/solver_ao.cpp:34)

static bool sampling(int kind) {
  return kind == FK_SOLVER_AO || kind == FK_SOLVER_BENT_NORMALS || kind == FK_SOLVER_THICKNESS;
}
static uint32_t floats_per_texel(int kind) {
  return (kind == FK_SOLVER_POSITION || kind == FK_SOLVER_NORMALS || kind == FK_SOLVER_BENT_NORMALS) ? 3 : 1;
}

static void solver_release(fk_solver* s) {
  if (s->result) fk_buf_free(s->ctx, s->result);
  if (s->hits) fk_buf_free(s->ctx, s->hits);
  if (s->samples) fk_buf_free(s->ctx, s->samples);
  s->result = s->hits = s->samples = nullptr;
  s->ready = false;
}

extern "C" {

int fk_solver_create(fk_ctx* ctx, const fk_solver_params* p, fk_solver** out) {
  if (!ctx || !p || !out) return FK_ERR_INVALID;
  if (p->kind < FK_SOLVER_HEIGHT || p->kind > FK_SOLVER_THICKNESS)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_solver_create: unknown solver kind");
  if (sampling(p->kind) && p->sample_count == 0) return fk_fail(ctx, FK_ERR_INVALID, "fk_solver_create: zero samples");
  fk_solver* s = new (std::nothrow) fk_solver();
  if (!s) return FK_ERR_NOMEM;
  s->ctx = ctx;
  s->p = *p;
  *out = s;
  return FK_OK;
}

// XxxSolver::init (e.g. Src/solver_ao.cpp:36-68): sample table, result buffers.
int fk_solver_init(fk_solver* s, const fk_texel_map* map, fk_meshmapping* mm) {
  if (!s || !map || !mm) return fk_fail(s ? s->ctx : nullptr, FK_ERR_INVALID, "fk_solver_init: null");
  if (!mm->ready || mm->map != map) return fk_fail(s->ctx, FK_ERR_STATE, "fk_solver_init: mesh mapping not initialised on this map");
  solver_release(s);
  s->map = map;
  s->mm = mm;
  s->count = map->count;
  s->work_count = round_up(s->count);
  size_t n = s->work_count ? s->work_count : kGroup;
  int rc = fk_buf_alloc(s->ctx, 4 * floats_per_texel(s->p.kind) * n, &s->result);
  if (rc != FK_OK) return rc;
  if (sampling(s->p.kind)) {
    rc = fk_buf_alloc(s->ctx, 4 * n, &s->hits);
    if (rc != FK_OK) return rc;
    std::vector<float> table(4 * (size_t)s->p.sample_count * kPerms);
    fk_samples_cosine(s->p.sample_count, kPerms, s->p.seed, table.data());
    rc = fk_buf_alloc(s->ctx, 4 * table.size(), &s->samples);
    if (rc == FK_OK) rc = fk_buf_upload(s->ctx, s->samples, 0, table.data(), 4 * table.size());
    if (rc != FK_OK) return rc;
  }
  s->done = 0;
  s->ready = true;
  return FK_OK;
}

int fk_solver_set_work_per_step(fk_solver* s, uint32_t texels) {
  if (!s) return FK_ERR_INVALID;
  s->per_step = texels;
  return FK_OK;
}

// XxxSolver::runStep: one chunk of texels through the solver's kernels.
int fk_solver_run_step(fk_solver* s, int* done) {
  if (!s) return FK_ERR_INVALID;
  if (!s->ready) return fk_fail(s->ctx, FK_ERR_STATE, "fk_solver_run_step: not initialised");
  if (s->mm->done < s->mm->count) return fk_fail(s->ctx, FK_ERR_STATE, "fk_solver_run_step: mesh mapping unfinished");
  uint32_t left = s->count - s->done;
  uint32_t n = (s->per_step && s->per_step < left) ? s->per_step : left;
  const fk_scene* sc = s->mm->scene;
  int rc = FK_OK;
  switch (s->p.kind) {
    case FK_SOLVER_HEIGHT:
      rc = fk_gather(s->ctx, sc, FK_GATHER_HEIGHT, s->mm->coords, s->mm->tidx, s->done, n, s->result);
      break;
    case FK_SOLVER_POSITION:
      rc = fk_gather(s->ctx, sc, FK_GATHER_POSITION, s->mm->coords, s->mm->tidx, s->done, n, s->result);
      break;
    case FK_SOLVER_NORMALS:
      rc = fk_gather(s->ctx, sc, FK_GATHER_NORMAL, s->mm->coords, s->mm->tidx, s->done, n, s->result);
      if (rc == FK_OK && s->p.tangent_space) rc = fk_tangent_space(s->ctx, s->map, s->done, n, s->result);
      break;
    default: {
      fk_sample_params sp{s->p.sample_count, kPerms, s->p.min_distance, s->p.max_distance};
      int kind = s->p.kind == FK_SOLVER_AO ? FK_AO : (s->p.kind == FK_SOLVER_BENT_NORMALS ? FK_BN : FK_THICK);
      rc = fk_hemisphere(s->ctx, sc, s->mm->coords, s->mm->tidx, kind, &sp, s->samples, s->done, n, s->p.traverse,
                         s->result, nullptr, s->hits, nullptr);
      if (rc == FK_OK && kind == FK_BN && s->p.tangent_space) rc = fk_tangent_space(s->ctx, s->map, s->done, n, s->result);
    }
  }
  if (rc != FK_OK) return rc;
  s->done += n;
  if (done) *done = s->done >= s->count;
  return FK_OK;
}

float fk_solver_progress(const fk_solver* s) {
  if (!s || !s->ready) return 0.0f;
  return s->count ? (float)s->done / (float)s->count : 1.0f;
}

size_t fk_solver_result_count(const fk_solver* s) {
  return s && s->ready ? (size_t)floats_per_texel(s->p.kind) * s->work_count : 0;
}

int fk_ctx_check(fk_ctx* ctx) {
  if (!ctx) return FK_ERR_INVALID;
  int st = 0;
  FK_CUDA(ctx, cudaMemcpyAsync(&st, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  FK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!st) return FK_OK;
  cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream);
  std::string msg;
  if (st & 1) msg += "a traversal exceeded its stack; ";
  if (st & 2) msg += "a texel names a triangle outside the scene; ";
  if (st & 4) msg += "a texel list holds an id beyond texel_count; ";
  if (st & 8) msg += "a training batch names a row beyond n_rows; ";
  if (st & 16) msg += "a tensor-core wait of the denoiser ran out; ";
  msg += "results are incomplete";
  return fk_fail(ctx, FK_ERR_DEVICE, msg.c_str());
}

// getResults (e.g. Src/solver_ao.cpp:70-75): the whole padded result buffer.
int fk_solver_results(fk_solver* s, float* out, size_t floats) {
  if (!s || !out) return FK_ERR_INVALID;
  if (!s->ready) return fk_fail(s->ctx, FK_ERR_STATE, "fk_solver_results: not initialised");
  size_t n = fk_solver_result_count(s);
  if (floats < n) return fk_fail(s->ctx, FK_ERR_INVALID, "fk_solver_results: host buffer too small");
  int rc = fk_ctx_check(s->ctx);
  if (rc != FK_OK) return rc;
  return fk_buf_download(s->ctx, s->result, 0, out, 4 * n);
}

int fk_solver_hits(fk_solver* s, uint32_t* out, size_t count) {
  if (!s || !out) return FK_ERR_INVALID;
  if (!s->ready || !s->hits) return fk_fail(s->ctx, FK_ERR_STATE, "fk_solver_hits: not a sampling solver");
  if (count > s->work_count) count = s->work_count;
  return fk_buf_download(s->ctx, s->hits, 0, out, 4 * count);
}

const fk_buf* fk_solver_result_buffer(const fk_solver* s) { return s ? s->result : nullptr; }

int fk_solver_free(fk_solver* s) {
  if (!s) return FK_ERR_INVALID;
  solver_release(s);
  delete s;
  return FK_OK;
}

}  // extern "C"
