// fk_hemisphere_noalloc: hemisphere sampling that allocates nothing.
//
// fk_hemisphere keeps its per-ray distances in context scratch that it grows
// with cudaMalloc.  Some callers cannot allow that: a host that runs one bake
// chunk per interactive frame (as the Fornos UI does, one runStep per frame),
// or an application that budgets all GPU memory through its own allocator.
// For them, cudaMalloc / cudaFree stall the frame (they synchronise the device)
// and can fail mid-bake under memory pressure.  This entry point instead uses
// one fixed array compiled into the library (a file-scope __device__ array,
// FK_NOALLOC_MAX_RAYS distances plus two control words).  Every GPU that loads
// the library holds that array until the process exits.
//
// Host code cannot pass the array's name to a kernel: on the host that name is
// only a stand-in, not a device address.  The device address is obtained once
// per device with cudaGetSymbolAddress, with that device current, on the first
// call made on that device, and kept for the life of the process (a device
// reset after that call is not supported: it also ends the context the scene
// belongs to).  All calls share the one array, which keeps whatever the last
// call left in it: the queue word is cleared at the start of each call (the
// distance slots are always written before they are read), and calls whose
// work overlaps on the GPU (different streams, or threads on one device
// without ordering) race on it and must be serialised by the caller.  Device
// errors (a traversal that overflowed its stack, a texel naming a triangle
// outside the scene) go to the context's own status word, which already
// exists, so fk_ctx_check reports them as it does for fk_hemisphere.
#include <mutex>
#include <string>

#include "fk_internal.h"

namespace {

constexpr uint32_t kMaxRays = FK_NOALLOC_MAX_RAYS;
constexpr size_t kWords = 64;  // control area after the distances: queue word, padding
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_scratch[kMaxRays + kWords];

std::mutex g_mutex;
void* g_address[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (which must be current).
cudaError_t scratch_address(int device, float** out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_address[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_address[device] = p;
  }
  *out = (float*)g_address[device];
  return cudaSuccess;
}

}  // namespace

extern "C" int fk_hemisphere_noalloc(const fk_scene* scene, const float* coords4, const uint32_t* tidx, int kind,
                                     const fk_sample_params* prm, const float* samples4, uint32_t offset,
                                     uint32_t count, int traverse, float* out0, float* out1, uint32_t* hits0,
                                     uint32_t* hits1, void* stream) {
  if (!scene) return FK_ERR_INVALID;
  fk_ctx* ctx = scene->ctx;
  if (!coords4 || !tidx || !prm || !samples4 || !out0 || (kind == FK_AO_BN && !out1))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_noalloc: null argument");
  if (kind < FK_AO || kind > FK_AO_BN) return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_noalloc: unknown kind");
  if (prm->sample_count == 0 || prm->perm_count == 0)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_noalloc: zero samples");
  if ((traverse & ~(FK_TRAVERSE_MASK | FK_SCHEDULE_MASK | FK_EXACT_BOX_TESTS)) ||
      (traverse & FK_TRAVERSE_MASK) > FK_TRAVERSE_SKIP)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_noalloc: unknown traversal");
  const uint64_t rays = (uint64_t)count * prm->sample_count;
  if (rays > kMaxRays)
    return fk_fail(ctx, FK_ERR_INVALID,
                   "fk_hemisphere_noalloc: " + std::to_string(count) + " texels x " +
                       std::to_string(prm->sample_count) + " samples = " + std::to_string(rays) +
                       " rays exceeds the fixed scratch of " + std::to_string(kMaxRays) +
                       " rays; split the texel range over several calls");
  if (count == 0) return FK_OK;
  int device = -1;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "cudaGetDevice");
  if (device != ctx->device || device >= kMaxDevices)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere_noalloc: the scene's device must be the current device");
  float* scratch = nullptr;
  e = scratch_address(device, &scratch);
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "cudaGetSymbolAddress");
  uint32_t* words = (uint32_t*)(scratch + kMaxRays);
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(words, 0, sizeof(uint32_t), st);  // the queue starts at zero
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "cudaMemsetAsync");
  fk::HemiLaunch h;
  h.kind = kind;
  h.spp = prm->sample_count;
  h.perms = prm->perm_count;
  h.min_d = prm->min_distance;
  h.max_d = prm->max_distance;
  h.samples = (const float4*)samples4;
  h.coords = (const float4*)coords4;
  h.tidx = tidx;
  h.offset = offset;
  h.count = count;
  h.traverse = traverse;
  h.out0 = out0;
  h.out1 = kind == FK_AO_BN ? out1 : nullptr;
  h.hits0 = hits0;
  h.hits1 = kind == FK_AO_BN ? hits1 : nullptr;
  std::string err;
  int rc = fk::launch_hemisphere_external(scene, h, st, ctx->sm_count, ctx->tuning, scratch, words, ctx->status,
                                          err);
  if (rc != FK_OK) return fk_fail(ctx, rc, "fk_hemisphere_noalloc: " + err);
  return FK_OK;
}
