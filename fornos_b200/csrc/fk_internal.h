// Internal host-side structures shared by the translation units of
// libfornos_b200.so.  Not part of the ABI (include/fornos_gpu.h is).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/fornos_gpu.h"

// ------------------------------------------------------------------ context
struct fk_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // fk_bake's result copies, beside the stream's work (made on first use)
  std::string err;
  uint64_t launches = 0;
  uint32_t* counters = nullptr;   // device work-queue counters for persistent kernels
  uint32_t counter_slots = 0;
  uint32_t next_counter = 0;
  int* status = nullptr;          // device status word (limits a kernel could not honour)
  void* scratch = nullptr;        // see fk_scratch
  // Stream-ordered pool behind every device allocation of the library; it
  // keeps freed memory (release threshold: all), so repeated uploads and
  // bakes reuse it instead of mapping and unmapping pages (fk_ctx_trim).
  cudaMemPool_t pool = nullptr;
  size_t scratch_bytes = 0;
  // Pinned host memory the scene upload lays the node arrays out in (kept
  // between uploads, released by fk_ctx_trim); stage_done is recorded after
  // the copies that read it, and the next upload waits for it.
  void* stage = nullptr;
  size_t stage_bytes = 0;
  cudaEvent_t stage_done = nullptr;
  fk_tuning tuning = {20, 8, 1, FK_RAY_ORDER_SECTOR, 0, FK_L2_NONE, 256, 64};  // fk_ctx_set_tuning
  // Persisting L2 set-aside (fk_tuning.l2_persist): the device's limit before
  // the context raised it, restored when the knob is turned off or the
  // context is destroyed.
  bool l2_raised = false;
  size_t l2_prev_limit = 0;
  std::set<fk_buf*> bufs;
  std::set<fk_scene*> scenes;
  std::set<fk_texel_map*> maps;
};

struct fk_buf {
  fk_ctx* ctx = nullptr;
  void* ptr = nullptr;
  size_t bytes = 0;
};

// High-poly mesh + BVH on the device.
struct fk_scene {
  fk_ctx* ctx = nullptr;
  uint32_t node_count = 0, corner_count = 0, depth = 0, leaf_count = 0;
  // Reference layout, one entry per flattened node (skip-pointer walk):
  float4* node_lo = nullptr;     // aabbMin.xyz, start (bits)
  float4* node_hi = nullptr;     // aabbMax.xyz, end (bits)
  float4* node_box = nullptr;    // node_lo[i], node_hi[i] side by side (one 32-byte sector), for the leaf phase
  uint32_t* node_jump = nullptr;
  float4* pos4 = nullptr;        // triangle corners, DFS leaf order
  float4* nrm4 = nullptr;
  // Ordered layout: one 64-byte record per inner node holding both children's
  // boxes (4 x float4), and one 64-byte precomputed record per triangle.
  float4* wide = nullptr;
  uint32_t wide_count = 0;
  uint32_t odepth = 0;           // levels of the ordered layouts' tree (the reference's, or a rebuilt one)
  int tree = 0;                  // FK_TREE_*: which inner tree wide / wide4 point into
  // Both inner trees' arrays once built, kept until the scene is freed (a
  // batch's job table may hold either): [FK_TREE_REFERENCE], [FK_TREE_SAH].
  float4* tree_wide[2] = {nullptr, nullptr};
  float4* tree_wide4[2] = {nullptr, nullptr};
  uint32_t tree_count[2] = {0, 0}, tree_count4[2] = {0, 0}, tree_depth[2] = {0, 0}, tree_depth4[2] = {0, 0};
  // Collapsed layout: 128-byte 4-wide nodes over the same leaves.
  float4* wide4 = nullptr;
  uint32_t wide4_count = 0, depth4 = 0;
  float4* tri_rec = nullptr;
  // The first inner records of the active 2-wide tree in breadth-first order
  // (fk_tuning.top_records), staged in shared memory by the ordered
  // traversal; a child ref >= wide_count names staged record ref - wide_count.
  // Built on first use for (top_tree, top_want).
  float4* top = nullptr;
  uint32_t top_count = 0, top_want = 0;
  int top_tree = -1;
  uint32_t root_is_leaf = 0;
  uint32_t filter_ok = 0;        // every coordinate below 2^24 in magnitude, box faces in order
  size_t bytes = 0;
};

struct fk_texel_map {
  fk_ctx* ctx = nullptr;
  uint32_t width = 0, height = 0, count = 0;
  float4* pix = nullptr;     // 2 float4 per texel: p, d
  float4* pixt = nullptr;    // 3 float4 per texel: n, t, b
  uint32_t* indices = nullptr;
};

namespace fk {
int texel_map_upload_async(fk_ctx* ctx, uint32_t w, uint32_t h, uint32_t count, const float* pix8,
                           const float* pixt12, const uint32_t* idx, fk_texel_map** out);
}

// ------------------------------------------------------------------ helpers
int fk_fail(fk_ctx* ctx, int code, const std::string& msg);
int fk_cuda_fail(fk_ctx* ctx, cudaError_t e, const char* what);

#define FK_CUDA(ctx, call)                                   \
  do {                                                       \
    cudaError_t fk_e_ = (call);                              \
    if (fk_e_ != cudaSuccess) return fk_cuda_fail((ctx), fk_e_, #call); \
  } while (0)

// Checks a launch just issued on ctx->stream and counts it.
int fk_after_launch(fk_ctx* ctx, const char* what);

// Device memory owned by the library (not visible as fk_buf): taken from the
// context's pool in the order of ctx->stream and given back in that order.
int fk_dev_alloc(fk_ctx* ctx, void** p, size_t bytes);
void fk_dev_free(fk_ctx* ctx, void* p);
// fk_buf_free for buffers used on ctx->stream only: no device-wide wait.
extern "C" int fk_buf_release(fk_ctx* ctx, fk_buf* b);

// Reserves a zeroed device counter for one persistent-kernel launch.
uint32_t* fk_take_counter(fk_ctx* ctx);

// Context-owned device scratch of at least `bytes` (grown on demand, kept for
// later calls; growing waits for the stream).  Null on allocation failure.
void* fk_scratch(fk_ctx* ctx, size_t bytes);

// Kernel launchers (fk_*.cu).
namespace fk {

// Device view of a scene, passed to kernels by value or kept in shared memory.
struct SceneDev {
  const float4* __restrict__ node_lo;
  const float4* __restrict__ node_hi;
  const float4* __restrict__ node_box;  // node_lo[i], node_hi[i] at 2 i, 2 i + 1
  const uint32_t* __restrict__ node_jump;
  const float4* __restrict__ pos4;
  const float4* __restrict__ nrm4;
  const float4* __restrict__ wide;
  const float4* __restrict__ wide4;
  // Triangle records in two blocks: rec[t] = (n, a.n), read by every
  // triangle test; rec_bary[3 t .. 3 t + 2] = (a, d01), (v0, d00), (v1, d11),
  // read only for hits inside the distance range.
  const float4* __restrict__ rec;
  const float4* __restrict__ rec_bary;
  uint32_t node_count;
  uint32_t root_is_leaf;
  uint32_t corner_count;
  uint32_t filter_ok;  // scene coordinates small enough for the filtered box test
};
SceneDev scene_dev(const fk_scene* s);

// Deepest collapsed (4-wide) tree the 4-wide traversal accepts: it defers at
// most 3 entries per level within its 64-entry stack.
constexpr uint32_t kMaxOrdered4Depth = 21;
// Deepest 2-wide tree the ordered traversal accepts.
constexpr uint32_t kMaxOrderedDepth = 48;

// Inner-tree layouts (fk_tree.cpp).  2-wide records: 4 float4 per inner node,
// child boxes, refs (record index, or -(flattened leaf index + 1)) and leaf
// triangle counts; root record 0.  build_sah_wide rebuilds them over the
// leaves of a flattened node array with a binned surface-area split and
// returns the tree's depth (root = 1, counting the leaf level).
uint32_t build_sah_wide(const float4* lo, const float4* hi, const uint32_t* jump, uint32_t nn,
                        std::vector<float4>& wide);
void collapse_wide4(const std::vector<float4>& wide, std::vector<float4>& wide4, uint32_t& n4, uint32_t& depth4);
// BVH::createBinary + fillMeshData on the device (fk_bvh_dev.cu): the
// flattened nodes (scene layout: lo / hi float4 with start / end bits, jump)
// and corner arrays of fk_bvh_build + fk_bvh_flatten, bit for bit, in
// library-owned device memory.
struct DevBvh {
  float4* lo = nullptr;
  float4* hi = nullptr;
  uint32_t* jump = nullptr;
  float4* pos4 = nullptr;
  float4* nrm4 = nullptr;
  uint32_t node_count = 0, corner_count = 0, triangle_count = 0;
};
int build_bvh_device(fk_ctx* ctx, const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, DevBvh* out);
// *ok: every coordinate of the n corners is below lim in magnitude.
int corners_below(fk_ctx* ctx, const float4* p, uint32_t n, float lim, bool* ok);

// The same tree built on the device (fk_sah.cu) from the scene's node boxes
// and its leaves' flattened indices (ascending): *wide gets 4 (L - 1) float4
// records, or stays null when the tree would be deeper than
// kMaxOrderedDepth (*depth then exceeds it); depth 1 for a single leaf.
int build_sah_device(fk_ctx* ctx, const float4* node_lo, const float4* node_hi, const std::vector<uint32_t>& leaves,
                     float4** wide, uint32_t* depth);
// The scene's 4-wide layout for its active tree, built on first use.
int ensure_wide4(fk_ctx* ctx, fk_scene* s);
// The scene's staged top records for `want` records of its active tree
// (fk_scene::top), built on first use.
int ensure_top(fk_ctx* ctx, fk_scene* s, uint32_t want);
// Raises the device's persisting L2 set-aside for a window of `bytes` (once
// per context) and gives the window's hit ratio; restore_l2 undoes it.
int raise_l2(fk_ctx* ctx, size_t bytes, float* hit_ratio);
void restore_l2(fk_ctx* ctx);

// One job of a batched hemisphere launch (device-side job table entry).
static constexpr uint32_t kMaxBatchJobs = 64;
struct BatchJobDev {
  SceneDev s;
  const float4* samples;
  const float4* coords;
  const uint32_t* tidx;
  float* out0;
  float* out1;
  uint32_t* hits0;
  uint32_t* hits1;
  unsigned long long ray_base;  // first ray of the job in the batch's ray space
  uint32_t texel_base;          // first texel of the job in the batch's texel space
  uint32_t texels, spp, perms;
  float lo, hi;
  // the job's place in the batch's concatenated scene arrays (BatchArgs::cat)
  uint32_t node_base, corner_base;  // flattened nodes; corners (a multiple of 3)
  int32_t root2, root4;             // root records of the 2-wide and 4-wide layouts
  uint32_t pad[2];
};
struct BatchArgs {
  // Every job's scene laid end to end: node, corner and triangle-record
  // arrays, and both inner layouts, with the jobs' child refs, leaf refs,
  // triangle ranges and skip pointers offset to the concatenated arrays, so a
  // traversal needs no per-job pointers.
  SceneDev cat;
  const BatchJobDev* jobs;
  uint32_t njobs;
  unsigned long long r0, r1;  // rays of this launch
  uint32_t t0, t1;            // texels folded by this launch
  unsigned long long stride;  // trace every stride-th ray (calibration), 1 otherwise
  float* scratch;             // one distance per traced ray, indexed from r0 / stride
  unsigned long long* queue;  // zeroed before the launch
  int* status;
  uint32_t refill, leaf_batch;
  uint32_t ray_order;  // FK_RAY_ORDER_*, per job (stride 1 only)
  uint32_t speculate;  // lanes holding a leaf keep visiting inner records
};
cudaError_t launch_batch(const BatchArgs& a, int kind, int trav, bool filter, cudaStream_t stream, int sm_count,
                         bool reduce);
// Copies scene `s` into the concatenated arrays of `cat` at the given bases
// (nodes, corners, 2-wide and 4-wide records), offsetting its refs.
int concat_batch_scene(cudaStream_t st, const fk_scene* s, uint32_t node_base, uint32_t corner_base, uint32_t rec2,
                       uint32_t rec4, const SceneDev& cat);
int launch_meshmap(fk_ctx* ctx, const fk_scene* s, const fk_texel_map* m, int cull, float max_d, uint32_t offset,
                   uint32_t count, float4* coords, uint32_t* tidx);
struct HemiLaunch {
  int kind;
  uint32_t spp, perms;
  float min_d, max_d;
  const float4* samples;
  const float4* coords;
  const uint32_t* tidx;
  uint32_t offset, count;
  int traverse;
  float* out0;
  float* out1;
  uint32_t* hits0;
  uint32_t* hits1;
  unsigned long long* tally = nullptr;  // non-null: counting variant
  uint32_t refill = 0;                  // dynamic schedule: idle lanes that trigger a refill (0 = context tuning)
  uint32_t leaf_batch = 0;              // postponed leaves that start a leaf phase (0 = context tuning)
  uint32_t speculate = 0;
  // Texel list (dynamic schedule only): ray texel g is texel ids[g] for the
  // mapping inputs, the sample permutation and the outputs; ids at or above
  // texel_limit are skipped and flag status bit 4.
  const uint32_t* ids = nullptr;
  uint32_t texel_limit = 0;
  // Per-ray distances in this buffer of scratch_rays floats instead of the
  // context's scratch (which may have to grow); at least one texel's rays.
  float* scratch = nullptr;
  unsigned long long scratch_rays = 0;
};
int launch_hemisphere(fk_ctx* ctx, const fk_scene* s, const HemiLaunch& h);
// Same kernels over caller-provided scratch: `dist` holds count x spp floats,
// `queue` and `status` are zeroed words.  Allocates nothing.
int launch_hemisphere_external(const fk_scene* s, const HemiLaunch& h, cudaStream_t stream, int sm_count,
                               const fk_tuning& tun, float* dist, uint32_t* queue, int* status, std::string& err);
int launch_gather(fk_ctx* ctx, const fk_scene* s, int kind, const float4* coords, const uint32_t* tidx,
                  uint32_t offset, uint32_t count, float* out);
int launch_tangent_space(fk_ctx* ctx, const fk_texel_map* m, uint32_t offset, uint32_t count, float* io3);
int launch_tri_records(fk_ctx* ctx, fk_scene* s);
// Fills box[2 i], box[2 i + 1] = lo[i], hi[i] for i < n on `stream`.
cudaError_t pair_node_boxes(cudaStream_t stream, const float4* lo, const float4* hi, uint32_t n, float4* box);
struct RasterTri;  // defined in fk_raster.cu

// Learned denoiser: parameter layout (fp32, row-major) and kernel launchers.
namespace dn {
constexpr int kInputs = 250, kK1 = 256, kHidden = 64, kOut = 4, kRows = 128;
constexpr int kW1 = 0;                        // [64][256], columns 250..255 zero
constexpr int kB1 = kW1 + kHidden * kK1;      // [64]
constexpr int kW2 = kB1 + kHidden;            // [64 out][64 in]
constexpr int kB2 = kW2 + kHidden * kHidden;  // [64]
constexpr int kW3 = kB2 + kHidden;            // [4 out][64 in]
constexpr int kB3 = kW3 + kOut * kHidden;     // [4]
constexpr int kParams = kB3 + kOut;
}  // namespace dn
// fp32 parameters (biases are read from here) and bf16 working copies:
// w1 [64][256], w2 [64][64] (out, in), w2t (in, out), w3 [8][64] (rows 4..7
// zero), w3t [64][8].
struct DnWeights {
  const float* params;
  const void *w1, *w2, *w2t, *w3, *w3t;
};
namespace dn {
size_t train_smem_bytes();
size_t apply_smem_bytes();
cudaError_t launch_features(cudaStream_t st, uint32_t n, uint32_t w, uint32_t h, const uint32_t* indices,
                            const uint32_t* tidx, const float4* coords, const float* ao, const float* bn3,
                            const float* pos3, const float* nrm3, float max_d, float4* image);
cudaError_t launch_rows(cudaStream_t st, const float4* image, uint32_t w, uint32_t h, const uint32_t* pixels,
                        uint32_t n, uint32_t* rows);
cudaError_t launch_train(cudaStream_t st, const uint32_t* rows, const float4* targets, const uint32_t* row_ids,
                         uint32_t nrows, uint32_t offset, uint32_t batch, const DnWeights& wt, float* partials,
                         float* loss, int* status);
cudaError_t launch_adam(cudaStream_t st, const float* partials, uint32_t tiles, float* params, float* m, float* v,
                        float* grad_out, int update, float lr, float beta1, float beta2, float eps, float c1, float c2,
                        const DnWeights& wt);
cudaError_t launch_refresh(cudaStream_t st, const DnWeights& wt);
cudaError_t launch_apply(cudaStream_t st, int sm_count, const float4* image, uint32_t w, uint32_t h,
                         const uint32_t* indices, const uint32_t* tidx, const float* ao_in, const float* bn_in,
                         uint32_t offset, uint32_t count, const DnWeights& wt, float* ao_out, float* bn_out,
                         const uint32_t* rows, float4* y_out);
// The same inference on tcgen05 / tensor memory (status bit 16: a bounded wait ran out).
cudaError_t launch_apply_tc(cudaStream_t st, int sm_count, const float4* image, uint32_t w, uint32_t h,
                            const uint32_t* indices, const uint32_t* tidx, const float* ao_in, const float* bn_in,
                            uint32_t offset, uint32_t count, const DnWeights& wt, float* ao_out, float* bn_out,
                            const uint32_t* rows, float4* y_out, int* status);
cudaError_t launch_inverse(cudaStream_t st, uint32_t n, const uint32_t* indices, uint32_t pixels, uint32_t* inv);
cudaError_t launch_verify_slots(cudaStream_t st, uint32_t w, uint32_t h, uint32_t tile, uint32_t cells,
                                const uint32_t* inv, const uint32_t* tidx, uint32_t* slots);
cudaError_t launch_tile_error(cudaStream_t st, uint32_t tiles, uint32_t per, const uint32_t* slots, const float* ao_d,
                              const float* bn_d, const float* ao_v, const float* bn_v, float* err);
cudaError_t launch_fallback_list(cudaStream_t st, uint32_t n, uint32_t w, uint32_t tile, const uint32_t* indices,
                                 const uint32_t* tidx, const uint8_t* failed, uint32_t* list, uint32_t* count);
}  // namespace dn
}  // namespace fk

// Host mesh (Src/mesh.h:35-63).
struct fk_mesh {
  std::vector<float> positions, texcoords, normals, tangents, bitangents;
  std::vector<uint32_t> vertices, triangles;
  uint32_t position_count() const { return (uint32_t)(positions.size() / 3); }
  uint32_t vertex_count() const { return (uint32_t)(vertices.size() / 3); }
  uint32_t triangle_count() const { return (uint32_t)(triangles.size() / 3); }
};

// Host BVH tree (Src/bvh.h:32-46).
struct fk_bvh_tree_node {
  float c[3], s[3];            // center, half size (Src/math.h:147-154)
  int32_t kid[2] = {-1, -1};
  uint32_t first = 0, count = 0;  // triangle range in fk_bvh::order (leaves)
  uint64_t subtree = 0;
};
struct fk_bvh {
  std::vector<fk_bvh_tree_node> nodes;  // nodes[0] = root
  std::vector<uint32_t> order;          // triangle ids, leaf ranges contiguous
  uint32_t triangle_count = 0;
};
