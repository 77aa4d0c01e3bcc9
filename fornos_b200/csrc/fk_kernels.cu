// Ray kernels of the bake path, sm_100a:
//   * per-triangle records            (precomputed terms of the ray/triangle test)
//   * mesh mapping                    Shaders/meshmapping_nobackfaces.comp, meshmapping.comp
//   * hemisphere sampling             Shaders/ao_step0/1/2, bentnormals_step1/2, thick_step1/2
//   * gathers and tangent space       Shaders/heights, positions, normals, tangentspace
//
// Every comparison and every float the shaders produce is reproduced with the
// same IEEE operations in the same order (fk_device.cuh), so hit identity,
// occluder counts and sums match the reference bit for bit.  Two traversals:
//   SKIP    the reference's skip-pointer walk over the flattened node array,
//           in array order (exact by construction);
//   ORDERED near-first stack traversal over a children-in-parent BVH2 layout
//           (64-byte records, both child boxes per 128-bit loads), with the
//           reference's pruning rule (entry distance < min(best, max)).  It
//           visits the same leaves the reference can improve from, so results
//           agree except where a triangle's hit distance rounds below its own
//           leaf box's entry distance (grazing hits on box faces).
#include <cuda_runtime.h>

#include <algorithm>

#include "fk_device.cuh"
#include "fk_internal.h"

namespace fk {

// A hit index read from a caller's buffer: a miss, or the first corner of a
// triangle inside the scene.  Anything else is reported and treated as a miss.
__device__ __forceinline__ bool valid_hit(uint32_t id, uint32_t corners) {
  return id % 3 == 0 && id < corners;
}

static SceneDev dev_of(const fk_scene* s) {
  SceneDev d;
  d.node_lo = s->node_lo;
  d.node_hi = s->node_hi;
  d.node_box = s->node_box;
  d.node_jump = s->node_jump;
  d.pos4 = s->pos4;
  d.nrm4 = s->nrm4;
  d.wide = s->wide;
  d.wide4 = s->wide4;
  d.rec = s->tri_rec;
  d.rec_bary = s->tri_rec + s->corner_count / 3;
  d.node_count = s->node_count;
  d.root_is_leaf = s->root_is_leaf;
  d.corner_count = s->corner_count;
  d.filter_ok = s->filter_ok;
  return d;
}

__device__ __forceinline__ uint32_t as_u32(float f) { return __float_as_uint(f); }

// ------------------------------------------------------------------ records
// Per triangle (a, b, c): n = normalize(cross(b - a, c - a)) and dot(a, n) as
// Shaders/ao_step1.comp:73-77 computes them, plus the barycentric terms of
// :54-62.  Two blocks (SceneDev::rec, rec_bary): (n, a.n) of every triangle,
// then (a, d01), (v0, d00), (v1, d11) of every triangle.  Every triangle test
// reads the first, a leaf's triangles' planes being 16 bytes apart; only hits
// inside the distance range read the second.
__global__ void tri_records_kernel(const float4* __restrict__ pos4, float4* __restrict__ rec, uint32_t ntri) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  f3 a = xyz(pos4[3 * (size_t)t]), b = xyz(pos4[3 * (size_t)t + 1]), c = xyz(pos4[3 * (size_t)t + 2]);
  f3 v0 = sub(b, a), v1 = sub(c, a);
  f3 n = normalize(cross(v0, v1));
  float an = dot(a, n);
  float4* bary = rec + ntri;
  rec[t] = make_float4(n.x, n.y, n.z, an);
  bary[3 * (size_t)t + 0] = make_float4(a.x, a.y, a.z, dot(v0, v1));
  bary[3 * (size_t)t + 1] = make_float4(v0.x, v0.y, v0.z, dot(v0, v0));
  bary[3 * (size_t)t + 2] = make_float4(v1.x, v1.y, v1.z, dot(v1, v1));
}

__global__ void pair_boxes_kernel(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                                  float4* __restrict__ box) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  box[2 * (size_t)i] = lo[i];
  box[2 * (size_t)i + 1] = hi[i];
}

cudaError_t pair_node_boxes(cudaStream_t stream, const float4* lo, const float4* hi, uint32_t n, float4* box) {
  if (n) pair_boxes_kernel<<<(n + 255) / 256, 256, 0, stream>>>(lo, hi, n, box);
  return cudaGetLastError();
}

int launch_tri_records(fk_ctx* ctx, fk_scene* s) {
  uint32_t nt = s->corner_count / 3;
  tri_records_kernel<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(s->pos4, s->tri_rec, nt);
  return fk_after_launch(ctx, "tri_records_kernel");
}

// ------------------------------------------------------------------ sampling test
// Shaders/ao_step1.comp:71-92 followed by the range test of :100-105: returns
// true and lowers `best` when the triangle is hit at t in [lo, best).  The
// barycentric part only runs for hits inside the range (rejecting earlier
// cannot change which t survive).
__device__ __forceinline__ void tri_sample(const SceneDev& s, uint32_t t, f3 o, f3 d, float lo, float& best) {
  float4 A = __ldg(s.rec + t);
  f3 n = xyz(A);
  float nd = dot(d, n);
  if (!(fabsf(nd) > 0.0f)) return;
  float pn = dot(o, n);
  float th = __fdiv_rn(__fsub_rn(A.w, pn), nd);
  if (!(th >= 0.0f && th >= lo && th < best)) return;
  float4 B = __ldg(s.rec_bary + 3 * (size_t)t);
  float4 C = __ldg(s.rec_bary + 3 * (size_t)t + 1);
  float4 D = __ldg(s.rec_bary + 3 * (size_t)t + 2);
  f3 p = add(o, scale(d, th));
  f3 v2 = sub(p, xyz(B));
  float d20 = dot(v2, xyz(C)), d21 = dot(v2, xyz(D));
  float d00 = C.w, d01 = B.w, d11 = D.w;
  float den = __fsub_rn(__fmul_rn(d00, d11), __fmul_rn(d01, d01));
  const float ny = __fsub_rn(__fmul_rn(d11, d20), __fmul_rn(d01, d21));
  const float nz = __fsub_rn(__fmul_rn(d00, d21), __fmul_rn(d01, d20));
  float y = __fdiv_rn(ny, den);
  float z = __fdiv_rn(nz, den);
  float x = __fsub_rn(__fsub_rn(1.0f, y), z);
  if (x >= 0.0f && y >= 0.0f && y <= 1.0f && z >= 0.0f && z <= 1.0f) best = th;
}

// Stop rules: which outcomes a caller needs.
enum Stop { kClosest = 0, kUnderMax = 1, kAnyHit = 2 };

template <int STOP>
__device__ __forceinline__ bool settled(float best, float hi) {
  if (STOP == kUnderMax) return best < hi;
  if (STOP == kAnyHit) return best != FLT_MAX;
  return false;
}

// Per-ray test counters of the counting variants (box tests, triangle tests).
struct Tally {
  uint32_t box = 0, tri = 0;
};

// raycastBVH of Shaders/ao_step1.comp:111-138, node order, skip pointers.
template <int STOP, bool COUNT>
__device__ float trace_skip(const SceneDev& s, f3 o, f3 d, float lo, float hi, Tally& c) {
  float best = FLT_MAX;
  uint32_t i = 0;
  while (i < s.node_count) {
    float4 L = __ldg(s.node_lo + i), H = __ldg(s.node_hi + i);
    float a = ray_box(o, d, xyz(L), xyz(H));
    if (COUNT) c.box++;
    if (a < best && a < hi) {
      uint32_t e = as_u32(H.w);
      if (COUNT) c.tri += (e - as_u32(L.w)) / 3;
      for (uint32_t k = as_u32(L.w); k < e; k += 3) tri_sample(s, k / 3, o, d, lo, best);
      if (settled<STOP>(best, hi)) break;
      ++i;
    } else {
      i = __ldg(s.node_jump + i);
    }
  }
  return best;
}

static constexpr int kStack = 64;
static_assert(kMaxOrderedDepth < kStack, "the ordered traversal defers at most one entry per level");
// The 4-wide traversal defers at most 3 entries per level.
static_assert(kMaxOrdered4Depth == (kStack - 1) / 3, "4-wide depth limit follows the stack size");
__host__ __device__ constexpr bool is_ordered(int trav) {
  return trav == FK_TRAVERSE_ORDERED || trav == FK_TRAVERSE_ORDERED4;
}

// Near-first traversal of the children-in-parent layout with the same
// pruning rule.  The host selects it only when the tree depth fits kStack;
// an overflow is still caught and reported through `status`.
template <int STOP, bool COUNT>
__device__ float trace_ordered(const SceneDev& s, f3 o, f3 d, float lo, float hi, int* status, Tally& tally) {
  float best = FLT_MAX;
  {
    float4 L = __ldg(s.node_lo), H = __ldg(s.node_hi);
    float a = ray_box(o, d, xyz(L), xyz(H));
    if (COUNT) tally.box++;
    if (!(a < hi)) return best;
    if (s.root_is_leaf) {
      uint32_t e = as_u32(H.w);
      if (COUNT) tally.tri += (e - as_u32(L.w)) / 3;
      for (uint32_t k = as_u32(L.w); k < e; k += 3) tri_sample(s, k / 3, o, d, lo, best);
      return best;
    }
  }
  int32_t stack_node[kStack];
  float stack_dist[kStack];
  int sp = 0;
  int32_t cur = 0;
  for (;;) {
    const float4* w = s.wide + 4 * (size_t)cur;
    float4 w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3);
    float aL = ray_box(o, d, mk3(w0.x, w0.z, w2.x), mk3(w0.y, w0.w, w2.y));
    float aR = ray_box(o, d, mk3(w1.x, w1.z, w2.z), mk3(w1.y, w1.w, w2.w));
    if (COUNT) tally.box += 2;
    int32_t ref[2] = {__float_as_int(w3.x), __float_as_int(w3.y)};
    int32_t cnt[2] = {__float_as_int(w3.z), __float_as_int(w3.w)};
    float dist[2] = {aL, aR};
    int first = aR < aL ? 1 : 0;
    int32_t next = -1;
    float next_d = 0.0f;
    for (int q = 0; q < 2; ++q) {
      int c = q == 0 ? first : 1 - first;
      if (!(dist[c] < fminf(best, hi))) continue;
      if (ref[c] < 0) {
        uint32_t t0 = as_u32(__ldg(s.node_lo + (-ref[c] - 1)).w) / 3;
        if (COUNT) tally.tri += (uint32_t)cnt[c];
        for (uint32_t t = t0; t < t0 + (uint32_t)cnt[c]; ++t) tri_sample(s, t, o, d, lo, best);
        if (settled<STOP>(best, hi)) return best;
      } else if (next < 0) {
        next = ref[c];
        next_d = dist[c];
      } else {
        if (sp >= kStack) {
          atomicOr(status, 1);
          return best;
        }
        stack_node[sp] = ref[c];
        stack_dist[sp] = dist[c];
        ++sp;
      }
    }
    (void)next_d;
    if (next >= 0) {
      cur = next;
      continue;
    }
    bool found = false;
    while (sp > 0) {
      --sp;
      if (stack_dist[sp] < fminf(best, hi)) {
        cur = stack_node[sp];
        found = true;
        break;
      }
    }
    if (!found) return best;
  }
}

template <int STOP, int TRAV, bool COUNT>
__device__ __forceinline__ float trace(const SceneDev& s, f3 o, f3 d, float lo, float hi, int* status, Tally& c) {
  if (TRAV == FK_TRAVERSE_ORDERED) return trace_ordered<STOP, COUNT>(s, o, d, lo, hi, status, c);
  return trace_skip<STOP, COUNT>(s, o, d, lo, hi, c);
}

// ------------------------------------------------------------------ hemisphere
struct HemiArgs {
  SceneDev s;
  const float4* __restrict__ samples;
  const float4* __restrict__ coords;
  const uint32_t* __restrict__ tidx;
  uint32_t spp, perms, offset, count;
  float lo, hi;
  float* out0;
  float* out1;
  uint32_t* hits0;
  uint32_t* hits1;
  uint32_t* queue;
  int* status;
  unsigned long long* tally;  // counting variant: total box tests, triangle tests
  const uint32_t* __restrict__ ids;  // texel list (dynamic schedule), or null
  uint32_t texel_limit;              // ids must stay below this
};

// Ray frame of Shaders/ao_step0.comp:39-50.
__device__ __forceinline__ void texel_frame(const SceneDev& s, float4 c, uint32_t id, f3& o, f3& d, f3& tx, f3& ty) {
  o = blend3(xyz(__ldg(s.pos4 + id)), xyz(__ldg(s.pos4 + id + 1)), xyz(__ldg(s.pos4 + id + 2)), c.y, c.z, c.w);
  d = normalize(blend3(xyz(__ldg(s.nrm4 + id)), xyz(__ldg(s.nrm4 + id + 1)), xyz(__ldg(s.nrm4 + id + 2)), c.y, c.z, c.w));
  ty = normalize(fabsf(d.x) > fabsf(d.y) ? mk3(d.z, 0.0f, -d.x) : mk3(0.0f, d.z, -d.y));
  tx = cross(d, ty);
}

// One warp per texel (texels pulled from an atomic queue), lanes = samples in
// rounds of 32.  Per-sample values are folded in sample order with shuffles,
// which reproduces the sequential sums of the *_step2 shaders exactly.
// KIND: FK_AO, FK_BN, FK_THICK, FK_AO_BN.
template <int KIND, int TRAV, bool COUNT>
__global__ void __launch_bounds__(256) hemi_kernel(HemiArgs p) {
  constexpr int STOP = KIND == FK_THICK ? kClosest : (KIND == FK_BN ? kAnyHit : kUnderMax);
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(p.queue, 1u);
    item = __shfl_sync(full, item, 0);
    if (item >= p.count) return;
    const uint32_t g = p.offset + item;
    uint32_t id = __ldg(p.tidx + g);
    if (id != kMiss && !valid_hit(id, p.s.corner_count)) {
      if (lane == 0) atomicOr(p.status, 2);
      id = kMiss;
    }
    if (id == kMiss) {
      if (lane == 0) {
        if (KIND == FK_AO || KIND == FK_AO_BN) p.out0[g] = 1.0f;
        if (KIND == FK_THICK) p.out0[g] = p.hi;
        float* bn = KIND == FK_BN ? p.out0 : (KIND == FK_AO_BN ? p.out1 : nullptr);
        if (bn) { bn[3 * (size_t)g] = 0.0f; bn[3 * (size_t)g + 1] = 0.0f; bn[3 * (size_t)g + 2] = 0.0f; }
        if (p.hits0) p.hits0[g] = 0;
        if (p.hits1) p.hits1[g] = 0;
      }
      continue;
    }
    f3 o, d, tx, ty;
    texel_frame(p.s, __ldg(p.coords + g), id, o, d, tx, ty);
    if (KIND == FK_THICK) d = neg(d);  // Shaders/thick_step1.comp:149
    const float4* row = p.samples + (size_t)(g % p.perms) * p.spp;
    uint32_t occ = 0, anyhit = 0;
    Tally tl;
    float acc = 0.0f;
    f3 vacc = mk3(0.0f, 0.0f, 0.0f);
    for (uint32_t k0 = 0; k0 < p.spp; k0 += 32) {
      const uint32_t k = k0 + lane;
      const bool active = k < p.spp;
      float t = FLT_MAX;
      f3 dir = mk3(0.0f, 0.0f, 0.0f);
      if (active) {
        float4 rs = __ldg(row + k);
        dir = normalize(add(add(scale(tx, rs.x), scale(ty, rs.y)), scale(d, rs.z)));
        t = trace<STOP, TRAV, COUNT>(p.s, o, dir, p.lo, p.hi, p.status, tl);
      }
      const bool hit = active && t != FLT_MAX;
      const bool under = hit && t < p.hi;
      if (KIND == FK_AO || KIND == FK_AO_BN) occ += __popc(__ballot_sync(full, under));
      anyhit += __popc(__ballot_sync(full, hit));
      const int nact = (int)min(32u, p.spp - k0);
      if (KIND == FK_BN || KIND == FK_AO_BN) {
        f3 v = hit ? mk3(0.0f, 0.0f, 0.0f) : dir;
        for (int j = 0; j < nact; ++j) {
          vacc.x = __fadd_rn(vacc.x, __shfl_sync(full, v.x, j));
          vacc.y = __fadd_rn(vacc.y, __shfl_sync(full, v.y, j));
          vacc.z = __fadd_rn(vacc.z, __shfl_sync(full, v.z, j));
        }
      }
      if (KIND == FK_THICK) {
        float v = hit ? t : p.hi;
        for (int j = 0; j < nact; ++j) acc = __fadd_rn(acc, __shfl_sync(full, v, j));
      }
    }
    if (COUNT) {
      unsigned long long b = tl.box, t = tl.tri;
      for (int off = 16; off > 0; off >>= 1) {
        b += __shfl_down_sync(full, b, off);
        t += __shfl_down_sync(full, t, off);
      }
      if (lane == 0) {
        atomicAdd(p.tally, b);
        atomicAdd(p.tally + 1, t);
      }
    }
    if (lane == 0) {
      const float fs = (float)p.spp;
      if (KIND == FK_AO || KIND == FK_AO_BN) p.out0[g] = __fsub_rn(1.0f, __fdiv_rn((float)occ, fs));
      if (KIND == FK_THICK) p.out0[g] = __fdiv_rn(acc, fs);
      if (KIND == FK_BN || KIND == FK_AO_BN) {
        float* bn = KIND == FK_BN ? p.out0 : p.out1;
        f3 v = normalize(vacc);
        bn[3 * (size_t)g] = v.x;
        bn[3 * (size_t)g + 1] = v.y;
        bn[3 * (size_t)g + 2] = v.z;
      }
      if (KIND == FK_AO_BN) {
        if (p.hits0) p.hits0[g] = occ;
        if (p.hits1) p.hits1[g] = anyhit;
      } else if (p.hits0) {
        p.hits0[g] = KIND == FK_AO ? occ : anyhit;
      }
    }
  }
}

template <int KIND, int TRAV>
static int run_hemi(fk_ctx* ctx, const HemiArgs& a) {
  auto kern = a.tally ? hemi_kernel<KIND, TRAV, true> : hemi_kernel<KIND, TRAV, false>;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "occupancy");
  if (per_sm < 1) per_sm = 1;
  uint32_t warps_needed = a.count;
  uint32_t blocks = (uint32_t)ctx->sm_count * (uint32_t)per_sm;
  uint32_t max_blocks = (warps_needed + 7) / 8;
  if (blocks > max_blocks) blocks = max_blocks;
  if (blocks == 0) return FK_OK;
  kern<<<blocks, 256, 0, ctx->stream>>>(a);
  return fk_after_launch(ctx, "hemi_kernel");
}

// What a dynamic trace launch adds beyond its arguments: staged top records
// and a persisting L2 window (fk_tuning.top_records / l2_persist).
struct TraceExtras {
  float* scratch = nullptr;  // the caller's per-ray scratch (HemiLaunch::scratch), or null
  unsigned long long scratch_rays = 0;
  uint32_t odepth = 0;  // levels of the tree walked
  const float4* top = nullptr;
  uint32_t top_count = 0, top_base = 0xFFFFFFFFu;
  const void* window = nullptr;
  size_t window_bytes = 0;
  float hit_ratio = 0.0f;
};

template <int KIND, int TRAV>
static int run_hemi_dynamic(fk_ctx* ctx, const HemiArgs& a, uint32_t refill, bool filter, uint32_t leaf_batch,
                            uint32_t speculate, const TraceExtras& x);

// Shared-memory carveout of a persistent trace kernel: just what its resident
// blocks need (static + dynamic shared memory and the 1 KB each block
// reserves, per_sm blocks), so that the rest of the SM's 256 KB array serves
// as L1 for node, leaf and triangle loads.  Left to itself the driver took
// 100 KB for 5 blocks of 8 KB; fitted, it takes 64 KB (L1 sector hit rate
// 51 % -> 53 % on the plane scene).
template <typename F>
static void fit_carveout(F fn, int per_sm, size_t dyn_smem, cudaStream_t stream) {
  // not while a graph is being recorded (the attribute was set by an earlier launch)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return;
  }
  cudaFuncAttributes fa;
  int max_sm = 0, dev = 0;
  if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess || max_sm <= 0) {
    cudaGetLastError();
    return;
  }
  const size_t need = (size_t)per_sm * (fa.sharedSizeBytes + dyn_smem + 1024);
  const int pct = (int)std::min<size_t>(100, (need * 100 + max_sm - 1) / max_sm);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct) != cudaSuccess) cudaGetLastError();
}

// Sector groups of the ray order (fk_tuning.ray_order): spp / 32 when the
// sector order applies, else 1 (sample order).
static uint32_t ray_sectors(uint32_t ray_order, uint32_t spp) {
  return ray_order == FK_RAY_ORDER_SECTOR && spp >= 64 && spp % 32 == 0 ? spp / 32 : 1;
}

int launch_hemisphere(fk_ctx* ctx, const fk_scene* s, const HemiLaunch& h) {
  if ((h.traverse & FK_TRAVERSE_MASK) == FK_TRAVERSE_ORDERED4) {
    // the scene's 4-wide layout is built on first use; the scene is otherwise unchanged
    const int rc = ensure_wide4(ctx, const_cast<fk_scene*>(s));
    if (rc != FK_OK) return rc;
  }
  HemiArgs a;
  a.s = dev_of(s);
  a.samples = h.samples;
  a.coords = h.coords;
  a.tidx = h.tidx;
  a.spp = h.spp;
  a.perms = h.perms;
  a.offset = h.offset;
  a.count = h.count;
  a.lo = h.min_d;
  a.hi = h.max_d;
  a.out0 = h.out0;
  a.out1 = h.out1;
  a.hits0 = h.hits0;
  a.hits1 = h.hits1;
  a.queue = fk_take_counter(ctx);
  a.status = ctx->status;
  a.tally = h.tally;
  a.ids = h.ids;
  a.texel_limit = h.texel_limit;
  int trav = h.traverse & FK_TRAVERSE_MASK;
  int sched = h.traverse & FK_SCHEDULE_MASK;
  if (trav == FK_TRAVERSE_AUTO) trav = s->odepth <= kMaxOrderedDepth ? FK_TRAVERSE_ORDERED : FK_TRAVERSE_SKIP;
  if (trav == FK_TRAVERSE_ORDERED && s->odepth > kMaxOrderedDepth)
    return fk_fail(ctx, FK_ERR_INVALID, "ordered traversal needs tree depth <= 48; use FK_TRAVERSE_SKIP");
  if (trav == FK_TRAVERSE_ORDERED4 && s->depth4 > kMaxOrdered4Depth)
    return fk_fail(ctx, FK_ERR_INVALID, "4-wide traversal needs a 4-wide depth <= 21; use FK_TRAVERSE_ORDERED");
  if (sched == 0) sched = FK_SCHEDULE_DYNAMIC;
  if (h.ids && sched != FK_SCHEDULE_DYNAMIC)
    return fk_fail(ctx, FK_ERR_UNSUPPORTED, "texel lists run on the dynamic schedule only");
  if (trav == FK_TRAVERSE_ORDERED4 && sched != FK_SCHEDULE_DYNAMIC)
    return fk_fail(ctx, FK_ERR_UNSUPPORTED, "the 4-wide traversal runs on the dynamic schedule only");
  const uint32_t refill = h.refill ? h.refill : ctx->tuning.refill;
  // the filtered box tests need every scene coordinate below 2^24 (fk_scene::filter_ok)
  const bool filter = !(h.traverse & FK_EXACT_BOX_TESTS) && s->filter_ok;
  const uint32_t leaf_batch = h.leaf_batch ? h.leaf_batch : ctx->tuning.leaf_batch;
  const uint32_t speculate = h.speculate ? h.speculate : ctx->tuning.speculate;
  TraceExtras x;
  x.odepth = s->odepth;
  x.scratch = h.scratch;
  x.scratch_rays = h.scratch_rays;
  if (sched == FK_SCHEDULE_DYNAMIC && trav == FK_TRAVERSE_ORDERED && ctx->tuning.top_records && !h.tally) {
    fk_scene* ms = const_cast<fk_scene*>(s);
    const int rc = ensure_top(ctx, ms, ctx->tuning.top_records);
    if (rc != FK_OK) return rc;
    if (ms->top) {
      x.top = ms->top;
      x.top_count = ms->top_count;
      x.top_base = ms->wide_count;
    }
  }
  if (sched == FK_SCHEDULE_DYNAMIC && ctx->tuning.l2_persist != FK_L2_NONE) {
    if (ctx->tuning.l2_persist == FK_L2_TREE) {
      x.window = trav == FK_TRAVERSE_ORDERED4 ? (const void*)s->wide4 : (const void*)s->wide;
      x.window_bytes = trav == FK_TRAVERSE_ORDERED4 ? 128 * (size_t)s->wide4_count : 64 * (size_t)s->wide_count;
      if (trav == FK_TRAVERSE_SKIP) x.window = s->node_lo, x.window_bytes = 16 * (size_t)s->node_count;
    } else {
      x.window = s->tri_rec;
      x.window_bytes = 64 * (size_t)(s->corner_count / 3);
    }
    int max_window = 0;
    cudaError_t e = cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, ctx->device);
    if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "cudaDevAttrMaxAccessPolicyWindowSize");
    x.window_bytes = std::min(x.window_bytes, (size_t)max_window);
    if (x.window && x.window_bytes) {
      const int rc = raise_l2(ctx, x.window_bytes, &x.hit_ratio);
      if (rc != FK_OK) return rc;
    }
  }
#define FK_HEMI_CASE(K)                                                                                       \
  case K:                                                                                                     \
    if (sched == FK_SCHEDULE_DYNAMIC) {                                                                       \
      if (trav == FK_TRAVERSE_ORDERED4)                                                                       \
        return run_hemi_dynamic<K, FK_TRAVERSE_ORDERED4>(ctx, a, refill, filter, leaf_batch, speculate, x);  \
      return trav == FK_TRAVERSE_ORDERED                                                                     \
                 ? run_hemi_dynamic<K, FK_TRAVERSE_ORDERED>(ctx, a, refill, filter, leaf_batch, speculate, x)  \
                 : run_hemi_dynamic<K, FK_TRAVERSE_SKIP>(ctx, a, refill, filter, leaf_batch, speculate, x);    \
    }                                                                                                         \
    return trav == FK_TRAVERSE_ORDERED ? run_hemi<K, FK_TRAVERSE_ORDERED>(ctx, a)                           \
                                       : run_hemi<K, FK_TRAVERSE_SKIP>(ctx, a);
  switch (h.kind) {
    FK_HEMI_CASE(FK_AO)
    FK_HEMI_CASE(FK_BN)
    FK_HEMI_CASE(FK_THICK)
    FK_HEMI_CASE(FK_AO_BN)
    default:
      return fk_fail(ctx, FK_ERR_INVALID, "fk_hemisphere: unknown kind");
  }
#undef FK_HEMI_CASE
}

// ------------------------------------------------------------------ hemisphere, dynamic
// Rays are scheduled one per lane from an atomic queue: whenever at least
// `refill` lanes of a warp are idle, one elected lane takes that many ray ids
// with a single atomicAdd and the idle lanes (ranked by ballot) start them.
// Lanes therefore stay busy while long rays of the same texel finish, and the
// per-ray closest distances land in a scratch array.  A second kernel folds
// each texel's samples in sample order, exactly as the *_step2 shaders do.

struct DynArgs {
  SceneDev s;
  const float4* __restrict__ samples;
  const float4* __restrict__ coords;
  const uint32_t* __restrict__ tidx;
  uint32_t spp, perms, texel0;  // rays [0, total) cover texels texel0 ...
  uint32_t total;
  uint32_t refill;
  uint32_t leaf_batch;  // postponed leaves that start a leaf phase early
  uint32_t speculate;   // lanes holding a leaf keep visiting inner records
  uint32_t sectors;     // ray order: queue slot q of a texel traces sample
                        // (q % 32) * sectors + q / 32 (1: sample order)
  float lo, hi;
  float* __restrict__ scratch;  // one distance per ray, in sample order
  uint32_t* queue;
  int* status;
  unsigned long long* tally;
  const uint32_t* __restrict__ ids;  // texel list, or null: ray texel g is ids[g]
  uint32_t texel_limit;
  // Top records staged in shared memory (2-wide ordered traversal): a record
  // ref >= top_base is staged record ref - top_base (top_base = ~0: none).
  const float4* __restrict__ top;
  uint32_t top_count, top_base;
};

// Texel of list position g: itself, or ids[g] for a texel list.  An id at or
// beyond the limit is reported (status bit 4) and yields kMiss, so nothing is
// read or written for it.
__device__ __forceinline__ uint32_t list_texel(const uint32_t* ids, uint32_t limit, uint32_t g, int* status) {
  if (!ids) return g;
  const uint32_t t = __ldg(ids + g);
  if (t >= limit) {
    atomicOr(status, 4);
    return kMiss;
  }
  return t;
}

// A lane's ray origin and direction live in shared memory, six words S
// apart starting at the lane's own word (ray_put), so that registers hold only
// the box-test terms: the inner visits need no more, the leaf phase and the
// skip walk read them back, and any lane of the warp can read another's.
template <int S>
__device__ __forceinline__ void ray_put(float* p, f3 o, f3 d) {
  p[0] = o.x, p[S] = o.y, p[2 * S] = o.z, p[3 * S] = d.x, p[4 * S] = d.y, p[5 * S] = d.z;
}
template <int S>
__device__ __forceinline__ f3 ray_o(const float* p) { return mk3(p[0], p[S], p[2 * S]); }
template <int S>
__device__ __forceinline__ f3 ray_d(const float* p) { return mk3(p[3 * S], p[4 * S], p[5 * S]); }

// Child box test of the traversal kernels: exact quotients, or the filtered
// form (fk_device.cuh: box_hit) whose decision is provably the same.
template <bool FILTER>
__device__ __forceinline__ bool child_hit(const RayPre& r, f3 o, f3 d, f3 lo, f3 hi, float thr, float& entry) {
  if (FILTER) return box_hit(r, o, d, lo, hi, thr, entry);
  entry = ray_box(o, d, lo, hi);
  return entry < thr;
}

// Inner-phase child test of the ordered traversals.  The filtered form is
// conservative (fk_device.cuh: box_near): a box there only prunes (the exact
// slab test is monotone, so a box inside one the ray misses is missed too),
// and every leaf's box is tested exactly when the leaf is visited, so
// accepting a box the exact test would reject only adds work.  That keeps the
// divisions out of the inner phase.  Its entry distance, a lower bound of the
// exact one, orders the two children.
template <bool FILTER, int S>
__device__ __forceinline__ bool child_maybe(const RayPre& r, const float* ray, f3 lo, f3 hi, float thr,
                                            float& entry) {
  if (FILTER) return box_near(r, lo, hi, thr, entry);
  entry = ray_box(ray_o<S>(ray), ray_d<S>(ray), lo, hi);
  return entry < thr;
}

// Lane state of the ordered traversal in the dynamic schedule.  A lane holds
// the next inner record to visit (cur) and at most one postponed leaf (pend,
// a flattened node index); the warp alternates between an inner phase and a
// leaf phase so that its lanes run the same kind of work together (Aila and
// Laine's while-while structure with postponed leaves).  Leaves are tested
// only after their box passed against a threshold no smaller than the
// current one, and re-checked against the current threshold before their
// triangles run, so the leaf set is that of the ordered traversal.
struct OState {
  int32_t cur, pend;
  int sp;
};

// Deferred entries are record refs, 4 bytes each: the entry distance is not
// kept.  A popped inner record is visited, which tests its children against
// the threshold of that moment, and a popped leaf is tested exactly in the
// leaf phase, so an entry that a shrunken threshold would have culled costs
// one visit and changes nothing.  (A ray that stops at its first hit under
// the maximum distance, or at its first hit at all, keeps its threshold at
// the maximum while it runs, so none of its entries could be culled anyway.)
// Half the bytes of (ref, distance) pairs keep more of L1 for nodes and
// triangles, which outweighs the closest-hit search's extra visits.

// Inner phase: tests both children of record `cur` against `thr` and takes
// them nearer entry first.  Their roles are decided by selects, in the order
// near child, far child: the first leaf becomes the postponed leaf when none
// is held, the first inner record the next one to visit, and the rest are
// deferred by predicated stores (near first, so the far one is popped first),
// with one overflow check per visit.  Straight-line code keeps the visit free
// of divergent branches.  TOP: records ref >= top_base are read from the
// staged copies in shared memory.
template <bool COUNT, bool FILTER, int S, int STACK = kStack, bool TOP = false>
__device__ __forceinline__ bool inner_visit(const SceneDev& s, const RayPre& rp, const float* ray, float thr,
                                            OState& st, int32_t* stk,
                                            int* status, Tally& tally, const float4* top = nullptr,
                                            uint32_t top_base = 0xFFFFFFFFu) {
  float4 w0, w1, w2, w3;
  if (TOP && (uint32_t)st.cur >= top_base) {
    const float4* w = top + 4 * ((uint32_t)st.cur - top_base);
    w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
  } else {
    const float4* w = s.wide + 4 * (size_t)st.cur;
    w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3);
  }
  float d0, d1;
  const bool h0 = child_maybe<FILTER, S>(rp, ray, mk3(w0.x, w0.z, w2.x), mk3(w0.y, w0.w, w2.y), thr, d0);
  const bool h1 = child_maybe<FILTER, S>(rp, ray, mk3(w1.x, w1.z, w2.z), mk3(w1.y, w1.w, w2.w), thr, d1);
  if (COUNT) tally.box += 2;
  const bool swap = d1 < d0;
  const bool hn = swap ? h1 : h0, hf = swap ? h0 : h1;
  const int32_t rn = __float_as_int(swap ? w3.y : w3.x), rf = __float_as_int(swap ? w3.x : w3.y);
  const bool nl = hn && rn < 0, ni = hn && rn >= 0, fl = hf && rf < 0, fi = hf && rf >= 0;
  const bool take_nl = nl && st.pend < 0;
  const bool take_fl = fl && st.pend < 0 && !take_nl;
  const bool push_n = nl && !take_nl;
  const bool push_f = (fl && !take_fl) || (fi && ni);
  int sp = st.sp;
  if (push_n && sp < STACK) stk[sp] = rn;
  sp += push_n;
  if (push_f && sp < STACK) stk[sp] = rf;
  sp += push_f;
  st.pend = take_nl ? -rn - 1 : (take_fl ? -rf - 1 : st.pend);
  st.cur = ni ? rn : (fi ? rf : -1);
  st.sp = sp;
  if (sp > STACK) {
    atomicOr(status, 1);
    return false;
  }
  return true;
}

// Compare-exchange of (key, ref) pairs: ascending keys.
__device__ __forceinline__ void cex(float& ka, int32_t& ra, float& kb, int32_t& rb) {
  const bool sw = kb < ka;
  const float k = sw ? kb : ka;
  kb = sw ? ka : kb;
  ka = k;
  const int32_t r = sw ? rb : ra;
  rb = sw ? ra : rb;
  ra = r;
}

// Inner phase over the collapsed layout: tests the 2 to 4 children of 4-wide
// node `cur` (four independent box tests), orders the hits by entry distance
// (a 5-comparator sorting network), keeps the nearest inner child as the next
// node and the nearest leaf as the postponed leaf when none is held, and
// defers the rest farthest first, so that the nearest is popped next.
template <bool COUNT, bool FILTER, int S, int STACK = kStack>
__device__ __forceinline__ bool inner_visit4(const SceneDev& s, const RayPre& rp, const float* ray, float thr,
                                             OState& st, int32_t* stk,
                                             int* status, Tally& tally) {
  const float4* w = s.wide4 + 8 * (size_t)st.cur;
  const float4 lx = __ldg(w), hx = __ldg(w + 1), ly = __ldg(w + 2), hy = __ldg(w + 3);
  const float4 lz = __ldg(w + 4), hz = __ldg(w + 5), rf = __ldg(w + 6);
  const int cnt = __float_as_int(__ldg(w + 7).x);
  const float inf = __int_as_float(0x7f800000);
  float k0, k1, k2, k3;
  const bool h0 = child_maybe<FILTER, S>(rp, ray, mk3(lx.x, ly.x, lz.x), mk3(hx.x, hy.x, hz.x), thr, k0);
  const bool h1 = child_maybe<FILTER, S>(rp, ray, mk3(lx.y, ly.y, lz.y), mk3(hx.y, hy.y, hz.y), thr, k1);
  const bool h2 = child_maybe<FILTER, S>(rp, ray, mk3(lx.z, ly.z, lz.z), mk3(hx.z, hy.z, hz.z), thr, k2) && cnt > 2;
  const bool h3 = child_maybe<FILTER, S>(rp, ray, mk3(lx.w, ly.w, lz.w), mk3(hx.w, hy.w, hz.w), thr, k3) && cnt > 3;
  if (COUNT) tally.box += cnt;
  // a hit's entry distance is finite (it is below thr); misses sort last as +inf
  k0 = h0 ? k0 : inf;
  k1 = h1 ? k1 : inf;
  k2 = h2 ? k2 : inf;
  k3 = h3 ? k3 : inf;
  int32_t r0 = __float_as_int(rf.x), r1 = __float_as_int(rf.y), r2 = __float_as_int(rf.z), r3 = __float_as_int(rf.w);
  cex(k0, r0, k1, r1);
  cex(k2, r2, k3, r3);
  cex(k0, r0, k2, r2);
  cex(k1, r1, k3, r3);
  cex(k1, r1, k2, r2);
  const bool v0 = k0 < inf, v1 = k1 < inf, v2 = k2 < inf, v3 = k3 < inf;
  const bool n0 = v0 && r0 >= 0, n1 = v1 && r1 >= 0, n2 = v2 && r2 >= 0, n3 = v3 && r3 >= 0;
  const bool l0 = v0 && r0 < 0, l1 = v1 && r1 < 0, l2 = v2 && r2 < 0, l3 = v3 && r3 < 0;
  const int ni = n0 ? 0 : (n1 ? 1 : (n2 ? 2 : (n3 ? 3 : 4)));
  const int nl = (l0 ? 0 : (l1 ? 1 : (l2 ? 2 : (l3 ? 3 : 4))));
  const int keep = st.pend < 0 ? nl : 4;  // the leaf that becomes the postponed leaf, if any
  // deferred entries farthest first, by predicated stores; one overflow check
  const bool p3 = v3 && ni != 3 && keep != 3, p2 = v2 && ni != 2 && keep != 2;
  const bool p1 = v1 && ni != 1 && keep != 1, p0 = v0 && ni != 0 && keep != 0;
  int sp = st.sp;
  if (p3 && sp < STACK) stk[sp] = r3;
  sp += p3;
  if (p2 && sp < STACK) stk[sp] = r2;
  sp += p2;
  if (p1 && sp < STACK) stk[sp] = r1;
  sp += p1;
  if (p0 && sp < STACK) stk[sp] = r0;
  sp += p0;
  st.sp = sp;
  const int32_t rk = keep == 0 ? r0 : (keep == 1 ? r1 : (keep == 2 ? r2 : r3));
  st.pend = keep < 4 ? -rk - 1 : st.pend;
  st.cur = ni == 0 ? r0 : (ni == 1 ? r1 : (ni == 2 ? r2 : (ni == 3 ? r3 : -1)));
  if (sp > STACK) {
    atomicOr(status, 1);
    return false;
  }
  return true;
}

template <int TRAV, bool COUNT, bool FILTER, int S, int STACK = kStack, bool TOP = false>
__device__ __forceinline__ bool visit_inner(const SceneDev& s, const RayPre& rp, const float* ray, float thr,
                                            OState& st, int32_t* stk, int* status, Tally& tally,
                                            const float4* top = nullptr, uint32_t top_base = 0xFFFFFFFFu) {
  if (TRAV == FK_TRAVERSE_ORDERED4)
    return inner_visit4<COUNT, FILTER, S, STACK>(s, rp, ray, thr, st, stk, status, tally);
  return inner_visit<COUNT, FILTER, S, STACK, TOP>(s, rp, ray, thr, st, stk, status, tally, top, top_base);
}

// Order-preserving key of a non-negative distance (total order, -0 below +0)
// for the leaf phase's shared-memory minimum.
__device__ __forceinline__ uint32_t dist_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float dist_unkey(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Leaf phase, warp-cooperative.  Every lane holding a postponed leaf tests
// the leaf's box exactly against its current threshold; the triangles of the
// leaves that pass are then laid end to end by a warp scan and spread over all
// 32 lanes: lane j of a round takes item base + j, finds the owning lane by a
// binary search over the scan and fetches that lane's ray and distance by
// shuffles.  A hit lowers the owner's distance through a key minimum in
// shared memory (`skey`, 32 words for this warp).  The closest distance is the
// minimum over the hits in [lo, best), so neither the order of the tests nor
// the owner's distance at the start of the phase (which only admits more
// candidates) changes it.  All lanes of the warp call this; returns whether
// this lane visited a leaf.  MULTI: lanes may trace different jobs of a
// batch, whose scenes lie in one concatenated array but whose distance
// ranges differ, so the owner's minimum distance is read from `wlo` (the
// warp's lanes' minimum distances in shared memory).
template <bool COUNT, bool FILTER, int S, bool MULTI = false>
__device__ __forceinline__ bool leaf_phase_warp(const SceneDev& s, const RayPre& rp, const float* wray, float lo,
                                                float hi, float& best, OState& st, bool active, uint32_t* skey,
                                                Tally& tally, const float* wlo = nullptr) {
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  uint32_t first = 0, cnt = 0;
  const bool mine = active && st.pend >= 0;
  __syncwarp();  // the lanes' rays, written at their set-up, are read by other lanes below
  if (mine) {
    const float4 L = __ldg(s.node_box + 2 * (size_t)st.pend), H = __ldg(s.node_box + 2 * (size_t)st.pend + 1);
    float entry;
    if (COUNT) tally.box++;
    if (child_hit<FILTER>(rp, ray_o<S>(wray + lane), ray_d<S>(wray + lane), xyz(L), xyz(H), fminf(best, hi),
                          entry)) {
      first = as_u32(L.w) / 3;
      cnt = (as_u32(H.w) - as_u32(L.w)) / 3;
      if (COUNT) tally.tri += cnt;
    }
    st.pend = -1;
  }
  uint32_t incl = cnt;
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(full, incl, d);
    if (lane >= d) incl += v;
  }
  const uint32_t total = __shfl_sync(full, incl, 31);
  if (total == 0) return mine;
  skey[lane] = dist_key(best);
  __syncwarp();
  const uint32_t excl = incl - cnt;
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t j = base + lane;
    // owner: the number of lanes whose inclusive count is <= j (steps sum to
    // 31, so o stays a lane index; for j < total it is the lane holding item j)
    int o = 0;
    for (int step = 16; step > 0; step >>= 1) {
      const uint32_t v = __shfl_sync(full, incl, o + step - 1);
      if (v <= j) o += step;
    }
    const f3 ro = ray_o<S>(wray + o), rd = ray_d<S>(wray + o);
    const float ob = __shfl_sync(full, best, o);
    const uint32_t tri = __shfl_sync(full, first, o) + (j - __shfl_sync(full, excl, o));
    float olo = lo;
    if (MULTI) olo = wlo[o];
    if (j < total) {
      float b = ob;
      tri_sample(s, tri, ro, rd, olo, b);
      if (b < ob) atomicMin(skey + o, dist_key(b));
    }
  }
  __syncwarp();
  if (cnt > 0) best = dist_unkey(skey[lane]);
  __syncwarp();  // the words are rewritten by the next leaf phase
  return mine;
}

// Takes the nearest deferred entry; false when none is left.
__device__ __forceinline__ bool pop(OState& st, const int32_t* stk) {
  if (st.sp == 0) return false;
  const int32_t r = stk[--st.sp];
  if (r < 0) st.pend = -r - 1;
  else st.cur = r;
  return true;
}

// Skip-pointer walk, one flattened node per call.
template <int STOP, bool COUNT, bool FILTER, int S>
__device__ __forceinline__ bool skip_step(const SceneDev& s, const RayPre& rp, const float* ray, float lo, float hi,
                                          float& best, int32_t& cur, Tally& tally) {
  uint32_t i = (uint32_t)cur;
  float4 L = __ldg(s.node_lo + i), H = __ldg(s.node_hi + i);
  float entry;
  const f3 o = ray_o<S>(ray), d = ray_d<S>(ray);
  bool h = child_hit<FILTER>(rp, o, d, xyz(L), xyz(H), fminf(best, hi), entry);
  if (COUNT) tally.box++;
  if (h) {
    uint32_t e = as_u32(H.w);
    if (COUNT) tally.tri += (e - as_u32(L.w)) / 3;
    for (uint32_t k = as_u32(L.w); k < e; k += 3) tri_sample(s, k / 3, o, d, lo, best);
    if (settled<STOP>(best, hi)) return true;
    ++i;
  } else {
    i = __ldg(s.node_jump + i);
  }
  cur = (int32_t)i;
  return i >= s.node_count;
}

// Inner visits a lane makes per iteration of the trace loop before the warp
// decides its next phase again (the phase ballots and the refill check are
// paid once per kInnerVisits visits).
#ifndef FK_INNER_VISITS
#define FK_INNER_VISITS 4
#endif
constexpr int kInnerVisits = FK_INNER_VISITS;

// BLOCK: threads per block; STACK: deferred entries per lane (the ordered
// traversals accept trees of depth below STACK, the 4-wide one of depth up
// to (STACK - 1) / 3); TOP: staged top records in shared memory (the 2-wide
// ordered traversal).  The launch bounds ask for 40 resident warps per SM
// (at most 51 registers a thread at 256 threads).
template <int KIND, int TRAV, bool COUNT, bool FILTER, int BLOCK = 256, int STACK = kStack, bool TOP = false>
__global__ void __launch_bounds__(BLOCK, BLOCK == 512 ? 2 : 1280 / BLOCK) hemi_trace_kernel(DynArgs p) {
  constexpr int STOP = KIND == FK_THICK ? kClosest : (KIND == FK_BN ? kAnyHit : kUnderMax);
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const unsigned lower = (1u << lane) - 1u;
  int32_t stk[is_ordered(TRAV) ? STACK : 1];  // deferred record refs
  __shared__ uint32_t leaf_keys[BLOCK / 32][32];  // leaf-phase distance minimum, per warp
  uint32_t* skey = leaf_keys[threadIdx.x >> 5];
  __shared__ float srays[6 * BLOCK];  // the lanes' ray origins and directions (ray_put)
  __shared__ uint32_t sslot[BLOCK];   // scratch slot of each lane's ray: its texel's row, its sample
  float* const myray = srays + threadIdx.x;
  const float* const wray = srays + (threadIdx.x & ~31u);
  extern __shared__ float4 top_smem[];  // p.top_count staged records (TOP)
  if (TOP) {
    for (uint32_t i = threadIdx.x; i < 4 * p.top_count; i += blockDim.x) top_smem[i] = __ldg(p.top + i);
    __syncthreads();
  }
  const uint32_t top_base = TOP ? p.top_base : 0xFFFFFFFFu;
  Tally tally;
  bool active = false, exhausted = false;
  RayPre rp = ray_pre(mk3(0.0f, 0.0f, 0.0f), mk3(1.0f, 1.0f, 1.0f));
  float best = FLT_MAX;
  int32_t cur = 0;  // skip walk: node index
  OState st = {-1, -1, 0};
  // counting variant, per warp: iterations, leaf-phase iterations, lanes at
  // work in inner / leaf phases, lanes holding a ray, refills
  unsigned long long wc[6] = {0, 0, 0, 0, 0, 0};
  for (;;) {
    unsigned idle = __ballot_sync(full, !active);
    if (!exhausted && (uint32_t)__popc(idle) >= p.refill) {
      if (COUNT) wc[5]++;
      const uint32_t n_idle = __popc(idle);
      const int leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(p.queue, n_idle);
      base = __shfl_sync(full, base, leader);
      if (base + n_idle >= p.total) exhausted = true;
      if (!active) {
        const uint32_t r = base + __popc(idle & lower);
        if (r < p.total) {
          // queue slot q of the texel -> sample k (a bijection of 0..spp-1)
          const uint32_t tq = r / p.spp;  // texel of the ray within the launch
          const uint32_t q = r - tq * p.spp;
          const uint32_t k = p.sectors > 1 ? (q & 31u) * p.sectors + (q >> 5) : q;
          const uint32_t slot = r - q + k;
          const uint32_t g = list_texel(p.ids, p.texel_limit, p.texel0 + tq, p.status);
          const uint32_t id = g == kMiss ? kMiss : __ldg(p.tidx + g);
          best = FLT_MAX;
          bool done = true;
          if (id != kMiss && valid_hit(id, p.s.corner_count)) {
            f3 o, d, tx, ty;
            texel_frame(p.s, __ldg(p.coords + g), id, o, d, tx, ty);
            if (KIND == FK_THICK) d = neg(d);
            float4 rs = __ldg(p.samples + (size_t)(g % p.perms) * p.spp + k);
            f3 dir = normalize(add(add(scale(tx, rs.x), scale(ty, rs.y)), scale(d, rs.z)));
            ray_put<BLOCK>(myray, o, dir);
            if (is_ordered(TRAV)) {
              const float4 L = __ldg(p.s.node_lo), H = __ldg(p.s.node_hi);
              rp = ray_pre_bounded(o, dir, xyz(L), xyz(H));
              if (!p.s.filter_ok) rp.exact_only = true;
              float a;
              if (COUNT) tally.box++;
              if (child_hit<FILTER>(rp, o, dir, xyz(L), xyz(H), p.hi, a)) {  // ray_box(o, dir, root) < hi, exactly
                st.sp = 0;
                st.cur = p.s.root_is_leaf ? -1 : (TOP ? (int32_t)top_base : 0);
                st.pend = p.s.root_is_leaf ? 0 : -1;
                done = false;
              }
            } else {
              rp = ray_pre(o, dir);
              if (!p.s.filter_ok) rp.exact_only = true;
              cur = 0;
              done = false;
            }
          } else if (id != kMiss) {
            atomicOr(p.status, 2);
          }
          if (done) p.scratch[slot] = best;
          else active = true;
          sslot[threadIdx.x] = slot;
        }
      }
      idle = __ballot_sync(full, !active);
    }
    if (exhausted && idle == full) break;
    if (COUNT) {
      wc[0]++;
      wc[4] += 32 - __popc(idle);
    }
    if (is_ordered(TRAV)) {
      // phase choice, uniform across the warp
      const bool spec_ok = st.sp < STACK - 4;
      const unsigned need = __ballot_sync(full, active && st.cur >= 0 && st.pend < 0);
      const unsigned leaves = __ballot_sync(full, active && st.pend >= 0);
      const bool leaf_phase = need == 0 || (uint32_t)__popc(leaves) >= p.leaf_batch;
      if (COUNT) {
        wc[1] += leaf_phase;
        wc[leaf_phase ? 3 : 2] += __popc(leaf_phase ? leaves : need);
      }
      const bool visited =
          leaf_phase && leaf_phase_warp<COUNT, FILTER, BLOCK>(p.s, rp, wray, p.lo, p.hi, best, st, active, skey, tally);
      if (active) {
        bool fin = false;
        if (leaf_phase) {
          if (visited) fin = settled<STOP>(best, p.hi);
        } else if (st.cur >= 0 && (st.pend < 0 || (p.speculate && spec_ok))) {
          if (!visit_inner<TRAV, COUNT, FILTER, BLOCK, STACK, TOP>(p.s, rp, myray, fminf(best, p.hi), st, stk,
                                                                    p.status, tally, top_smem, top_base))
            fin = true;
          // further visits in the same iteration, continuing from the stack
          for (int v = 1; v < kInnerVisits && !fin; ++v) {
            if (st.cur < 0 && st.pend < 0 && !pop(st, stk)) {
              fin = true;
              break;
            }
            if (!(st.cur >= 0 && (st.pend < 0 || (p.speculate && st.sp < STACK - 4)))) break;
            if (!visit_inner<TRAV, COUNT, FILTER, BLOCK, STACK, TOP>(p.s, rp, myray, fminf(best, p.hi), st, stk,
                                                                      p.status, tally, top_smem, top_base))
              fin = true;
          }
        }
        if (!fin && st.cur < 0 && st.pend < 0) fin = !pop(st, stk);
        if (fin) {
          p.scratch[sslot[threadIdx.x]] = best;
          active = false;
        }
      }
    } else if (active) {
      if (skip_step<STOP, COUNT, FILTER, BLOCK>(p.s, rp, myray, p.lo, p.hi, best, cur, tally)) {
        p.scratch[sslot[threadIdx.x]] = best;
        active = false;
      }
    }
  }
  if (COUNT) {
    unsigned long long b = tally.box, t = tally.tri;
    for (int off = 16; off > 0; off >>= 1) {
      b += __shfl_down_sync(full, b, off);
      t += __shfl_down_sync(full, t, off);
    }
    if (lane == 0) {
      atomicAdd(p.tally, b);
      atomicAdd(p.tally + 1, t);
      for (int k = 0; k < 6; ++k) atomicAdd(p.tally + 2 + k, wc[k]);
    }
  }
}

// ------------------------------------------------------------------ staged top records
// The first k inner records of a 2-wide tree in breadth-first order (its top
// levels), one level per pass: record i of `top` copies a tree record, and
// those of its inner children that are staged as well are referred to as
// base + their staged index (base = the tree's record count), so a traversal
// tells staged records by ref >= base.  Leaf refs and unstaged children are
// kept.  One block of 1024 threads; k <= 1024 (a level then has at most 1024
// records).
__global__ void __launch_bounds__(1024) top_records_kernel(const float4* __restrict__ wide, uint32_t base,
                                                           uint32_t k, float4* __restrict__ top) {
  __shared__ int32_t ids[2][1024];
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t level_total;
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) ids[0][0] = 0;
  __syncthreads();
  uint32_t first = 0, n = 1;  // staged index of the level's first record; the level's size
  int cur = 0;
  while (n > 0) {
    float4 w0 = {}, w1 = {}, w2 = {}, w3 = {};
    int32_t r0 = -1, r1 = -1;
    uint32_t c = 0;
    if (t < n) {
      const float4* w = wide + 4 * (size_t)ids[cur][t];
      w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
      r0 = __float_as_int(w3.x);
      r1 = __float_as_int(w3.y);
      c = (r0 >= 0) + (r1 >= 0);
    }
    // exclusive scan of the inner-child counts over the block
    uint32_t incl = c;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= (uint32_t)d) incl += v;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t v = warp_sum[lane], x = v;
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) x += y;
      }
      warp_sum[lane] = x - v;  // exclusive prefix of the warp totals
    }
    __syncthreads();
    const uint32_t excl = warp_sum[warp] + incl - c;
    const uint32_t next = first + n;  // staged index of the next level's first record
    if (t < n) {
      uint32_t q = excl;
      if (r0 >= 0) {
        if (next + q < k) {
          ids[cur ^ 1][q] = r0;
          r0 = (int32_t)(base + next + q);
        }
        ++q;
      }
      if (r1 >= 0) {
        if (next + q < k) {
          ids[cur ^ 1][q] = r1;
          r1 = (int32_t)(base + next + q);
        }
        ++q;
      }
      w3.x = __int_as_float(r0);
      w3.y = __int_as_float(r1);
      float4* o = top + 4 * (size_t)(first + t);
      o[0] = w0, o[1] = w1, o[2] = w2, o[3] = w3;
    }
    if (t == 1023) level_total = excl + c;
    __syncthreads();
    n = next < k ? min(level_total, k - next) : 0;
    first = next;
    cur ^= 1;
    __syncthreads();  // ids[cur] of this level and level_total are rewritten by the next pass
  }
}

int ensure_top(fk_ctx* ctx, fk_scene* s, uint32_t want) {
  if (want == 0 || !s->wide || s->root_is_leaf) return FK_OK;
  if (s->top && s->top_want == want && s->top_tree == s->tree) return FK_OK;
  const uint32_t k = std::min(want, s->wide_count);
  if (s->top) {
    fk_dev_free(ctx, s->top);
    s->top = nullptr;
    s->top_count = 0;
  }
  int rc = fk_dev_alloc(ctx, (void**)&s->top, 4 * sizeof(float4) * (size_t)k);
  if (rc != FK_OK) return rc;
  top_records_kernel<<<1, 1024, 0, ctx->stream>>>(s->wide, s->wide_count, k, s->top);
  rc = fk_after_launch(ctx, "top_records_kernel");
  if (rc != FK_OK) return rc;
  s->top_count = k;
  s->top_want = want;
  s->top_tree = s->tree;
  return FK_OK;
}

// Folds each texel's per-sample distances in sample order (the *_step2
// shaders' sequential sums), one thread per texel: a thread walks its
// texel's samples 0 .. spp-1 and adds each sample's term as the shader does
// (a bent-normal term of zero for a hit), so the sums are the shader's bit for
// bit, and the 32 lanes of a warp fold 32 texels at once.
template <int KIND>
__global__ void __launch_bounds__(256) hemi_reduce_kernel(HemiArgs p, const float* __restrict__ scratch,
                                                          uint32_t texel0) {
  const uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= p.count) return;
  uint32_t g = texel0 + item;
  if (p.ids) {
    g = __ldg(p.ids + g);
    if (g >= p.texel_limit) return;  // reported by the trace kernel
  }
  uint32_t id = __ldg(p.tidx + g);
  if (id != kMiss && !valid_hit(id, p.s.corner_count)) id = kMiss;
  float* bn = KIND == FK_BN ? p.out0 : (KIND == FK_AO_BN ? p.out1 : nullptr);
  if (id == kMiss) {
    if (KIND == FK_AO || KIND == FK_AO_BN) p.out0[g] = 1.0f;
    if (KIND == FK_THICK) p.out0[g] = p.hi;
    if (bn) { bn[3 * (size_t)g] = 0.0f; bn[3 * (size_t)g + 1] = 0.0f; bn[3 * (size_t)g + 2] = 0.0f; }
    if (p.hits0) p.hits0[g] = 0;
    if (p.hits1) p.hits1[g] = 0;
    return;
  }
  f3 o, d, tx, ty;
  if (KIND == FK_BN || KIND == FK_AO_BN) texel_frame(p.s, __ldg(p.coords + g), id, o, d, tx, ty);
  const float4* row = p.samples + (size_t)(g % p.perms) * p.spp;
  const float* ts = scratch + (size_t)item * p.spp;
  uint32_t occ = 0, anyhit = 0;
  float acc = 0.0f;
  f3 vacc = mk3(0.0f, 0.0f, 0.0f);
  for (uint32_t k = 0; k < p.spp; ++k) {
    const float t = __ldg(ts + k);
    const bool hit = t != FLT_MAX;
    if (KIND == FK_AO || KIND == FK_AO_BN) occ += (hit && t < p.hi) ? 1u : 0u;
    anyhit += hit ? 1u : 0u;
    if (KIND == FK_BN || KIND == FK_AO_BN) {
      f3 v = mk3(0.0f, 0.0f, 0.0f);
      if (!hit) {
        const float4 rs = __ldg(row + k);
        v = normalize(add(add(scale(tx, rs.x), scale(ty, rs.y)), scale(d, rs.z)));
      }
      vacc = add(vacc, v);
    }
    if (KIND == FK_THICK) acc = __fadd_rn(acc, hit ? t : p.hi);
  }
  const float fs = (float)p.spp;
  if (KIND == FK_AO || KIND == FK_AO_BN) p.out0[g] = __fsub_rn(1.0f, __fdiv_rn((float)occ, fs));
  if (KIND == FK_THICK) p.out0[g] = __fdiv_rn(acc, fs);
  if (KIND == FK_BN || KIND == FK_AO_BN) {
    const f3 v = normalize(vacc);
    bn[3 * (size_t)g] = v.x;
    bn[3 * (size_t)g + 1] = v.y;
    bn[3 * (size_t)g + 2] = v.z;
  }
  if (KIND == FK_AO_BN) {
    if (p.hits0) p.hits0[g] = occ;
    if (p.hits1) p.hits1[g] = anyhit;
  } else if (p.hits0) {
    p.hits0[g] = KIND == FK_AO ? occ : anyhit;
  }
}

// The trace kernel for a launch: the counting and unfiltered variants at 256
// threads and a 64-entry stack; the production variant (filtered box tests)
// of the 2-wide ordered traversal in every block shape and stack depth.
template <int KIND, int TRAV>
static void (*pick_trace(bool count, bool filter, uint32_t block, uint32_t stack, bool top))(DynArgs) {
  if (count) return filter ? hemi_trace_kernel<KIND, TRAV, true, true> : hemi_trace_kernel<KIND, TRAV, true, false>;
  if (!filter) return hemi_trace_kernel<KIND, TRAV, false, false>;
  if (TRAV == FK_TRAVERSE_ORDERED && top) return hemi_trace_kernel<KIND, TRAV, false, true, 256, kStack, true>;
  if (TRAV == FK_TRAVERSE_ORDERED) {
    if (stack == 32) {
      if (block == 128) return hemi_trace_kernel<KIND, TRAV, false, true, 128, 32>;
      if (block == 512) return hemi_trace_kernel<KIND, TRAV, false, true, 512, 32>;
      return hemi_trace_kernel<KIND, TRAV, false, true, 256, 32>;
    }
    if (block == 128) return hemi_trace_kernel<KIND, TRAV, false, true, 128, kStack>;
    if (block == 512) return hemi_trace_kernel<KIND, TRAV, false, true, 512, kStack>;
  }
  return hemi_trace_kernel<KIND, TRAV, false, true>;
}

// Block shape and stack depth a launch uses: the tuning's where the
// production variant applies and the tree fits the stack, else 256 / 64.
static void trace_shape(const fk_tuning& t, const HemiArgs& a, int trav, bool filter, uint32_t odepth, bool top,
                        uint32_t* block, uint32_t* stack) {
  *block = 256;
  *stack = kStack;
  if (a.tally || !filter || trav != FK_TRAVERSE_ORDERED || top) return;
  *block = t.block_threads;
  if (t.stack_depth == 32 && odepth <= 24) *stack = 32;
}

template <int KIND, int TRAV>
static int run_hemi_dynamic(fk_ctx* ctx, const HemiArgs& a, uint32_t refill, bool filter, uint32_t leaf_batch,
                            uint32_t speculate, const TraceExtras& x) {
  uint32_t block = 256, stack = kStack;
  trace_shape(ctx->tuning, a, TRAV, filter, x.odepth, x.top_count > 0, &block, &stack);
  auto trace = pick_trace<KIND, TRAV>(a.tally != nullptr, filter, block, stack, x.top_count > 0);
  const size_t smem = 64 * (size_t)x.top_count;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(trace, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "cudaFuncSetAttribute");
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace, (int)block, smem);
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "occupancy");
  if (per_sm < 1) per_sm = 1;
  fit_carveout(trace, per_sm, smem, ctx->stream);
  // Scratch: one float per ray, texels processed in chunks that fit it.
  const uint64_t max_rays = x.scratch ? std::min<uint64_t>(1ull << 27, x.scratch_rays) : 1ull << 27;  // 512 MB
  uint32_t chunk = (uint32_t)std::min<uint64_t>(a.count, std::max<uint64_t>(1, max_rays / a.spp));
  if (x.scratch && (uint64_t)chunk * a.spp > x.scratch_rays)
    return fk_fail(ctx, FK_ERR_INVALID, "hemisphere: the given scratch holds less than one texel's rays");
  float* scratch = x.scratch ? x.scratch : (float*)fk_scratch(ctx, (size_t)chunk * a.spp * sizeof(float));
  if (!scratch) return fk_fail(ctx, FK_ERR_NOMEM, "hemisphere scratch allocation failed");
  for (uint32_t done = 0; done < a.count; done += chunk) {
    uint32_t n = std::min(chunk, a.count - done);
    DynArgs d;
    d.s = a.s;
    d.samples = a.samples;
    d.coords = a.coords;
    d.tidx = a.tidx;
    d.spp = a.spp;
    d.perms = a.perms;
    d.texel0 = a.offset + done;
    d.total = n * a.spp;
    d.refill = refill;
    d.leaf_batch = leaf_batch;
    d.speculate = speculate;
    d.sectors = ray_sectors(ctx->tuning.ray_order, a.spp);
    d.lo = a.lo;
    d.hi = a.hi;
    d.scratch = scratch;
    d.queue = fk_take_counter(ctx);
    d.status = a.status;
    d.tally = a.tally;
    d.ids = a.ids;
    d.texel_limit = a.texel_limit;
    d.top = x.top;
    d.top_count = x.top_count;
    d.top_base = x.top_base;
    uint32_t blocks = (uint32_t)ctx->sm_count * (uint32_t)per_sm;
    uint32_t need = (d.total + block - 1) / block;
    if (blocks > need) blocks = need;
    if (x.window_bytes) {
      // the window rides on this launch only: the stream's attributes stay as the caller set them
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(blocks);
      cfg.blockDim = dim3(block);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = ctx->stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeAccessPolicyWindow;
      at[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(x.window);
      at[0].val.accessPolicyWindow.num_bytes = x.window_bytes;
      at[0].val.accessPolicyWindow.hitRatio = x.hit_ratio;
      at[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
      at[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      e = cudaLaunchKernelEx(&cfg, trace, d);
      if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "hemi_trace_kernel launch");
    } else {
      trace<<<blocks, block, smem, ctx->stream>>>(d);
    }
    int rc = fk_after_launch(ctx, "hemi_trace_kernel");
    if (rc != FK_OK) return rc;
    HemiArgs r = a;
    r.count = n;
    hemi_reduce_kernel<KIND><<<(n + 255) / 256, 256, 0, ctx->stream>>>(r, scratch, d.texel0);
    rc = fk_after_launch(ctx, "hemi_reduce_kernel");
    if (rc != FK_OK) return rc;
  }
  return FK_OK;
}

// ------------------------------------------------------------------ hemisphere, batched jobs
// Many bake jobs (each its own scene, texels, sample table, parameters and
// outputs) share one persistent launch.  The global ray space is the jobs'
// rays end to end (64-bit ids); a lane maps its ray to a job by binary search
// over the job table, which every block keeps in shared memory, and traverses
// that job's scene in place.  `stride` > 1 traces every stride-th ray only
// (the autotuner's calibration sample).
#ifndef FK_BATCH_MIN_BLOCKS
#define FK_BATCH_MIN_BLOCKS 5
#endif
template <int KIND, int TRAV, bool FILTER>
__global__ void __launch_bounds__(256, FK_BATCH_MIN_BLOCKS) batch_trace_kernel(BatchArgs p) {
  constexpr int STOP = KIND == FK_THICK ? kClosest : (KIND == FK_BN ? kAnyHit : kUnderMax);
  // the job table is read at ray set-up only (through the cache): node visits
  // need nothing per job, since the scenes are concatenated
  const BatchJobDev* __restrict__ jobs = p.jobs;
  // Per-lane state read only at ray set-up, at a ray's end or in the leaf
  // phase lives in shared memory, so that registers serve the traversal: the
  // lane's job (found once for the launch's first ray by binary search, then
  // advanced, since a lane's rays come from the queue in increasing order), its
  // ray's scratch slot and minimum distance.
  __shared__ int sjob[256];
  __shared__ uint32_t sslot[256];
  __shared__ float slo[256];
  {
    int job = 0, b = (int)p.njobs - 1;  // last job whose ray_base <= r0
    while (job < b) {
      const int m = (job + b + 1) >> 1;
      if (jobs[m].ray_base <= p.r0) job = m; else b = m - 1;
    }
    sjob[threadIdx.x] = job;
    slo[threadIdx.x] = 0.0f;
  }
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const unsigned lower = (1u << lane) - 1u;
  // a launch traces at most the scratch's 2^27 rays: lane indices fit 32 bits
  const uint32_t total = (uint32_t)((p.r1 - p.r0 + p.stride - 1) / p.stride);
  int32_t stk[is_ordered(TRAV) ? kStack : 1];  // deferred record refs
  __shared__ uint32_t leaf_keys[256 / 32][32];  // leaf-phase distance minimum, per warp
  uint32_t* skey = leaf_keys[threadIdx.x >> 5];
  __shared__ float srays[6 * 256];  // the lanes' ray origins and directions (ray_put)
  float* const myray = srays + threadIdx.x;
  const float* const wray = srays + (threadIdx.x & ~31u);
  Tally tally;
  bool active = false, exhausted = false;
  RayPre rp = ray_pre(mk3(0.0f, 0.0f, 0.0f), mk3(1.0f, 1.0f, 1.0f));
  float best = FLT_MAX, hi = 0.0f;
  int32_t cur = 0;
  uint32_t end = 0;  // skip walk: one past the job's last node
  OState st = {-1, -1, 0};
  const SceneDev& s = p.cat;  // every job's scene, concatenated
  for (;;) {
    unsigned idle = __ballot_sync(full, !active);
    if (!exhausted && (uint32_t)__popc(idle) >= p.refill) {
      const uint32_t n_idle = __popc(idle);
      const int leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if (lane == leader) base = (uint32_t)atomicAdd(p.queue, (unsigned long long)n_idle);
      base = __shfl_sync(full, base, leader);
      if ((unsigned long long)base + n_idle >= total) exhausted = true;
      if (!active) {
        const uint32_t q = base + __popc(idle & lower);
        if (q < total) {
          const unsigned long long r = p.r0 + (unsigned long long)q * p.stride;
          int job = sjob[threadIdx.x];
          while (job + 1 < (int)p.njobs && jobs[job + 1].ray_base <= r) ++job;
          sjob[threadIdx.x] = job;
          const BatchJobDev& J = jobs[job];
          const unsigned long long local = r - J.ray_base;
          // texel and sample of the ray within its job: 32-bit division when the
          // job's ray index fits (a 64-bit one is a long subroutine)
          uint32_t g, k;
          if (local < 0x100000000ull) {
            g = (uint32_t)local / J.spp;
            k = (uint32_t)local - g * J.spp;
          } else {
            g = (uint32_t)(local / J.spp);
            k = (uint32_t)(local - (unsigned long long)g * J.spp);
          }
          uint32_t slot = q;
          if (p.ray_order == FK_RAY_ORDER_SECTOR && p.stride == 1 && J.spp >= 64 && (J.spp & 31u) == 0) {
            // queue slot k of the texel traces sample (k % 32) * (spp / 32) + k / 32
            const uint32_t ks = (k & 31u) * (J.spp >> 5) + (k >> 5);
            slot = q - k + ks;
            k = ks;
          }
          const uint32_t id = __ldg(J.tidx + g);
          best = FLT_MAX;
          slo[threadIdx.x] = J.lo;
          hi = J.hi;
          bool done = true;
          if (id != kMiss && valid_hit(id, J.s.corner_count)) {
            f3 o, d, tx, ty;
            texel_frame(s, __ldg(J.coords + g), id + J.corner_base, o, d, tx, ty);
            if (KIND == FK_THICK) d = neg(d);
            float4 rs = __ldg(J.samples + (size_t)(g % J.perms) * J.spp + k);
            f3 dir = normalize(add(add(scale(tx, rs.x), scale(ty, rs.y)), scale(d, rs.z)));
            ray_put<256>(myray, o, dir);
            if (is_ordered(TRAV)) {
              const float4 L = __ldg(s.node_lo + J.node_base), H = __ldg(s.node_hi + J.node_base);
              rp = ray_pre_bounded(o, dir, xyz(L), xyz(H));
              if (!J.s.filter_ok) rp.exact_only = true;
              float aa;
              if (child_hit<FILTER>(rp, o, dir, xyz(L), xyz(H), hi, aa)) {  // ray_box(o, dir, root) < hi, exactly
                st.sp = 0;
                st.cur = J.s.root_is_leaf ? -1 : (TRAV == FK_TRAVERSE_ORDERED4 ? J.root4 : J.root2);
                st.pend = J.s.root_is_leaf ? (int32_t)J.node_base : -1;
                done = false;
              }
            } else {
              rp = ray_pre(o, dir);
              if (!J.s.filter_ok) rp.exact_only = true;
              cur = (int32_t)J.node_base;
              end = J.node_base + J.s.node_count;
              done = false;
            }
          } else if (id != kMiss) {
            atomicOr(p.status, 2);
          }
          if (done) p.scratch[slot] = best;
          else active = true;
          sslot[threadIdx.x] = slot;
        }
      }
      idle = __ballot_sync(full, !active);
    }
    if (exhausted && idle == full) break;
    if (is_ordered(TRAV)) {
      const bool spec_ok = st.sp < kStack - 4;
      const unsigned need = __ballot_sync(full, active && st.cur >= 0 && st.pend < 0);
      const unsigned leaves = __ballot_sync(full, active && st.pend >= 0);
      const bool leaf_phase = need == 0 || (uint32_t)__popc(leaves) >= p.leaf_batch;
      const bool visited =
          leaf_phase && leaf_phase_warp<false, FILTER, 256, true>(s, rp, wray, 0.0f, hi, best, st, active, skey,
                                                                  tally, slo + (threadIdx.x & ~31u));
      if (active) {
        bool fin = false;
        if (leaf_phase) {
          if (visited) fin = settled<STOP>(best, hi);
        } else if (st.cur >= 0 && (st.pend < 0 || (p.speculate && spec_ok))) {
          if (!visit_inner<TRAV, false, FILTER, 256>(s, rp, myray, fminf(best, hi), st, stk, p.status, tally))
            fin = true;
          for (int v = 1; v < kInnerVisits && !fin; ++v) {  // as in hemi_trace_kernel
            if (st.cur < 0 && st.pend < 0 && !pop(st, stk)) {
              fin = true;
              break;
            }
            if (!(st.cur >= 0 && (st.pend < 0 || (p.speculate && st.sp < kStack - 4)))) break;
            if (!visit_inner<TRAV, false, FILTER, 256>(s, rp, myray, fminf(best, hi), st, stk, p.status, tally))
              fin = true;
          }
        }
        if (!fin && st.cur < 0 && st.pend < 0) fin = !pop(st, stk);
        if (fin) {
          p.scratch[sslot[threadIdx.x]] = best;
          active = false;
        }
      }
    } else if (active) {
      if (skip_step<STOP, false, FILTER, 256>(s, rp, myray, slo[threadIdx.x], hi, best, cur, tally) ||
          (uint32_t)cur >= end) {
        p.scratch[sslot[threadIdx.x]] = best;
        active = false;
      }
    }
  }
}

// ------------------------------------------------------------------ batch scene concatenation
// One job's scene copied into the batch's concatenated arrays: triangle ranges
// (corner indices in the .w bits) and skip pointers offset by the job's corner
// and node bases, inner-record refs by its record base, leaf refs
// -(flat + 1) by its node base.
__device__ __forceinline__ float cat_ref(float r, uint32_t rec_base, uint32_t node_base) {
  const int32_t v = __float_as_int(r);
  return __int_as_float(v >= 0 ? v + (int32_t)rec_base : v - (int32_t)node_base);
}

__global__ void cat_nodes_kernel(const float4* __restrict__ lo, const float4* __restrict__ hi,
                                 const uint32_t* __restrict__ jump, uint32_t n, uint32_t node_base,
                                 uint32_t corner_base, float4* clo, float4* chi, uint32_t* cjump) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 L = lo[i], H = hi[i];
  L.w = __uint_as_float(__float_as_uint(L.w) + corner_base);
  H.w = __uint_as_float(__float_as_uint(H.w) + corner_base);
  clo[node_base + i] = L;
  chi[node_base + i] = H;
  cjump[node_base + i] = jump[i] + node_base;
}

// `width` float4 per record; the refs are float4 `ref_at` of a record, its
// first `refs` components.
__global__ void cat_records_kernel(const float4* __restrict__ rec, uint32_t n, uint32_t width, uint32_t ref_at,
                                   uint32_t refs, uint32_t rec_base, uint32_t node_base, float4* crec) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  float4 v = rec[i];
  if (i % width == ref_at) {
    v.x = cat_ref(v.x, rec_base, node_base);
    v.y = cat_ref(v.y, rec_base, node_base);
    if (refs > 2) {
      v.z = cat_ref(v.z, rec_base, node_base);
      v.w = cat_ref(v.w, rec_base, node_base);
    }
  }
  crec[(size_t)rec_base * width + i] = v;
}

int concat_batch_scene(cudaStream_t st, const fk_scene* s, uint32_t node_base, uint32_t corner_base, uint32_t rec2,
                       uint32_t rec4, const SceneDev& cat) {
  const uint32_t nn = s->node_count;
  if (nn) {
    cat_nodes_kernel<<<(nn + 255) / 256, 256, 0, st>>>(s->node_lo, s->node_hi, s->node_jump, nn, node_base,
                                                       corner_base, const_cast<float4*>(cat.node_lo),
                                                       const_cast<float4*>(cat.node_hi),
                                                       const_cast<uint32_t*>(cat.node_jump));
    if (cudaGetLastError() != cudaSuccess) return FK_ERR_CUDA;
  }
  if (s->wide && s->wide_count) {
    const uint32_t n = s->wide_count;
    cat_records_kernel<<<(4 * n + 255) / 256, 256, 0, st>>>(s->wide, n, 4, 3, 2, rec2, node_base,
                                                            const_cast<float4*>(cat.wide));
    if (cudaGetLastError() != cudaSuccess) return FK_ERR_CUDA;
  }
  if (s->wide4 && s->wide4_count) {
    const uint32_t n = s->wide4_count;
    cat_records_kernel<<<(8 * n + 255) / 256, 256, 0, st>>>(s->wide4, n, 8, 6, 4, rec4, node_base,
                                                            const_cast<float4*>(cat.wide4));
    if (cudaGetLastError() != cudaSuccess) return FK_ERR_CUDA;
  }
  const size_t nc = s->corner_count;
  if (nc) {
    if (cudaMemcpyAsync(const_cast<float4*>(cat.pos4) + corner_base, s->pos4, 16 * nc, cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess ||
        cudaMemcpyAsync(const_cast<float4*>(cat.nrm4) + corner_base, s->nrm4, 16 * nc, cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess ||
        cudaMemcpyAsync(const_cast<float4*>(cat.rec) + corner_base / 3, s->tri_rec, 16 * (nc / 3),
                        cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(const_cast<float4*>(cat.rec_bary) + 3 * (size_t)(corner_base / 3), s->tri_rec + nc / 3,
                        48 * (nc / 3), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return FK_ERR_CUDA;
  }
  return FK_OK;
}

// Per-texel folds for a batch chunk: global texels [t0, t1), one thread each,
// in sample order as hemi_reduce_kernel folds them.
template <int KIND>
__global__ void __launch_bounds__(256) batch_reduce_kernel(BatchArgs p) {
  __shared__ BatchJobDev jobs[kMaxBatchJobs];
  for (uint32_t i = threadIdx.x; i < p.njobs * (uint32_t)(sizeof(BatchJobDev) / 4); i += blockDim.x)
    ((uint32_t*)jobs)[i] = ((const uint32_t*)p.jobs)[i];
  __syncthreads();
  const uint32_t t = p.t0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.t1) return;
  int a = 0, b = (int)p.njobs - 1;
  while (a < b) {
    int m = (a + b + 1) >> 1;
    if (jobs[m].texel_base <= t) a = m; else b = m - 1;
  }
  const BatchJobDev& J = jobs[a];
  const uint32_t g = t - J.texel_base;
  const float* ts = p.scratch + (J.ray_base + (unsigned long long)g * J.spp - p.r0);
  uint32_t id = __ldg(J.tidx + g);
  if (id != kMiss && !valid_hit(id, J.s.corner_count)) id = kMiss;
  float* bn = KIND == FK_BN ? J.out0 : (KIND == FK_AO_BN ? J.out1 : nullptr);
  if (id == kMiss) {
    if (KIND == FK_AO || KIND == FK_AO_BN) J.out0[g] = 1.0f;
    if (KIND == FK_THICK) J.out0[g] = J.hi;
    if (bn) { bn[3 * (size_t)g] = 0.0f; bn[3 * (size_t)g + 1] = 0.0f; bn[3 * (size_t)g + 2] = 0.0f; }
    if (J.hits0) J.hits0[g] = 0;
    if (J.hits1) J.hits1[g] = 0;
    return;
  }
  f3 o, d, tx, ty;
  if (KIND == FK_BN || KIND == FK_AO_BN) texel_frame(J.s, __ldg(J.coords + g), id, o, d, tx, ty);
  const float4* row = J.samples + (size_t)(g % J.perms) * J.spp;
  uint32_t occ = 0, anyhit = 0;
  float acc = 0.0f;
  f3 vacc = mk3(0.0f, 0.0f, 0.0f);
  for (uint32_t k = 0; k < J.spp; ++k) {
    const float tk = __ldg(ts + k);
    const bool hit = tk != FLT_MAX;
    if (KIND == FK_AO || KIND == FK_AO_BN) occ += (hit && tk < J.hi) ? 1u : 0u;
    anyhit += hit ? 1u : 0u;
    if (KIND == FK_BN || KIND == FK_AO_BN) {
      f3 v = mk3(0.0f, 0.0f, 0.0f);
      if (!hit) {
        const float4 rs = __ldg(row + k);
        v = normalize(add(add(scale(tx, rs.x), scale(ty, rs.y)), scale(d, rs.z)));
      }
      vacc = add(vacc, v);
    }
    if (KIND == FK_THICK) acc = __fadd_rn(acc, hit ? tk : J.hi);
  }
  const float fs = (float)J.spp;
  if (KIND == FK_AO || KIND == FK_AO_BN) J.out0[g] = __fsub_rn(1.0f, __fdiv_rn((float)occ, fs));
  if (KIND == FK_THICK) J.out0[g] = __fdiv_rn(acc, fs);
  if (KIND == FK_BN || KIND == FK_AO_BN) {
    const f3 v = normalize(vacc);
    bn[3 * (size_t)g] = v.x;
    bn[3 * (size_t)g + 1] = v.y;
    bn[3 * (size_t)g + 2] = v.z;
  }
  if (KIND == FK_AO_BN) {
    if (J.hits0) J.hits0[g] = occ;
    if (J.hits1) J.hits1[g] = anyhit;
  } else if (J.hits0) {
    J.hits0[g] = KIND == FK_AO ? occ : anyhit;
  }
}

SceneDev scene_dev(const fk_scene* s) { return dev_of(s); }

template <int KIND, int TRAV, bool FILTER>
static cudaError_t batch_launch(const BatchArgs& a, cudaStream_t stream, int sm_count, bool reduce) {
  auto trace = batch_trace_kernel<KIND, TRAV, FILTER>;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace, 256, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  fit_carveout(trace, per_sm, 0, stream);
  const unsigned long long rays = (a.r1 - a.r0 + a.stride - 1) / a.stride;
  unsigned long long blocks = (unsigned long long)sm_count * per_sm;
  if (blocks > (rays + 255) / 256) blocks = (rays + 255) / 256;
  if (blocks == 0) return cudaSuccess;
  trace<<<(uint32_t)blocks, 256, 0, stream>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess || !reduce) return e;
  const uint32_t rblocks = (a.t1 - a.t0 + 255) / 256;
  if (rblocks) batch_reduce_kernel<KIND><<<rblocks, 256, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_batch(const BatchArgs& a, int kind, int trav, bool filter, cudaStream_t stream, int sm_count,
                         bool reduce) {
#define FK_BATCH_CASE(K)                                                                                   \
  case K:                                                                                                  \
    if (trav == FK_TRAVERSE_ORDERED4)                                                                      \
      return filter ? batch_launch<K, FK_TRAVERSE_ORDERED4, true>(a, stream, sm_count, reduce)            \
                    : batch_launch<K, FK_TRAVERSE_ORDERED4, false>(a, stream, sm_count, reduce);          \
    if (trav == FK_TRAVERSE_ORDERED)                                                                       \
      return filter ? batch_launch<K, FK_TRAVERSE_ORDERED, true>(a, stream, sm_count, reduce)             \
                    : batch_launch<K, FK_TRAVERSE_ORDERED, false>(a, stream, sm_count, reduce);           \
    return filter ? batch_launch<K, FK_TRAVERSE_SKIP, true>(a, stream, sm_count, reduce)                  \
                  : batch_launch<K, FK_TRAVERSE_SKIP, false>(a, stream, sm_count, reduce);
  switch (kind) {
    FK_BATCH_CASE(FK_AO)
    FK_BATCH_CASE(FK_BN)
    FK_BATCH_CASE(FK_THICK)
    FK_BATCH_CASE(FK_AO_BN)
    default:
      return cudaErrorInvalidValue;
  }
#undef FK_BATCH_CASE
}

// ------------------------------------------------------------------ hemisphere, caller scratch
// The dynamic trace + reduce pair over scratch the caller supplies (one float
// per ray, a queue word and a status word, both already zero), in a single
// pass: the caller guarantees count x spp fits its scratch.  Nothing here
// allocates; errors come back as a CUDA error code.
template <int KIND, int TRAV>
static cudaError_t run_hemi_external(const HemiArgs& a, cudaStream_t stream, int sm_count, const fk_tuning& tun,
                                     bool filter, float* dist, uint32_t* queue) {
  auto trace = filter ? hemi_trace_kernel<KIND, TRAV, false, true> : hemi_trace_kernel<KIND, TRAV, false, false>;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace, 256, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  DynArgs d;
  d.s = a.s;
  d.samples = a.samples;
  d.coords = a.coords;
  d.tidx = a.tidx;
  d.spp = a.spp;
  d.perms = a.perms;
  d.texel0 = a.offset;
  d.total = a.count * a.spp;
  d.refill = tun.refill;
  d.leaf_batch = tun.leaf_batch;
  d.speculate = tun.speculate;
  d.sectors = ray_sectors(tun.ray_order, a.spp);
  d.lo = a.lo;
  d.hi = a.hi;
  d.scratch = dist;
  d.queue = queue;
  d.status = a.status;
  d.tally = nullptr;
  d.ids = nullptr;
  d.texel_limit = 0;
  d.top = nullptr;
  d.top_count = 0;
  d.top_base = 0xFFFFFFFFu;
  uint32_t blocks = (uint32_t)sm_count * (uint32_t)per_sm;
  uint32_t need = (d.total + 255) / 256;
  if (blocks > need) blocks = need;
  trace<<<blocks, 256, 0, stream>>>(d);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  hemi_reduce_kernel<KIND><<<(a.count + 255) / 256, 256, 0, stream>>>(a, dist, a.offset);
  return cudaGetLastError();
}

int launch_hemisphere_external(const fk_scene* s, const HemiLaunch& h, cudaStream_t stream, int sm_count,
                               const fk_tuning& tun, float* dist, uint32_t* queue, int* status, std::string& err) {
  HemiArgs a;
  a.s = dev_of(s);
  a.samples = h.samples;
  a.coords = h.coords;
  a.tidx = h.tidx;
  a.spp = h.spp;
  a.perms = h.perms;
  a.offset = h.offset;
  a.count = h.count;
  a.lo = h.min_d;
  a.hi = h.max_d;
  a.out0 = h.out0;
  a.out1 = h.out1;
  a.hits0 = h.hits0;
  a.hits1 = h.hits1;
  a.queue = queue;
  a.status = status;
  a.tally = nullptr;
  a.ids = nullptr;
  a.texel_limit = 0;
  int trav = h.traverse & FK_TRAVERSE_MASK;
  if (trav == FK_TRAVERSE_AUTO) trav = s->odepth <= kMaxOrderedDepth ? FK_TRAVERSE_ORDERED : FK_TRAVERSE_SKIP;
  if (trav == FK_TRAVERSE_ORDERED && s->odepth > kMaxOrderedDepth) {
    err = "ordered traversal needs tree depth <= 48; use FK_TRAVERSE_SKIP";
    return FK_ERR_INVALID;
  }
  if (trav == FK_TRAVERSE_ORDERED4 && s->depth4 > kMaxOrdered4Depth) {
    err = "4-wide traversal needs a 4-wide depth <= 21; use FK_TRAVERSE_ORDERED";
    return FK_ERR_INVALID;
  }
  const bool filter = !(h.traverse & FK_EXACT_BOX_TESTS) && s->filter_ok;
  cudaError_t e = cudaSuccess;
#define FK_EXT_CASE(K)                                                                                     \
  case K:                                                                                                  \
    e = trav == FK_TRAVERSE_ORDERED4                                                                       \
            ? run_hemi_external<K, FK_TRAVERSE_ORDERED4>(a, stream, sm_count, tun, filter, dist, queue)   \
        : trav == FK_TRAVERSE_ORDERED                                                                      \
            ? run_hemi_external<K, FK_TRAVERSE_ORDERED>(a, stream, sm_count, tun, filter, dist, queue)    \
            : run_hemi_external<K, FK_TRAVERSE_SKIP>(a, stream, sm_count, tun, filter, dist, queue);      \
    break;
  switch (h.kind) {
    FK_EXT_CASE(FK_AO)
    FK_EXT_CASE(FK_BN)
    FK_EXT_CASE(FK_THICK)
    FK_EXT_CASE(FK_AO_BN)
    default:
      err = "unknown kind";
      return FK_ERR_INVALID;
  }
#undef FK_EXT_CASE
  if (e != cudaSuccess) {
    err = std::string("hemisphere launch: ") + cudaGetErrorName(e);
    return FK_ERR_CUDA;
  }
  return FK_OK;
}

// ------------------------------------------------------------------ mesh mapping
__device__ __forceinline__ bool bary_ok_map(f3 w) {
  return w.x >= -1e-5f && w.y >= -1e-5f && w.y <= 1.0f && w.z >= -1e-5f && w.z <= 1.0f;
}

// raycastBVH / raycastBackBVH of Shaders/meshmapping_nobackfaces.comp:102-180:
// accepts triangles facing along +d (SIGN > 0) or against it (SIGN < 0) with
// t in [0, cur); the closest so far is threaded through both passes.
template <int SIGN>
__device__ void walk_oneside(const SceneDev& s, f3 o, f3 d, float& cur, uint32_t& id, f3& w) {
  uint32_t i = 0;
  while (i < s.node_count) {
    float4 L = __ldg(s.node_lo + i), H = __ldg(s.node_hi + i);
    float a = ray_box(o, d, xyz(L), xyz(H));
    if (a < cur) {
      uint32_t e = as_u32(H.w);
      for (uint32_t k = as_u32(L.w); k < e; k += 3) {
        float4 A = __ldg(s.rec + k / 3);
        f3 n = xyz(A);
        float nd = dot(d, n);
        if (SIGN > 0 ? !(nd > 0.0f) : !(nd < 0.0f)) continue;
        float pn = dot(o, n);
        float t = __fdiv_rn(__fsub_rn(A.w, pn), nd);
        if (!(t >= 0.0f && t < cur)) continue;
        f3 q = bary_f64(add(o, scale(d, t)), xyz(__ldg(s.pos4 + k)), xyz(__ldg(s.pos4 + k + 1)),
                        xyz(__ldg(s.pos4 + k + 2)));
        if (bary_ok_map(q)) {
          cur = t;
          id = k;
          w = q;
        }
      }
      ++i;
    } else {
      i = __ldg(s.node_jump + i);
    }
  }
}

// raycastBVH of Shaders/meshmapping.comp:87-137 (either facing, t >= 0).
__device__ float walk_twoside(const SceneDev& s, f3 o, f3 d, float mint, uint32_t& id, f3& w) {
  uint32_t i = 0;
  while (i < s.node_count) {
    float4 L = __ldg(s.node_lo + i), H = __ldg(s.node_hi + i);
    float a = ray_box(o, d, xyz(L), xyz(H));
    if (a < mint) {
      float lm = FLT_MAX;
      uint32_t lid = 0;
      f3 lw = mk3(0.0f, 0.0f, 0.0f);
      uint32_t e = as_u32(H.w);
      for (uint32_t k = as_u32(L.w); k < e; k += 3) {
        float4 A = __ldg(s.rec + k / 3);
        f3 n = xyz(A);
        float nd = dot(d, n);
        if (!(fabsf(nd) > 0.0f)) continue;
        float pn = dot(o, n);
        float t = __fdiv_rn(__fsub_rn(A.w, pn), nd);
        if (!(t >= 0.0f && t < lm)) continue;
        f3 q = bary_f64(add(o, scale(d, t)), xyz(__ldg(s.pos4 + k)), xyz(__ldg(s.pos4 + k + 1)),
                        xyz(__ldg(s.pos4 + k + 2)));
        if (bary_ok_map(q)) {
          lm = t;
          lid = k;
          lw = q;
        }
      }
      if (lm < mint) {
        mint = lm;
        id = lid;
        w = lw;
      }
      ++i;
    } else {
      i = __ldg(s.node_jump + i);
    }
  }
  return mint;
}

// max_d: the walks' initial closest distance (FLT_MAX in the shaders); a
// miss writes t = FLT_MAX whatever it is.
template <int CULL>
__global__ void __launch_bounds__(128) meshmap_kernel(SceneDev s, const float4* __restrict__ pix, float max_d,
                                                      uint32_t offset, uint32_t count, float4* __restrict__ coords,
                                                      uint32_t* __restrict__ tidx) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  uint32_t g = offset + j;
  f3 p = xyz(__ldg(pix + 2 * (size_t)g)), d = xyz(__ldg(pix + 2 * (size_t)g + 1));
  uint32_t id = kMiss;
  f3 w = mk3(0.0f, 0.0f, 0.0f);
  float t = max_d;
  if (CULL) {
    walk_oneside<+1>(s, p, d, t, id, w);
    walk_oneside<-1>(s, p, neg(d), t, id, w);
  } else {
    t = fminf(t, walk_twoside(s, p, d, t, id, w));
    t = fminf(t, walk_twoside(s, p, neg(d), t, id, w));
  }
  if (id == kMiss) t = FLT_MAX;
  coords[g] = make_float4(t, w.x, w.y, w.z);
  tidx[g] = id;
}

int launch_meshmap(fk_ctx* ctx, const fk_scene* s, const fk_texel_map* m, int cull, float max_d, uint32_t offset,
                   uint32_t count, float4* coords, uint32_t* tidx) {
  if (count == 0) return FK_OK;
  uint32_t blocks = (count + 127) / 128;
  if (cull) meshmap_kernel<1><<<blocks, 128, 0, ctx->stream>>>(dev_of(s), m->pix, max_d, offset, count, coords, tidx);
  else meshmap_kernel<0><<<blocks, 128, 0, ctx->stream>>>(dev_of(s), m->pix, max_d, offset, count, coords, tidx);
  return fk_after_launch(ctx, "meshmap_kernel");
}

// ------------------------------------------------------------------ gathers
// Shaders/heights.comp:13-19, positions.comp:17-32, normals.comp:13-28.
template <int KIND>
__global__ void gather_kernel(SceneDev s, const float4* __restrict__ coords, const uint32_t* __restrict__ tidx,
                              uint32_t offset, uint32_t count, float* __restrict__ out) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  uint32_t g = offset + j;
  float4 c = __ldg(coords + g);
  if (KIND == FK_GATHER_HEIGHT) {
    out[g] = c.x != FLT_MAX ? c.x : 0.0f;
    return;
  }
  uint32_t id = __ldg(tidx + g);
  f3 v = mk3(0.0f, 0.0f, 0.0f);
  if (id != kMiss && valid_hit(id, s.corner_count)) {
    const float4* src = KIND == FK_GATHER_POSITION ? s.pos4 : s.nrm4;
    v = blend3(xyz(__ldg(src + id)), xyz(__ldg(src + id + 1)), xyz(__ldg(src + id + 2)), c.y, c.z, c.w);
    if (KIND == FK_GATHER_NORMAL) v = normalize(v);
  }
  out[3 * (size_t)g] = v.x;
  out[3 * (size_t)g + 1] = v.y;
  out[3 * (size_t)g + 2] = v.z;
}

int launch_gather(fk_ctx* ctx, const fk_scene* s, int kind, const float4* coords, const uint32_t* tidx,
                  uint32_t offset, uint32_t count, float* out) {
  if (count == 0) return FK_OK;
  uint32_t blocks = (count + 255) / 256;
  SceneDev d = dev_of(s);
  switch (kind) {
    case FK_GATHER_HEIGHT: gather_kernel<FK_GATHER_HEIGHT><<<blocks, 256, 0, ctx->stream>>>(d, coords, tidx, offset, count, out); break;
    case FK_GATHER_POSITION: gather_kernel<FK_GATHER_POSITION><<<blocks, 256, 0, ctx->stream>>>(d, coords, tidx, offset, count, out); break;
    case FK_GATHER_NORMAL: gather_kernel<FK_GATHER_NORMAL><<<blocks, 256, 0, ctx->stream>>>(d, coords, tidx, offset, count, out); break;
    default: return fk_fail(ctx, FK_ERR_INVALID, "fk_gather: unknown kind");
  }
  return fk_after_launch(ctx, "gather_kernel");
}

// Shaders/tangentspace.comp:22-41: rows of the adjugate of (n, t, b).
__global__ void tangent_kernel(const float4* __restrict__ pixt, uint32_t offset, uint32_t count, float* io3) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  uint32_t g = offset + j;
  f3 v = mk3(io3[3 * (size_t)g], io3[3 * (size_t)g + 1], io3[3 * (size_t)g + 2]);
  f3 n = xyz(__ldg(pixt + 3 * (size_t)g)), t = xyz(__ldg(pixt + 3 * (size_t)g + 1)), b = xyz(__ldg(pixt + 3 * (size_t)g + 2));
  f3 d0 = mk3(__fsub_rn(__fmul_rn(n.z, b.y), __fmul_rn(n.y, b.z)), __fsub_rn(__fmul_rn(n.x, b.z), __fmul_rn(n.z, b.x)),
              __fsub_rn(__fmul_rn(n.y, b.x), __fmul_rn(n.x, b.y)));
  f3 d1 = mk3(__fsub_rn(__fmul_rn(t.z, n.y), __fmul_rn(t.y, n.z)), __fsub_rn(__fmul_rn(t.x, n.z), __fmul_rn(n.x, t.z)),
              __fsub_rn(__fmul_rn(n.x, t.y), __fmul_rn(t.x, n.y)));
  f3 d2 = mk3(__fsub_rn(__fmul_rn(t.y, b.z), __fmul_rn(t.z, b.y)), __fsub_rn(__fmul_rn(t.z, b.x), __fmul_rn(t.x, b.z)),
              __fsub_rn(__fmul_rn(t.x, b.y), __fmul_rn(t.y, b.x)));
  f3 r = normalize(mk3(dot(v, d0), dot(v, d1), dot(v, d2)));
  io3[3 * (size_t)g] = r.x;
  io3[3 * (size_t)g + 1] = r.y;
  io3[3 * (size_t)g + 2] = r.z;
}

int launch_tangent_space(fk_ctx* ctx, const fk_texel_map* m, uint32_t offset, uint32_t count, float* io3) {
  if (count == 0) return FK_OK;
  tangent_kernel<<<(count + 255) / 256, 256, 0, ctx->stream>>>(m->pixt, offset, count, io3);
  return fk_after_launch(ctx, "tangent_kernel");
}

}  // namespace fk
