// BVH::createBinary (Src/bvh.cpp:128-314) and fillMeshData
// (Src/meshmapping.cpp:62-125) on the device: the flattened nodes and corner
// arrays of fk_bvh_build + fk_bvh_flatten, bit for bit.
//
// The host build's arithmetic is shared through fk_bvh_rules.h; its min / max
// do not depend on the order of a fold, so a parallel reduction gives the
// sequential result.  The reductions carry float keys (order-preserving, the
// two zeros merged) with a per-component flag for a -0 seen, which restores
// the rule's sign of a zero extreme.
//
// Nodes of more than kSmall triangles are split level by level: per level,
// blocks of kChunk triangles reduce each node's centroid box, bin its
// triangles into 16 buckets per axis (shared-memory atomics, flushed to the
// node's bins), one thread per node runs the host's split sweep, blocks reduce
// the two sides' boxes and count the left side, and the host turns the counts
// into offsets for a stable partition.  Nodes of at most kSmall triangles are
// built by one thread each with the host's recursion (explicit stack in global
// scratch).  The top of the tree stays on the host, which recomputes its boxes
// from the children after the subtrees are done and assigns the preorder
// indices; kernels then write the flattened records and the corners.
#include <algorithm>
#include <vector>

#include "fk_bvh_rules.h"
#include "fk_internal.h"

namespace fk {
namespace {

constexpr uint32_t kSmall = 128;   // subtrees of at most this many triangles: one thread each
constexpr uint32_t kChunk = 4096;  // triangles per block in the level passes
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kBox = 7;            // keys lo xyz, hi xyz; word 6: -0 flags (bit j: component j)
constexpr int kBinWords = 8;       // a box and its triangle count
constexpr int kBinsOff = kBox;     // per node: centroid box, 3 x 16 buckets, left box, right box
constexpr int kLeftOff = kBinsOff + 3 * 16 * kBinWords;
constexpr int kRightOff = kLeftOff + kBox;
constexpr int kTaskWords = kRightOff + kBox;

struct Task {
  uint32_t b, e, depth, pad;
};
struct Chunk {
  uint32_t task, b, e;
};
struct Split {
  int axis;
  float value;
};
// A node of a subtree built by one thread (slots [2 b, 2 e) of its range).
struct DNode {
  float c[3], s[3];
  int32_t kid[2];
  uint32_t first, count, size, pad;
};
// One level of the subtree recursion (global scratch, slots [b, e)).
struct Frame {
  uint32_t node, b, e, w, depth, stage;
};
// A subtree root: its range, depth and the box its parent's partition gave it.
struct SmallTask {
  uint32_t b, e, depth, pre;
  float c[3], s[3];
};

__host__ __device__ __forceinline__ uint32_t f2u(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(f);
#else
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
#endif
}
__host__ __device__ __forceinline__ float u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}
// Order-preserving key with the two zeros merged.
__host__ __device__ __forceinline__ uint32_t zkey(float f) {
  uint32_t u = f2u(f);
  if ((u << 1) == 0) u = 0;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float zval(uint32_t k, bool neg_zero) {
  const float f = u2f((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
  return (f == 0.0f && neg_zero) ? -0.0f : f;
}
__host__ __device__ __forceinline__ bool is_neg_zero(float f) { return f2u(f) == 0x80000000u; }

// Box accumulator in memory: lo keys (min), hi keys (max), -0 flags.
__host__ __device__ __forceinline__ void box_init(uint32_t* w) {
  for (int q = 0; q < 3; ++q) {
    w[q] = zkey(FLT_MAX);
    w[3 + q] = zkey(-FLT_MAX);
  }
  w[6] = 0;
}
__host__ __device__ __forceinline__ void box_read(const uint32_t* w, float lo[3], float hi[3]) {
  for (int q = 0; q < 3; ++q) {
    lo[q] = zval(w[q], (w[6] >> q) & 1u);
    hi[q] = zval(w[3 + q], (w[6] >> (3 + q)) & 1u);
  }
}
// Folds a partial box (lo / hi, each already a rule fold of its part) into
// the accumulator; NaN components never arrive here (a NaN loses every fold).
__device__ __forceinline__ void box_atomic(uint32_t* w, const float lo[3], const float hi[3]) {
  uint32_t flags = 0;
  for (int q = 0; q < 3; ++q) {
    if (lo[q] == lo[q]) {
      atomicMin(w + q, zkey(lo[q]));
      if (is_neg_zero(lo[q])) flags |= 1u << q;
    }
    if (hi[q] == hi[q]) {
      atomicMax(w + 3 + q, zkey(hi[q]));
      if (is_neg_zero(hi[q])) flags |= 1u << (3 + q);
    }
  }
  if (flags) atomicOr(w + 6, flags);
}

__device__ __forceinline__ void fold_warp(float lo[3], float hi[3]) {
  for (int d = 16; d > 0; d >>= 1)
    for (int q = 0; q < 3; ++q) {
      lo[q] = bvh::fmin(lo[q], __shfl_xor_sync(0xFFFFFFFFu, lo[q], d));
      hi[q] = bvh::fmax(hi[q], __shfl_xor_sync(0xFFFFFFFFu, hi[q], d));
    }
}

// Block fold of per-thread partial boxes into the accumulator `w`.
__device__ __forceinline__ void fold_block(float lo[3], float hi[3], uint32_t* w) {
  __shared__ float red[kWarps][6];
  fold_warp(lo, hi);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < 3; ++q) {
      red[warp][q] = lo[q];
      red[warp][3 + q] = hi[q];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    float L[3], H[3];
    for (int q = 0; q < 3; ++q) {
      L[q] = red[0][q];
      H[q] = red[0][3 + q];
      for (int k = 1; k < kWarps; ++k) {
        L[q] = bvh::fmin(L[q], red[k][q]);
        H[q] = bvh::fmax(H[q], red[k][3 + q]);
      }
    }
    box_atomic(w, L, H);
  }
  __syncthreads();
}

__device__ __forceinline__ float comp(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// ------------------------------------------------------------ per triangle
// Src/bvh.cpp:139 / :227 centroids and the triangle's box (the fold of its
// corners, as addPoint of the three corners gives it).
__global__ void bvh_pre_kernel(uint32_t nf, const float* __restrict__ pos, const uint32_t* __restrict__ verts,
                           const uint32_t* __restrict__ tris, float4* pc, float4* pm, float4* plo, float4* phi) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  float p[3][3];
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = __ldg(tris + 3 * (size_t)f + k);
    const uint32_t pi = __ldg(verts + 3 * (size_t)v);
    for (int a = 0; a < 3; ++a) p[k][a] = __ldg(pos + 3 * (size_t)pi + a);
  }
  float cd[3], cm[3], lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    const float s = __fadd_rn(__fadd_rn(p[0][a], p[1][a]), p[2][a]);
    cd[a] = __fdiv_rn(s, 3.0f);
    cm[a] = __fmul_rn(s, 1.0f / 3.0f);
    lo[a] = bvh::fmin(p[0][a], bvh::fmin(p[1][a], p[2][a]));
    hi[a] = bvh::fmax(p[0][a], bvh::fmax(p[1][a], p[2][a]));
  }
  pc[f] = make_float4(cd[0], cd[1], cd[2], 0.0f);
  pm[f] = make_float4(cm[0], cm[1], cm[2], 0.0f);
  plo[f] = make_float4(lo[0], lo[1], lo[2], 0.0f);
  phi[f] = make_float4(hi[0], hi[1], hi[2], 0.0f);
}

// Root box over every position (Src/bvh.cpp:287-297), referenced or not.
__global__ void __launch_bounds__(kThreads) bvh_points_kernel(const float* __restrict__ pos, uint32_t np, uint32_t* w) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < np; i += gridDim.x * kThreads)
    for (int q = 0; q < 3; ++q) {
      const float v = __ldg(pos + 3 * (size_t)i + q);
      lo[q] = bvh::fmin(lo[q], v);
      hi[q] = bvh::fmax(hi[q], v);
    }
  fold_block(lo, hi, w);
}

// ------------------------------------------------------------ level passes
__global__ void bvh_init_kernel(uint32_t* acc, uint32_t nt) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  uint32_t* w = acc + (size_t)t * kTaskWords;
  box_init(w);
  for (int k = 0; k < 48; ++k) {
    box_init(w + kBinsOff + k * kBinWords);
    w[kBinsOff + k * kBinWords + 7] = 0;
  }
  box_init(w + kLeftOff);
  box_init(w + kRightOff);
}

__global__ void __launch_bounds__(kThreads) bvh_centroid_kernel(const Chunk* chunks, const uint32_t* __restrict__ perm,
                                                            const float4* __restrict__ pc, uint32_t* acc) {
  const Chunk c = chunks[blockIdx.x];
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += kThreads) {
    const float4 v = __ldg(pc + perm[i]);
    for (int q = 0; q < 3; ++q) {
      lo[q] = bvh::fmin(comp(v, q), lo[q]);
      hi[q] = bvh::fmax(comp(v, q), hi[q]);
    }
  }
  fold_block(lo, hi, acc + (size_t)c.task * kTaskWords);
}

__global__ void __launch_bounds__(kThreads) bvh_bucket_kernel(const Chunk* chunks, const uint32_t* __restrict__ perm,
                                                          const float4* __restrict__ pc,
                                                          const float4* __restrict__ plo,
                                                          const float4* __restrict__ phi, uint32_t* acc) {
  __shared__ uint32_t sb[48 * kBinWords];
  for (int k = threadIdx.x; k < 48; k += kThreads) {
    box_init(sb + k * kBinWords);
    sb[k * kBinWords + 7] = 0;
  }
  const Chunk c = chunks[blockIdx.x];
  uint32_t* w = acc + (size_t)c.task * kTaskWords;
  float clo[3], chi[3], ext[3];
  box_read(w, clo, chi);
  for (int q = 0; q < 3; ++q) ext[q] = __fsub_rn(chi[q], clo[q]);
  __syncthreads();
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += kThreads) {
    const uint32_t t = perm[i];
    const float4 v = __ldg(pc + t), L = __ldg(plo + t), H = __ldg(phi + t);
    const float lo[3] = {L.x, L.y, L.z}, hi[3] = {H.x, H.y, H.z};
    for (int a = 0; a < 3; ++a) {
      const uint32_t k = bvh::bucket(comp(v, a), clo[a], ext[a]);
      uint32_t* bw = sb + (a * 16 + k) * kBinWords;
      box_atomic(bw, lo, hi);
      atomicAdd(bw + 7, 1u);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 48; k += kThreads) {
    const uint32_t* s = sb + k * kBinWords;
    if (s[7] == 0) continue;
    uint32_t* g = w + kBinsOff + k * kBinWords;
    for (int q = 0; q < 3; ++q) {
      atomicMin(g + q, s[q]);
      atomicMax(g + 3 + q, s[3 + q]);
    }
    if (s[6]) atomicOr(g + 6, s[6]);
    atomicAdd(g + 7, s[7]);
  }
}

__global__ void bvh_choose_kernel(const Task* tasks, uint32_t nt, const uint32_t* acc, Split* splits) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const uint32_t* w = acc + (size_t)t * kTaskWords;
  float clo[3], chi[3];
  box_read(w, clo, chi);
  float blo[3][16][3], bhi[3][16][3];
  uint32_t cnt[3][16];
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 16; ++k) {
      const uint32_t* b = w + kBinsOff + (a * 16 + k) * kBinWords;
      box_read(b, blo[a][k], bhi[a][k]);
      cnt[a][k] = b[7];
    }
  int axis;
  float value;
  bvh::pick_split(blo, bhi, cnt, (int)(tasks[t].e - tasks[t].b), clo, chi, &axis, &value);
  splits[t] = Split{axis, value};
}

// Left / right boxes and the left count per chunk (Src/bvh.cpp:222-247).
__global__ void __launch_bounds__(kThreads) bvh_side_kernel(const Chunk* chunks, const uint32_t* __restrict__ perm,
                                                        const float4* __restrict__ pm,
                                                        const float4* __restrict__ plo,
                                                        const float4* __restrict__ phi, const Split* splits,
                                                        uint32_t* acc, uint32_t* chunk_left) {
  const Chunk c = chunks[blockIdx.x];
  const Split sp = splits[c.task];
  float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  uint32_t n = 0;
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += kThreads) {
    const uint32_t t = perm[i];
    const float4 L = __ldg(plo + t), H = __ldg(phi + t);
    if (comp(__ldg(pm + t), sp.axis) <= sp.value) {
      ++n;
      for (int q = 0; q < 3; ++q) {
        llo[q] = bvh::fmin(llo[q], comp(L, q));
        lhi[q] = bvh::fmax(lhi[q], comp(H, q));
      }
    } else {
      for (int q = 0; q < 3; ++q) {
        rlo[q] = bvh::fmin(rlo[q], comp(L, q));
        rhi[q] = bvh::fmax(rhi[q], comp(H, q));
      }
    }
  }
  uint32_t* w = acc + (size_t)c.task * kTaskWords;
  fold_block(llo, lhi, w + kLeftOff);
  fold_block(rlo, rhi, w + kRightOff);
  for (int d = 16; d > 0; d >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, d);
  __shared__ uint32_t red[kWarps];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int k = 0; k < kWarps; ++k) s += red[k];
    chunk_left[blockIdx.x] = s;
  }
}

// Stable partition of the chunk into `out` (offs: this chunk's start on the
// left and on the right side of its node); chunks of nodes that stay leaves
// are not launched.
__global__ void __launch_bounds__(kThreads) bvh_scatter_kernel(const Chunk* chunks, const uint32_t* node_left,
                                                           const uint32_t* __restrict__ perm, uint32_t* out,
                                                           const float4* __restrict__ pm, const Split* splits,
                                                           const uint32_t* offs, const uint32_t* task_b) {
  const Chunk c = chunks[blockIdx.x];
  const Split sp = splits[c.task];
  uint32_t lbase = task_b[c.task] + offs[2 * blockIdx.x];
  uint32_t rbase = task_b[c.task] + node_left[c.task] + offs[2 * blockIdx.x + 1];
  __shared__ uint32_t wl[kWarps], wr[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t below = (1u << lane) - 1u;
  for (uint32_t base = c.b; base < c.e; base += kThreads) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < c.e;
    const uint32_t t = valid ? perm[i] : 0u;
    const bool left = valid && comp(__ldg(pm + t), sp.axis) <= sp.value;
    const bool right = valid && !left;
    const uint32_t bl = __ballot_sync(0xFFFFFFFFu, left), br = __ballot_sync(0xFFFFFFFFu, right);
    if (lane == 0) {
      wl[warp] = __popc(bl);
      wr[warp] = __popc(br);
    }
    __syncthreads();
    uint32_t pl = 0, pr = 0, tl = 0, tr = 0;
    for (int k = 0; k < kWarps; ++k) {
      if (k < warp) {
        pl += wl[k];
        pr += wr[k];
      }
      tl += wl[k];
      tr += wr[k];
    }
    if (left) out[lbase + pl + __popc(bl & below)] = t;
    if (right) out[rbase + pr + __popc(br & below)] = t;
    lbase += tl;
    rbase += tr;
    __syncthreads();
  }
}

__global__ void bvh_copy_back_kernel(const Chunk* chunks, const uint32_t* __restrict__ from, uint32_t* to) {
  const Chunk c = chunks[blockIdx.x];
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += blockDim.x) to[i] = from[i];
}

// ------------------------------------------------------------ small subtrees
__device__ __forceinline__ void set_box(DNode& n, const float lo[3], const float hi[3]) {
  for (int a = 0; a < 3; ++a) {
    n.c[a] = __fmul_rn(__fadd_rn(lo[a], hi[a]), 0.5f);
    n.s[a] = __fmul_rn(__fsub_rn(hi[a], lo[a]), 0.5f);
  }
}

// status: 1 = a subtree ran out of its node slots or stack (cannot happen:
// a subtree over n triangles has at most 2 n - 1 nodes and depth n).
__global__ void __launch_bounds__(64) bvh_small_kernel(const SmallTask* tasks, uint32_t ns, uint32_t* perm,
                                                   uint32_t* scratch, Frame* frames, const float4* __restrict__ pc,
                                                   const float4* __restrict__ pm, const float4* __restrict__ plo,
                                                   const float4* __restrict__ phi, DNode* nodes, uint32_t max_tris,
                                                   uint32_t max_depth, uint32_t* status) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const SmallTask T = tasks[k];
  const uint32_t slot0 = 2 * T.b, slot_end = 2 * T.e;
  uint32_t next = slot0 + 1;
  {
    DNode& r = nodes[slot0];
    for (int a = 0; a < 3; ++a) {
      r.c[a] = T.c[a];
      r.s[a] = T.s[a];
    }
    r.kid[0] = r.kid[1] = -1;
  }
  Frame* st = frames + T.b;
  const uint32_t cap = T.e - T.b;
  int sp = 0;
  st[sp++] = Frame{slot0, T.b, T.e, 0, T.depth, 0};
  while (sp > 0) {
    Frame& f = st[sp - 1];
    DNode& nd = nodes[f.node];
    if (f.stage == 0) {
      nd.first = f.b;
      nd.count = f.e - f.b;
      nd.kid[0] = nd.kid[1] = -1;
      if (f.e - f.b <= max_tris || f.depth >= max_depth) {
        nd.size = 1;
        --sp;
        continue;
      }
      // choose (Src/bvh.cpp:128-203)
      float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      for (uint32_t i = f.b; i < f.e; ++i) {
        const float4 v = __ldg(pc + perm[i]);
        for (int q = 0; q < 3; ++q) {
          clo[q] = bvh::fmin(comp(v, q), clo[q]);
          chi[q] = bvh::fmax(comp(v, q), chi[q]);
        }
      }
      float ext[3];
      for (int q = 0; q < 3; ++q) ext[q] = __fsub_rn(chi[q], clo[q]);
      float blo[3][16][3], bhi[3][16][3];
      uint32_t cnt[3][16];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 16; ++b) {
          cnt[a][b] = 0;
          for (int q = 0; q < 3; ++q) {
            blo[a][b][q] = FLT_MAX;
            bhi[a][b][q] = -FLT_MAX;
          }
        }
      for (uint32_t i = f.b; i < f.e; ++i) {
        const uint32_t t = perm[i];
        const float4 v = __ldg(pc + t), L = __ldg(plo + t), H = __ldg(phi + t);
        for (int a = 0; a < 3; ++a) {
          const uint32_t b = bvh::bucket(comp(v, a), clo[a], ext[a]);
          cnt[a][b]++;
          for (int q = 0; q < 3; ++q) {
            blo[a][b][q] = bvh::fmin(comp(L, q), blo[a][b][q]);
            bhi[a][b][q] = bvh::fmax(comp(H, q), bhi[a][b][q]);
          }
        }
      }
      int axis;
      float split;
      bvh::pick_split(blo, bhi, cnt, (int)(f.e - f.b), clo, chi, &axis, &split);
      // order-preserving partition (Src/bvh.cpp:222-258)
      float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      uint32_t w = f.b, nr = 0;
      for (uint32_t i = f.b; i < f.e; ++i) {
        const uint32_t t = perm[i];
        const float4 L = __ldg(plo + t), H = __ldg(phi + t);
        if (comp(__ldg(pm + t), axis) <= split) {
          perm[w++] = t;
          for (int q = 0; q < 3; ++q) {
            llo[q] = bvh::fmin(llo[q], comp(L, q));
            lhi[q] = bvh::fmax(lhi[q], comp(H, q));
          }
        } else {
          scratch[f.b + nr++] = t;
          for (int q = 0; q < 3; ++q) {
            rlo[q] = bvh::fmin(rlo[q], comp(L, q));
            rhi[q] = bvh::fmax(rhi[q], comp(H, q));
          }
        }
      }
      for (uint32_t j = 0; j < nr; ++j) perm[w + j] = scratch[f.b + j];
      if (w == f.b || w == f.e) {  // cannot split: stays a leaf
        nd.size = 1;
        --sp;
        continue;
      }
      if (next + 2 > slot_end || sp + 1 > (int)cap) {
        atomicOr(status, 1u);
        return;
      }
      nd.count = 0;
      const uint32_t li = next, ri = next + 1;
      next += 2;
      set_box(nodes[li], llo, lhi);
      set_box(nodes[ri], rlo, rhi);
      nd.kid[0] = (int32_t)li;
      nd.kid[1] = (int32_t)ri;
      f.w = w;
      f.stage = 1;
      const Frame child{li, f.b, w, 0, f.depth + 1, 0};
      st[sp++] = child;
    } else if (f.stage == 1) {
      f.stage = 2;
      if (sp + 1 > (int)cap) {
        atomicOr(status, 1u);
        return;
      }
      const Frame child{(uint32_t)nd.kid[1], f.w, f.e, 0, f.depth + 1, 0};
      st[sp++] = child;
    } else {
      const DNode& A = nodes[nd.kid[0]];
      const DNode& B = nodes[nd.kid[1]];
      for (int a = 0; a < 3; ++a) {
        const float lo = bvh::fmin(__fsub_rn(A.c[a], A.s[a]), __fsub_rn(B.c[a], B.s[a]));
        const float hi = bvh::fmax(__fadd_rn(A.c[a], A.s[a]), __fadd_rn(B.c[a], B.s[a]));
        nd.c[a] = __fmul_rn(__fadd_rn(hi, lo), 0.5f);
        nd.s[a] = __fmul_rn(__fsub_rn(hi, lo), 0.5f);
      }
      nd.size = 1 + A.size + B.size;
      --sp;
    }
  }
}

__global__ void bvh_small_roots_kernel(const SmallTask* tasks, uint32_t ns, const DNode* nodes, DNode* roots) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ns) roots[k] = nodes[2 * tasks[k].b];
}

// Flattened records of one subtree, its root at preorder index tasks[k].pre:
// aabbMin = c - s, aabbMax = c + s, start / end corners, jump (Src/meshmapping.cpp:62-125).
// status bit 2: a preorder index fell outside the node arrays (not written).
__global__ void __launch_bounds__(64) bvh_small_flatten_kernel(const SmallTask* tasks, uint32_t ns, const DNode* nodes,
                                                           uint32_t* stack, float4* lo, float4* hi,
                                                           uint32_t* jump, uint32_t nn, uint32_t* status) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const SmallTask T = tasks[k];
  // (slot, preorder) pairs, words [2 b, 2 e) of a 6-words-per-triangle array:
  // at most depth + 1 <= e - b pairs are live
  uint32_t* st = stack + 2 * (size_t)T.b;
  int sp = 0;
  st[0] = 2 * T.b;
  st[1] = T.pre;
  sp = 1;
  while (sp > 0) {
    --sp;
    const uint32_t slot = st[2 * sp], pre = st[2 * sp + 1];
    if (pre >= nn || slot < 2 * T.b || slot >= 2 * T.e) {
      atomicOr(status, 2u);
      return;
    }
    const DNode& n = nodes[slot];
    const bool leaf = n.kid[0] < 0;
    const uint32_t start = 3 * n.first, end = leaf ? 3 * (n.first + n.count) : 3 * n.first;
    lo[pre] = make_float4(__fsub_rn(n.c[0], n.s[0]), __fsub_rn(n.c[1], n.s[1]), __fsub_rn(n.c[2], n.s[2]),
                          __uint_as_float(start));
    hi[pre] = make_float4(__fadd_rn(n.c[0], n.s[0]), __fadd_rn(n.c[1], n.s[1]), __fadd_rn(n.c[2], n.s[2]),
                          __uint_as_float(end));
    jump[pre] = pre + n.size;
    if (!leaf) {
      const uint32_t ls = nodes[n.kid[0]].size;
      st[2 * sp] = (uint32_t)n.kid[1];
      st[2 * sp + 1] = pre + 1 + ls;
      ++sp;
      st[2 * sp] = (uint32_t)n.kid[0];
      st[2 * sp + 1] = pre + 1;
      ++sp;
    }
  }
}

struct FlatRec {
  float4 lo, hi;
  uint32_t pre, jump, pad[2];
};
__global__ void bvh_host_records_kernel(const FlatRec* recs, uint32_t n, float4* lo, float4* hi, uint32_t* jump) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const FlatRec r = recs[k];
  lo[r.pre] = r.lo;
  hi[r.pre] = r.hi;
  jump[r.pre] = r.jump;
}

// Corners in leaf order (Src/meshmapping.cpp:94-109): position and normal of
// each corner of the i-th triangle of the final order, w = 0.
__global__ void bvh_corners_kernel(uint32_t nf, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ tris,
                               const uint32_t* __restrict__ verts, const float* __restrict__ pos,
                               const float* __restrict__ nrm, float4* pos4, float4* nrm4) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const uint32_t f = perm[i];
  for (int k = 0; k < 3; ++k) {
    const uint32_t v = __ldg(tris + 3 * (size_t)f + k);
    const uint32_t pi = __ldg(verts + 3 * (size_t)v), ni = __ldg(verts + 3 * (size_t)v + 2);
    pos4[3 * (size_t)i + k] =
        make_float4(__ldg(pos + 3 * (size_t)pi), __ldg(pos + 3 * (size_t)pi + 1), __ldg(pos + 3 * (size_t)pi + 2), 0.0f);
    nrm4[3 * (size_t)i + k] =
        make_float4(__ldg(nrm + 3 * (size_t)ni), __ldg(nrm + 3 * (size_t)ni + 1), __ldg(nrm + 3 * (size_t)ni + 2), 0.0f);
  }
}

// Whether every corner coordinate is below `lim` in magnitude (a NaN is not).
__global__ void bvh_corners_below_kernel(const float4* __restrict__ p, uint32_t n, float lim, uint32_t* bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 v = p[i];
    if (!(fabsf(v.x) < lim && fabsf(v.y) < lim && fabsf(v.z) < lim)) {
      atomicOr(bad, 1u);
      return;
    }
  }
}

// ------------------------------------------------------------ host side
struct HNode {
  float c[3], s[3];
  int32_t kid[2] = {-1, -1};  // >= 0: host node; < 0: -(subtree index) - 1
  uint32_t first = 0, count = 0, size = 1, pre = 0;
  bool leaf = true;
  bool sub = false;  // handed to a subtree thread (its records come from there)
};

void host_set_box(HNode& n, const float lo[3], const float hi[3]) {
  for (int a = 0; a < 3; ++a) {
    n.c[a] = (lo[a] + hi[a]) * 0.5f;
    n.s[a] = (hi[a] - lo[a]) * 0.5f;
  }
}

template <class T>
T* carve(char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += (sizeof(T) * count + 255) & ~(size_t)255;
  return r;
}

}  // namespace

int corners_below(fk_ctx* ctx, const float4* p, uint32_t n, float lim, bool* ok) {
  *ok = true;
  if (n == 0) return FK_OK;
  uint32_t* bad = nullptr;
  int rc = fk_dev_alloc(ctx, (void**)&bad, 4);
  if (rc != FK_OK) return rc;
  uint32_t h = 0;
  cudaError_t e = cudaMemsetAsync(bad, 0, 4, ctx->stream);
  if (e == cudaSuccess) {
    bvh_corners_below_kernel<<<std::min<uint32_t>((n + 255) / 256, (uint32_t)ctx->sm_count * 8), 256, 0, ctx->stream>>>(
        p, n, lim, bad);
    rc = fk_after_launch(ctx, "corner bound");
    if (rc == FK_OK) e = cudaMemcpyAsync(&h, bad, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (rc == FK_OK && e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  }
  fk_dev_free(ctx, bad);
  if (rc != FK_OK) return rc;
  if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "corner bound");
  *ok = h == 0;
  return FK_OK;
}

int build_bvh_device(fk_ctx* ctx, const fk_mesh* mesh, uint32_t max_tris, uint32_t max_depth, DevBvh* out) {
  *out = DevBvh{};
  const uint32_t nf = mesh->triangle_count(), nv = mesh->vertex_count(), np = mesh->position_count();
  const uint32_t nnrm = (uint32_t)(mesh->normals.size() / 3);
  // every index the kernels follow is checked here
  for (uint32_t i = 0; i < 3 * nf; ++i)
    if (mesh->triangles[i] >= nv) return fk_fail(ctx, FK_ERR_INVALID, "device BVH build: triangle index out of range");
  for (uint32_t v = 0; v < nv; ++v)
    if (mesh->vertices[3 * (size_t)v] >= np || mesh->vertices[3 * (size_t)v + 2] >= nnrm)
      return fk_fail(ctx, FK_ERR_INVALID, "device BVH build: vertex index out of range");
  cudaStream_t st = ctx->stream;
  int rc = FK_OK;

  // device inputs and work arrays
  const size_t F = nf ? nf : 1;
  const uint32_t max_tasks = nf / (kSmall + 1) + 1, max_chunks = nf / kChunk + max_tasks + 1;
  // work arrays, carved from one allocation; the size comes from the same
  // carve sequence run over offsets
  float* d_pos;
  float* d_nrm;
  uint32_t *d_verts, *d_tris, *perm, *tmp, *scratch, *acc, *d_node_left, *d_task_b, *d_chunk_left, *d_offs, *d_status;
  float4 *pc, *pm, *plo, *phi;
  Frame* frames;
  DNode* dnodes;
  Task* d_tasks;
  Split* d_splits;
  Chunk* d_chunks;
  auto layout = [&](char* base) -> size_t {
    char* p = base;
    d_pos = carve<float>(p, mesh->positions.size() + 1);
    d_nrm = carve<float>(p, mesh->normals.size() + 1);
    d_verts = carve<uint32_t>(p, mesh->vertices.size() + 1);
    d_tris = carve<uint32_t>(p, mesh->triangles.size() + 1);
    pc = carve<float4>(p, F);
    pm = carve<float4>(p, F);
    plo = carve<float4>(p, F);
    phi = carve<float4>(p, F);
    perm = carve<uint32_t>(p, F);
    tmp = carve<uint32_t>(p, F);
    scratch = carve<uint32_t>(p, F);
    frames = carve<Frame>(p, F);
    dnodes = carve<DNode>(p, 2 * F);
    acc = carve<uint32_t>(p, (size_t)kTaskWords * max_tasks + kBox);
    d_tasks = carve<Task>(p, max_tasks);
    d_splits = carve<Split>(p, max_tasks);
    d_node_left = carve<uint32_t>(p, max_tasks);
    d_task_b = carve<uint32_t>(p, max_tasks);
    d_chunks = carve<Chunk>(p, max_chunks);
    d_chunk_left = carve<uint32_t>(p, max_chunks);
    d_offs = carve<uint32_t>(p, 2 * (size_t)max_chunks);
    d_status = carve<uint32_t>(p, 1);
    return (size_t)(p - base);
  };
  char* base = nullptr;
  {
    char probe_base[1];
    const size_t bytes = layout(probe_base);  // offsets only: nothing is written through these pointers
    if ((rc = fk_dev_alloc(ctx, (void**)&base, bytes)) != FK_OK) return rc;
    layout(base);
  }
  auto done = [&](int code) {
    cudaStreamSynchronize(st);
    fk_dev_free(ctx, base);
    return code;
  };
#define FK_BVH_TRY(call)                                                   \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) return done(fk_cuda_fail(ctx, e_, #call));      \
  } while (0)
#define FK_BVH_LAUNCHED(what)                                              \
  do {                                                                     \
    if ((rc = fk_after_launch(ctx, what)) != FK_OK) return done(rc);      \
  } while (0)
  auto up = [&](void* dst, const void* src, size_t n) -> cudaError_t {
    return n ? cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) : cudaSuccess;
  };
  FK_BVH_TRY(up(d_pos, mesh->positions.data(), sizeof(float) * mesh->positions.size()));
  FK_BVH_TRY(up(d_nrm, mesh->normals.data(), sizeof(float) * mesh->normals.size()));
  FK_BVH_TRY(up(d_verts, mesh->vertices.data(), sizeof(uint32_t) * mesh->vertices.size()));
  FK_BVH_TRY(up(d_tris, mesh->triangles.data(), sizeof(uint32_t) * mesh->triangles.size()));
  FK_BVH_TRY(cudaMemsetAsync(d_status, 0, 4, st));
  if (nf) {
    bvh_pre_kernel<<<(nf + 255) / 256, 256, 0, st>>>(nf, d_pos, d_verts, d_tris, pc, pm, plo, phi);
    FK_BVH_LAUNCHED("bvh pre");
  }
  {  // identity order
    std::vector<uint32_t> id(nf);
    for (uint32_t i = 0; i < nf; ++i) id[i] = i;
    FK_BVH_TRY(up(perm, id.data(), 4 * (size_t)nf));
  }
  // root box over all positions
  uint32_t* root_w = acc + (size_t)kTaskWords * max_tasks;
  {
    uint32_t w[kBox];
    box_init(w);
    FK_BVH_TRY(up(root_w, w, sizeof(w)));
    if (np) {
      bvh_points_kernel<<<std::min<uint32_t>((np + kThreads - 1) / kThreads, (uint32_t)ctx->sm_count * 4), kThreads, 0,
                      st>>>(d_pos, np, root_w);
      FK_BVH_LAUNCHED("bvh root box");
    }
  }
  uint32_t rw[kBox];
  FK_BVH_TRY(cudaMemcpyAsync(rw, root_w, sizeof(rw), cudaMemcpyDeviceToHost, st));
  FK_BVH_TRY(cudaStreamSynchronize(st));

  std::vector<HNode> hn(1);
  {
    float lo[3], hi[3];
    box_read(rw, lo, hi);
    host_set_box(hn[0], lo, hi);
    hn[0].first = 0;
    hn[0].count = nf;
  }
  std::vector<SmallTask> small;
  struct Level {
    uint32_t b, e, depth, node;
  };
  std::vector<Level> cur;
  int32_t root_ref = 0;  // the tree's root: host node 0, or a subtree
  auto place = [&](uint32_t node, uint32_t b, uint32_t e, uint32_t depth, std::vector<Level>& next) -> int32_t {
    // Src/bvh.cpp:205-213: a node stays a leaf at <= max_tris triangles or at the depth limit
    HNode& h = hn[node];
    h.first = b;
    h.count = e - b;
    if (e - b <= max_tris || depth >= max_depth) return (int32_t)node;
    if (e - b <= kSmall) {
      h.sub = true;
      SmallTask t{b, e, depth, 0, {h.c[0], h.c[1], h.c[2]}, {h.s[0], h.s[1], h.s[2]}};
      small.push_back(t);
      return -(int32_t)small.size();
    }
    next.push_back(Level{b, e, depth, node});
    return (int32_t)node;
  };
  root_ref = place(0, 0, nf, 0, cur);
  std::vector<Chunk> hch;
  std::vector<Task> htasks;
  std::vector<uint32_t> hleft, hoffs, hnode_left, htask_b, hside;
  while (!cur.empty()) {
    const uint32_t nt = (uint32_t)cur.size();
    htasks.resize(nt);
    hch.clear();
    for (uint32_t t = 0; t < nt; ++t) {
      htasks[t] = Task{cur[t].b, cur[t].e, cur[t].depth, 0};
      for (uint32_t b = cur[t].b; b < cur[t].e; b += kChunk) hch.push_back(Chunk{t, b, std::min(b + kChunk, cur[t].e)});
    }
    const uint32_t nc = (uint32_t)hch.size();
    if (nt > max_tasks || nc > max_chunks)
      return done(fk_fail(ctx, FK_ERR_DEVICE, "device BVH build: task overflow"));
    FK_BVH_TRY(up(d_tasks, htasks.data(), sizeof(Task) * nt));
    FK_BVH_TRY(up(d_chunks, hch.data(), sizeof(Chunk) * nc));
    bvh_init_kernel<<<(nt + 127) / 128, 128, 0, st>>>(acc, nt);
    FK_BVH_LAUNCHED("bvh init");
    bvh_centroid_kernel<<<nc, kThreads, 0, st>>>(d_chunks, perm, pc, acc);
    FK_BVH_LAUNCHED("bvh centroids");
    bvh_bucket_kernel<<<nc, kThreads, 0, st>>>(d_chunks, perm, pc, plo, phi, acc);
    FK_BVH_LAUNCHED("bvh buckets");
    bvh_choose_kernel<<<(nt + 63) / 64, 64, 0, st>>>(d_tasks, nt, acc, d_splits);
    FK_BVH_LAUNCHED("bvh choose");
    bvh_side_kernel<<<nc, kThreads, 0, st>>>(d_chunks, perm, pm, plo, phi, d_splits, acc, d_chunk_left);
    FK_BVH_LAUNCHED("bvh sides");
    hleft.resize(nc);
    hside.resize((size_t)nt * kTaskWords);
    FK_BVH_TRY(cudaMemcpyAsync(hleft.data(), d_chunk_left, 4 * (size_t)nc, cudaMemcpyDeviceToHost, st));
    FK_BVH_TRY(cudaMemcpyAsync(hside.data(), acc, 4 * (size_t)nt * kTaskWords, cudaMemcpyDeviceToHost, st));
    FK_BVH_TRY(cudaStreamSynchronize(st));
    // per node: left count; per chunk: its offsets on both sides
    hnode_left.assign(nt, 0);
    htask_b.resize(nt);
    hoffs.resize(2 * (size_t)nc);
    for (uint32_t c = 0; c < nc; ++c) {
      const uint32_t t = hch[c].task;
      hoffs[2 * c] = hnode_left[t];
      hoffs[2 * c + 1] = (hch[c].b - cur[t].b) - hnode_left[t];
      hnode_left[t] += hleft[c];
    }
    for (uint32_t t = 0; t < nt; ++t) htask_b[t] = cur[t].b;
    // chunks of the nodes that split
    std::vector<Chunk> split_chunks;
    std::vector<uint32_t> split_offs;
    for (uint32_t c = 0; c < nc; ++c) {
      const uint32_t t = hch[c].task, n = cur[t].e - cur[t].b;
      if (hnode_left[t] == 0 || hnode_left[t] == n) continue;  // Src/bvh.cpp:248-256: stays a leaf
      split_chunks.push_back(hch[c]);
      split_offs.push_back(hoffs[2 * c]);
      split_offs.push_back(hoffs[2 * c + 1]);
    }
    if (!split_chunks.empty()) {
      const uint32_t ns = (uint32_t)split_chunks.size();
      FK_BVH_TRY(up(d_chunks, split_chunks.data(), sizeof(Chunk) * ns));
      FK_BVH_TRY(up(d_offs, split_offs.data(), 4 * (size_t)ns * 2));
      FK_BVH_TRY(up(d_node_left, hnode_left.data(), 4 * (size_t)nt));
      FK_BVH_TRY(up(d_task_b, htask_b.data(), 4 * (size_t)nt));
      bvh_scatter_kernel<<<ns, kThreads, 0, st>>>(d_chunks, d_node_left, perm, tmp, pm, d_splits, d_offs, d_task_b);
      FK_BVH_LAUNCHED("bvh scatter");
      bvh_copy_back_kernel<<<ns, kThreads, 0, st>>>(d_chunks, tmp, perm);
      FK_BVH_LAUNCHED("bvh copy back");
    }
    std::vector<Level> next;
    for (uint32_t t = 0; t < nt; ++t) {
      const Level L = cur[t];
      const uint32_t n = L.e - L.b, nl = hnode_left[t];
      if (nl == 0 || nl == n) continue;  // leaf, as placed
      float llo[3], lhi[3], rlo[3], rhi[3];
      box_read(&hside[(size_t)t * kTaskWords + kLeftOff], llo, lhi);
      box_read(&hside[(size_t)t * kTaskWords + kRightOff], rlo, rhi);
      const uint32_t li = (uint32_t)hn.size();
      hn.emplace_back();
      hn.emplace_back();
      host_set_box(hn[li], llo, lhi);
      host_set_box(hn[li + 1], rlo, rhi);
      hn[L.node].leaf = false;
      hn[L.node].count = 0;
      const int32_t a = place(li, L.b, L.b + nl, L.depth + 1, next);
      const int32_t b = place(li + 1, L.b + nl, L.e, L.depth + 1, next);
      hn[L.node].kid[0] = a;
      hn[L.node].kid[1] = b;
    }
    cur.swap(next);
  }
  // subtrees
  const uint32_t nsm = (uint32_t)small.size();
  std::vector<DNode> roots(nsm);
  SmallTask* d_small = nullptr;
  DNode* d_roots = nullptr;
  auto done2 = [&](int code) {
    fk_dev_free(ctx, d_small);
    fk_dev_free(ctx, d_roots);
    return done(code);
  };
  if (nsm) {
    if ((rc = fk_dev_alloc(ctx, (void**)&d_small, sizeof(SmallTask) * nsm)) != FK_OK ||
        (rc = fk_dev_alloc(ctx, (void**)&d_roots, sizeof(DNode) * nsm)) != FK_OK)
      return done2(rc);
    cudaError_t e = up(d_small, small.data(), sizeof(SmallTask) * nsm);
    if (e != cudaSuccess) return done2(fk_cuda_fail(ctx, e, "device BVH build: subtrees"));
    bvh_small_kernel<<<(nsm + 63) / 64, 64, 0, st>>>(d_small, nsm, perm, scratch, frames, pc, pm, plo, phi, dnodes,
                                                max_tris, max_depth, d_status);
    if ((rc = fk_after_launch(ctx, "bvh subtrees")) != FK_OK) return done2(rc);
    bvh_small_roots_kernel<<<(nsm + 127) / 128, 128, 0, st>>>(d_small, nsm, dnodes, d_roots);
    if ((rc = fk_after_launch(ctx, "bvh subtree roots")) != FK_OK) return done2(rc);
    e = cudaMemcpyAsync(roots.data(), d_roots, sizeof(DNode) * nsm, cudaMemcpyDeviceToHost, st);
    uint32_t status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, d_status, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done2(fk_cuda_fail(ctx, e, "device BVH build: subtrees"));
    if (status) return done2(fk_fail(ctx, FK_ERR_DEVICE, "device BVH build: subtree check failed"));
  }
  // top of the tree: boxes from the children (Src/bvh.cpp:266-276), sizes, preorder
  auto kid_box = [&](int32_t r, float c[3], float s[3], uint32_t& size) {
    if (r >= 0) {
      for (int a = 0; a < 3; ++a) { c[a] = hn[r].c[a]; s[a] = hn[r].s[a]; }
      size = hn[r].size;
    } else {
      const DNode& d = roots[-r - 1];
      for (int a = 0; a < 3; ++a) { c[a] = d.c[a]; s[a] = d.s[a]; }
      size = d.size;
    }
  };
  for (size_t i = hn.size(); i-- > 0;) {
    HNode& h = hn[i];
    if (h.leaf) continue;
    float ac[3], as[3], bc[3], bs[3];
    uint32_t sa, sb;
    kid_box(h.kid[0], ac, as, sa);
    kid_box(h.kid[1], bc, bs, sb);
    for (int a = 0; a < 3; ++a) {
      const float lo = bvh::fmin(ac[a] - as[a], bc[a] - bs[a]);
      const float hi = bvh::fmax(ac[a] + as[a], bc[a] + bs[a]);
      h.c[a] = (hi + lo) * 0.5f;
      h.s[a] = (hi - lo) * 0.5f;
    }
    h.size = 1 + sa + sb;
  }
  uint32_t nn = 0;
  std::vector<FlatRec> recs;
  if (root_ref < 0) {
    small[-root_ref - 1].pre = 0;
    nn = roots[-root_ref - 1].size;
  } else if (nf > 0) {
    nn = hn[0].size;
    // hn is in creation order: parents before children
    hn[0].pre = 0;
    for (size_t i = 0; i < hn.size(); ++i) {
      HNode& h = hn[i];
      if (h.sub) continue;
      FlatRec r{};
      const uint32_t start = 3 * h.first, end = h.leaf ? 3 * (h.first + h.count) : 3 * h.first;
      r.lo = make_float4(h.c[0] - h.s[0], h.c[1] - h.s[1], h.c[2] - h.s[2], u2f(start));
      r.hi = make_float4(h.c[0] + h.s[0], h.c[1] + h.s[1], h.c[2] + h.s[2], u2f(end));
      r.pre = h.pre;
      r.jump = h.pre + h.size;
      recs.push_back(r);
      if (!h.leaf) {
        float c[3], s[3];
        uint32_t ls;
        kid_box(h.kid[0], c, s, ls);
        const uint32_t pre_l = h.pre + 1, pre_r = h.pre + 1 + ls;
        if (h.kid[0] >= 0) hn[h.kid[0]].pre = pre_l;
        else small[-h.kid[0] - 1].pre = pre_l;
        if (h.kid[1] >= 0) hn[h.kid[1]].pre = pre_r;
        else small[-h.kid[1] - 1].pre = pre_r;
      }
    }
  }
  // outputs
  DevBvh o;
  o.node_count = nn;
  o.corner_count = 3 * nf;
  o.triangle_count = nf;
  auto free_out = [&]() {
    fk_dev_free(ctx, o.lo);
    fk_dev_free(ctx, o.hi);
    fk_dev_free(ctx, o.jump);
    fk_dev_free(ctx, o.pos4);
    fk_dev_free(ctx, o.nrm4);
  };
  if ((rc = fk_dev_alloc(ctx, (void**)&o.lo, sizeof(float4) * (nn ? nn : 1))) != FK_OK ||
      (rc = fk_dev_alloc(ctx, (void**)&o.hi, sizeof(float4) * (nn ? nn : 1))) != FK_OK ||
      (rc = fk_dev_alloc(ctx, (void**)&o.jump, sizeof(uint32_t) * (nn ? nn : 1))) != FK_OK ||
      (rc = fk_dev_alloc(ctx, (void**)&o.pos4, sizeof(float4) * 3 * F)) != FK_OK ||
      (rc = fk_dev_alloc(ctx, (void**)&o.nrm4, sizeof(float4) * 3 * F)) != FK_OK) {
    free_out();
    return done2(rc);
  }
  for (const FlatRec& r : recs)
    if (r.pre >= nn) {
      free_out();
      return done2(fk_fail(ctx, FK_ERR_DEVICE, "device BVH build: node index out of range"));
    }
  FlatRec* d_recs = nullptr;
  if (!recs.empty()) {
    if ((rc = fk_dev_alloc(ctx, (void**)&d_recs, sizeof(FlatRec) * recs.size())) != FK_OK) {
      free_out();
      return done2(rc);
    }
    cudaError_t e = up(d_recs, recs.data(), sizeof(FlatRec) * recs.size());
    if (e == cudaSuccess) {
      bvh_host_records_kernel<<<((uint32_t)recs.size() + 127) / 128, 128, 0, st>>>(d_recs, (uint32_t)recs.size(), o.lo,
                                                                               o.hi, o.jump);
      rc = fk_after_launch(ctx, "bvh top records");
    } else {
      rc = fk_cuda_fail(ctx, e, "device BVH build: top records");
    }
  }
  if (rc == FK_OK && nsm) {
    cudaError_t e = up(d_small, small.data(), sizeof(SmallTask) * nsm);  // with their preorder indices
    if (e == cudaSuccess) {
      // the subtree stacks are free again: their frames hold the walk's (slot, preorder) pairs
      bvh_small_flatten_kernel<<<(nsm + 63) / 64, 64, 0, st>>>(d_small, nsm, dnodes, reinterpret_cast<uint32_t*>(frames),
                                                            o.lo, o.hi, o.jump, nn, d_status);
      rc = fk_after_launch(ctx, "bvh flatten");
    } else {
      rc = fk_cuda_fail(ctx, e, "device BVH build: flatten");
    }
  }
  if (rc == FK_OK && nf) {
    bvh_corners_kernel<<<(nf + 255) / 256, 256, 0, st>>>(nf, perm, d_tris, d_verts, d_pos, d_nrm, o.pos4, o.nrm4);
    rc = fk_after_launch(ctx, "bvh corners");
  }
  if (rc == FK_OK) {
    uint32_t status = 0;
    cudaError_t e = cudaMemcpyAsync(&status, d_status, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "device BVH build");
    else if (status) rc = fk_fail(ctx, FK_ERR_DEVICE, "device BVH build: flatten check failed");
  }
  fk_dev_free(ctx, d_recs);
  if (rc != FK_OK) {
    free_out();
    return done2(rc);
  }
#undef FK_BVH_TRY
#undef FK_BVH_LAUNCHED
  *out = o;
  return done2(FK_OK);
}

}  // namespace fk
