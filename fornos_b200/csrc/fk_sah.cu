// Surface-area inner tree built on the device, record for record the tree
// of the host builder (fk_tree.cpp; shared rules in fk_sah_rules.h).
//
// Nodes of more than kSmall leaves are split level by level.  Per level,
// blocks of up to kChunk leaves reduce each node's box and centre bounds, bin
// its leaves (3 axes x 32 bins in shared memory, flushed with atomics), one
// warp per node sweeps the bins for the split, and blocks stably partition
// the node's index range (per-chunk left counts; the host turns them into
// offsets).  Subtrees of at most kSmall leaves are then built one per warp,
// depth first, with their leaf boxes, indices, bins and stack in shared
// memory.  Minima and maxima are taken over float keys and sums are integer
// sums, so no result depends on the order of the atomics.
//
// Index arrays hold flattened node indices (leaf boxes are read from the
// scene's node_lo / node_hi), start in ascending order and are only ever
// partitioned stably, so every node's leaves are in flattened order, which is
// what the fallback split and the host builder assume.
#include <algorithm>
#include <vector>

#include "fk_internal.h"
#include "fk_sah_rules.h"

namespace fk {
namespace {

using sah::bin_of;
using sah::bin_scale;
using sah::centre;
using sah::half_area;
using sah::key;
using sah::kmax;
using sah::kmin;
using sah::unkey;
constexpr int kBins = sah::kBins;

constexpr uint32_t kSmall = 256;      // subtrees of at most this many leaves: one warp each
constexpr uint32_t kChunk = 2048;     // leaves per block in the level passes
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kBinWords = 8;          // lo keys xyz, hi keys xyz, triangles, leaves
constexpr int kNodeBins = 3 * kBins * kBinWords;
constexpr int kAccWords = 12;         // box lo keys, box hi keys, centre lo keys, centre hi keys
constexpr uint32_t kNoSlot = 0xffffffffu;
constexpr int kSmallWarps = 4;
constexpr int kStack = 16;            // smaller child first: at most log2(kSmall) + 1 entries

// A node to split: leaves [b, e) of index array `src`, its record `rec`, its
// level (root = 1) and the record slot (record * 2 + side) its box goes to.
struct Task {
  uint32_t b, e, rec, level, slot, src;
};
struct Chunk {
  uint32_t task, b, e;
};
struct Split {
  int axis, bin;
  uint32_t nleft;
  float cmin, scale;  // of the split axis
  uint32_t pad[3];
};

__host__ __device__ constexpr bool acc_is_min(int j) { return j < 3 || (j >= 6 && j < 9); }

__device__ __forceinline__ uint32_t wmin(uint32_t v) {
  for (int d = 16; d > 0; d >>= 1) v = kmin(v, __shfl_xor_sync(0xffffffffu, v, d));
  return v;
}
__device__ __forceinline__ uint32_t wmax(uint32_t v) {
  for (int d = 16; d > 0; d >>= 1) v = kmax(v, __shfl_xor_sync(0xffffffffu, v, d));
  return v;
}

__device__ __forceinline__ float comp(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ uint32_t tris_of(const float4& l, const float4& h) {
  return (__float_as_uint(h.w) - __float_as_uint(l.w)) / 3u;
}

// One child slot of a 2-wide record (layout of fk_tree.cpp's put_record):
// floats 0-3 / 4-7 the left / right child's x and y bounds, 8-9 / 10-11 its z
// bounds, ints 12 / 13 its ref, 14 / 15 its triangle count.
__device__ __forceinline__ void put_slot(float4* wide, uint32_t slot, const float b[6], int32_t ref, int32_t cnt) {
  float* w = reinterpret_cast<float*>(wide + 4 * (size_t)(slot >> 1));
  const int s = (int)(slot & 1u);
  w[4 * s + 0] = b[0];
  w[4 * s + 1] = b[1];
  w[4 * s + 2] = b[2];
  w[4 * s + 3] = b[3];
  w[8 + 2 * s] = b[4];
  w[9 + 2 * s] = b[5];
  int32_t* wi = reinterpret_cast<int32_t*>(w);
  wi[12 + s] = ref;
  wi[14 + s] = cnt;
}

// Box from keys v[0..5] (lo xyz, hi xyz) in slot order.
__device__ __forceinline__ void box_of(const uint32_t* v, float b[6]) {
  b[0] = unkey(v[0]);
  b[1] = unkey(v[3]);
  b[2] = unkey(v[1]);
  b[3] = unkey(v[4]);
  b[4] = unkey(v[2]);
  b[5] = unkey(v[5]);
}

struct Choice {
  int axis, bin;
  uint32_t nleft;
};

// Split choice from a node's bins ([3][kBins][kBinWords], shared or global
// memory), the whole warp calling: lane q holds bin q; suffix and prefix
// merges are shuffle scans, the first strict minimum over (axis, bin) wins.
// No candidate: axis -1 and the first half of the n leaves.
__device__ Choice sweep(const uint32_t* bins, const float scale[3], uint32_t n) {
  const int lane = threadIdx.x & 31;
  double best = 1e300;
  Choice ch{-1, 0, n / 2};
  for (int k = 0; k < 3; ++k) {
    if (!(scale[k] > 0.0f)) continue;
    const uint32_t* bb = bins + (k * kBins + lane) * kBinWords;
    uint32_t b[6];
    for (int j = 0; j < 6; ++j) b[j] = bb[j];
    const uint32_t t = bb[6], c = bb[7];
    uint32_t r[6], rt = t;
    for (int j = 0; j < 6; ++j) r[j] = b[j];
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t o[6];
      for (int j = 0; j < 6; ++j) o[j] = __shfl_down_sync(0xffffffffu, r[j], d);
      const uint32_t ot = __shfl_down_sync(0xffffffffu, rt, d);
      if (lane + d < 32) {
        for (int j = 0; j < 3; ++j) r[j] = kmin(r[j], o[j]);
        for (int j = 3; j < 6; ++j) r[j] = kmax(r[j], o[j]);
        rt += ot;
      }
    }
    const double rcost =
        rt > 0 ? half_area(unkey(r[0]), unkey(r[3]), unkey(r[1]), unkey(r[4]), unkey(r[2]), unkey(r[5])) * (double)rt
               : 0.0;
    uint32_t l[6], lt = t, lc = c;
    for (int j = 0; j < 6; ++j) l[j] = b[j];
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t o[6];
      for (int j = 0; j < 6; ++j) o[j] = __shfl_up_sync(0xffffffffu, l[j], d);
      const uint32_t ot = __shfl_up_sync(0xffffffffu, lt, d), oc = __shfl_up_sync(0xffffffffu, lc, d);
      if (lane >= d) {
        for (int j = 0; j < 3; ++j) l[j] = kmin(l[j], o[j]);
        for (int j = 3; j < 6; ++j) l[j] = kmax(l[j], o[j]);
        lt += ot;
        lc += oc;
      }
    }
    const double rnext = __shfl_down_sync(0xffffffffu, rcost, 1);
    double cost = 1e308;  // not a candidate
    if (lane < kBins - 1 && lt != 0 && rnext != 0.0)
      cost = half_area(unkey(l[0]), unkey(l[3]), unkey(l[1]), unkey(l[4]), unkey(l[2]), unkey(l[5])) * (double)lt +
             rnext;
    int arg = lane;
    for (int d = 16; d > 0; d >>= 1) {
      const double oc = __shfl_xor_sync(0xffffffffu, cost, d);
      const int oa = __shfl_xor_sync(0xffffffffu, arg, d);
      if (oc < cost || (oc == cost && oa < arg)) {
        cost = oc;
        arg = oa;
      }
    }
    const uint32_t left = __shfl_sync(0xffffffffu, lc, arg);
    if (cost < best) {
      best = cost;
      ch.axis = k;
      ch.bin = arg;
      ch.nleft = left;
    }
  }
  return ch;
}

__device__ __forceinline__ void centre_bounds(const uint32_t* acc, float cmin[3], float scale[3]) {
  for (int k = 0; k < 3; ++k) {
    cmin[k] = unkey(acc[6 + k]);
    scale[k] = bin_scale(unkey(acc[9 + k]) - cmin[k]);
  }
}

// ------------------------------------------------------------ level passes
__global__ void sah_init_kernel(uint32_t* acc, uint32_t* bins, uint32_t nt) {
  const size_t na = (size_t)nt * kAccWords, nb = (size_t)nt * kNodeBins;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < na + nb; i += (size_t)gridDim.x * blockDim.x) {
    if (i < na) acc[i] = acc_is_min((int)(i % kAccWords)) ? 0xffffffffu : 0u;
    else bins[i - na] = ((i - na) % kBinWords) < 3 ? 0xffffffffu : 0u;
  }
}

__global__ void __launch_bounds__(kThreads) sah_bounds_kernel(const Chunk* chunks, const uint32_t* __restrict__ perm,
                                                          const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                          uint32_t* acc) {
  const Chunk c = chunks[blockIdx.x];
  uint32_t v[kAccWords];
  for (int j = 0; j < kAccWords; ++j) v[j] = acc_is_min(j) ? 0xffffffffu : 0u;
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += kThreads) {
    const uint32_t f = perm[i];
    const float4 l = lo[f], h = hi[f];
    for (int k = 0; k < 3; ++k) {
      const float a = comp(l, k), z = comp(h, k);
      const uint32_t ck = key(centre(a, z));
      v[k] = kmin(v[k], key(a));
      v[3 + k] = kmax(v[3 + k], key(z));
      v[6 + k] = kmin(v[6 + k], ck);
      v[9 + k] = kmax(v[9 + k], ck);
    }
  }
  __shared__ uint32_t red[kWarps][kAccWords];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = 0; j < kAccWords; ++j) v[j] = acc_is_min(j) ? wmin(v[j]) : wmax(v[j]);
  if (lane == 0)
    for (int j = 0; j < kAccWords; ++j) red[warp][j] = v[j];
  __syncthreads();
  if (threadIdx.x < kAccWords) {
    const int j = threadIdx.x;
    uint32_t r = red[0][j];
    for (int w = 1; w < kWarps; ++w) r = acc_is_min(j) ? kmin(r, red[w][j]) : kmax(r, red[w][j]);
    if (acc_is_min(j)) atomicMin(&acc[(size_t)c.task * kAccWords + j], r);
    else atomicMax(&acc[(size_t)c.task * kAccWords + j], r);
  }
}

__global__ void __launch_bounds__(kThreads) sah_bin_kernel(const Chunk* chunks, const uint32_t* __restrict__ perm,
                                                       const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                       const uint32_t* acc, uint32_t* bins) {
  __shared__ uint32_t sb[kNodeBins];
  for (int w = threadIdx.x; w < kNodeBins; w += kThreads) sb[w] = (w % kBinWords) < 3 ? 0xffffffffu : 0u;
  const Chunk c = chunks[blockIdx.x];
  float cmin[3], scale[3];
  centre_bounds(acc + (size_t)c.task * kAccWords, cmin, scale);
  __syncthreads();
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += kThreads) {
    const uint32_t f = perm[i];
    const float4 l = lo[f], h = hi[f];
    const uint32_t t = tris_of(l, h);
    for (int k = 0; k < 3; ++k) {
      if (!(scale[k] > 0.0f)) continue;
      const int q = bin_of(centre(comp(l, k), comp(h, k)), cmin[k], scale[k]);
      uint32_t* s = sb + (k * kBins + q) * kBinWords;
      atomicMin(s + 0, key(l.x));
      atomicMin(s + 1, key(l.y));
      atomicMin(s + 2, key(l.z));
      atomicMax(s + 3, key(h.x));
      atomicMax(s + 4, key(h.y));
      atomicMax(s + 5, key(h.z));
      atomicAdd(s + 6, t);
      atomicAdd(s + 7, 1u);
    }
  }
  __syncthreads();
  uint32_t* g = bins + (size_t)c.task * kNodeBins;
  for (int w = threadIdx.x; w < kNodeBins; w += kThreads) {
    const int f = w % kBinWords;
    if (sb[w - f + 7] == 0) continue;  // empty bin
    if (f < 3) atomicMin(g + w, sb[w]);
    else if (f < 6) atomicMax(g + w, sb[w]);
    else atomicAdd(g + w, sb[w]);
  }
}

__global__ void __launch_bounds__(kThreads) sah_split_kernel(const Task* tasks, uint32_t nt, const uint32_t* acc,
                                                         const uint32_t* bins, Split* splits, float4* wide) {
  const uint32_t t = (blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (t >= nt) return;  // whole warps
  const int lane = threadIdx.x & 31;
  const Task tk = tasks[t];
  const uint32_t* a = acc + (size_t)t * kAccWords;
  if (tk.slot != kNoSlot && lane == 0) {
    float b[6];
    box_of(a, b);
    put_slot(wide, tk.slot, b, (int32_t)tk.rec, 0);
  }
  float cmin[3], scale[3];
  centre_bounds(a, cmin, scale);
  const Choice ch = sweep(bins + (size_t)t * kNodeBins, scale, tk.e - tk.b);
  if (lane == 0) {
    Split s{};
    s.axis = ch.axis;
    s.bin = ch.bin;
    s.nleft = ch.nleft;
    s.cmin = ch.axis >= 0 ? cmin[ch.axis] : 0.0f;
    s.scale = ch.axis >= 0 ? scale[ch.axis] : 0.0f;
    splits[t] = s;
  }
}

__device__ __forceinline__ bool goes_left(const Split& s, uint32_t pos, const float4* lo, const float4* hi,
                                          uint32_t f) {
  if (s.axis < 0) return pos < s.nleft;
  const float4 l = lo[f], h = hi[f];
  return bin_of(centre(comp(l, s.axis), comp(h, s.axis)), s.cmin, s.scale) <= s.bin;
}

__global__ void __launch_bounds__(kThreads) sah_count_kernel(const Chunk* chunks, const Task* tasks,
                                                         const uint32_t* __restrict__ perm,
                                                         const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                         const Split* splits, uint32_t* chunk_left) {
  const Chunk c = chunks[blockIdx.x];
  const Split s = splits[c.task];
  const uint32_t tb = tasks[c.task].b;
  uint32_t n = 0;
  for (uint32_t i = c.b + threadIdx.x; i < c.e; i += kThreads) n += goes_left(s, i - tb, lo, hi, perm[i]) ? 1u : 0u;
  for (int d = 16; d > 0; d >>= 1) n += __shfl_xor_sync(0xffffffffu, n, d);
  __shared__ uint32_t red[kWarps];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t sum = 0;
    for (int w = 0; w < kWarps; ++w) sum += red[w];
    chunk_left[blockIdx.x] = sum;
  }
}

// offs[2 c], offs[2 c + 1]: leaves of the chunk's node that earlier chunks
// send left / right.
__global__ void __launch_bounds__(kThreads) sah_scatter_kernel(const Chunk* chunks, const Task* tasks,
                                                           const uint32_t* __restrict__ perm_in, uint32_t* perm_out,
                                                           const float4* __restrict__ lo,
                                                           const float4* __restrict__ hi, const Split* splits,
                                                           const uint32_t* offs) {
  const Chunk c = chunks[blockIdx.x];
  const Task tk = tasks[c.task];
  const Split s = splits[c.task];
  uint32_t lbase = tk.b + offs[2 * blockIdx.x], rbase = tk.b + s.nleft + offs[2 * blockIdx.x + 1];
  __shared__ uint32_t wl[kWarps], wr[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t below = (1u << lane) - 1u;
  for (uint32_t base = c.b; base < c.e; base += kThreads) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < c.e;
    const uint32_t f = valid ? perm_in[i] : 0u;
    const bool left = valid && goes_left(s, i - tk.b, lo, hi, f);
    const bool right = valid && !left;
    const uint32_t bl = __ballot_sync(0xffffffffu, left), br = __ballot_sync(0xffffffffu, right);
    if (lane == 0) {
      wl[warp] = __popc(bl);
      wr[warp] = __popc(br);
    }
    __syncthreads();
    uint32_t pl = 0, pr = 0, tl = 0, tr = 0;
    for (int w = 0; w < kWarps; ++w) {
      if (w < warp) {
        pl += wl[w];
        pr += wr[w];
      }
      tl += wl[w];
      tr += wr[w];
    }
    if (left) perm_out[lbase + pl + __popc(bl & below)] = f;
    if (right) perm_out[rbase + pr + __popc(br & below)] = f;
    lbase += tl;
    rbase += tr;
    __syncthreads();
  }
}

// ------------------------------------------------------------ small subtrees
struct WarpSmem {
  float4 lo[kSmall];
  float4 hi[kSmall];
  uint32_t bins[kNodeBins];
  uint16_t idx[kSmall], tmp[kSmall];
  uint32_t stack[kStack][5];  // b, e, rec, level, slot
};
constexpr size_t kSmallSmem = sizeof(WarpSmem) * kSmallWarps;

// status bits: 1 = a partition disagreed with its bins, 2 = stack overflow
__global__ void __launch_bounds__(kSmallWarps * 32) sah_small_kernel(const Task* tasks, uint32_t ns,
                                                                 const uint32_t* perm0, const uint32_t* perm1,
                                                                 const float4* __restrict__ lo,
                                                                 const float4* __restrict__ hi, float4* wide,
                                                                 uint32_t* depth, uint32_t* status) {
  extern __shared__ float4 smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& S = reinterpret_cast<WarpSmem*>(smem_raw)[warp];
  const uint32_t below = (1u << lane) - 1u;
  for (uint32_t t = blockIdx.x * kSmallWarps + warp; t < ns; t += gridDim.x * kSmallWarps) {
    const Task tk = tasks[t];
    const uint32_t* perm = tk.src ? perm1 : perm0;
    const uint32_t n = tk.e - tk.b;  // 1 .. kSmall
    for (uint32_t i = lane; i < n; i += 32) {
      const uint32_t f = perm[tk.b + i];
      S.lo[i] = lo[f];
      S.hi[i] = hi[f];
      S.idx[i] = (uint16_t)i;
    }
    __syncwarp();
    uint32_t nb = 0, ne = n, rec = tk.rec, level = tk.level, slot = tk.slot, maxlevel = 0;
    int sp = 0;
    bool failed = false;
    while (true) {
      if (ne - nb == 1) {
        if (lane == 0) {
          const uint32_t j = S.idx[nb];
          const float4 l = S.lo[j], h = S.hi[j];
          const float b[6] = {l.x, h.x, l.y, h.y, l.z, h.z};
          put_slot(wide, slot, b, -(int32_t)perm[tk.b + j] - 1, (int32_t)tris_of(l, h));
        }
        maxlevel = max(maxlevel, level);
      } else {
        uint32_t v[kAccWords];
        for (int j = 0; j < kAccWords; ++j) v[j] = acc_is_min(j) ? 0xffffffffu : 0u;
        for (uint32_t i = nb + lane; i < ne; i += 32) {
          const uint32_t j = S.idx[i];
          const float4 l = S.lo[j], h = S.hi[j];
          for (int k = 0; k < 3; ++k) {
            const float a = comp(l, k), z = comp(h, k);
            const uint32_t ck = key(centre(a, z));
            v[k] = kmin(v[k], key(a));
            v[3 + k] = kmax(v[3 + k], key(z));
            v[6 + k] = kmin(v[6 + k], ck);
            v[9 + k] = kmax(v[9 + k], ck);
          }
        }
        for (int j = 0; j < kAccWords; ++j) v[j] = acc_is_min(j) ? wmin(v[j]) : wmax(v[j]);
        if (slot != kNoSlot && lane == 0) {
          float b[6];
          box_of(v, b);
          put_slot(wide, slot, b, (int32_t)rec, 0);
        }
        float cmin[3], scale[3];
        centre_bounds(v, cmin, scale);
        for (int w = lane; w < kNodeBins; w += 32) S.bins[w] = (w % kBinWords) < 3 ? 0xffffffffu : 0u;
        __syncwarp();
        for (uint32_t i = nb + lane; i < ne; i += 32) {
          const uint32_t j = S.idx[i];
          const float4 l = S.lo[j], h = S.hi[j];
          const uint32_t tr = tris_of(l, h);
          for (int k = 0; k < 3; ++k) {
            if (!(scale[k] > 0.0f)) continue;
            const int q = bin_of(centre(comp(l, k), comp(h, k)), cmin[k], scale[k]);
            uint32_t* s = S.bins + (k * kBins + q) * kBinWords;
            atomicMin(s + 0, key(l.x));
            atomicMin(s + 1, key(l.y));
            atomicMin(s + 2, key(l.z));
            atomicMax(s + 3, key(h.x));
            atomicMax(s + 4, key(h.y));
            atomicMax(s + 5, key(h.z));
            atomicAdd(s + 6, tr);
            atomicAdd(s + 7, 1u);
          }
        }
        __syncwarp();
        const Choice ch = sweep(S.bins, scale, ne - nb);
        const float pc = ch.axis >= 0 ? cmin[ch.axis] : 0.0f, ps = ch.axis >= 0 ? scale[ch.axis] : 0.0f;
        uint32_t nl = 0, nr = 0;
        for (uint32_t base = nb; base < ne; base += 32) {
          const uint32_t i = base + lane;
          const bool valid = i < ne;
          const uint32_t j = valid ? S.idx[i] : 0u;
          bool left = false;
          if (valid) {
            if (ch.axis >= 0) {
              const float4 l = S.lo[j], h = S.hi[j];
              left = bin_of(centre(comp(l, ch.axis), comp(h, ch.axis)), pc, ps) <= ch.bin;
            } else {
              left = i - nb < ch.nleft;
            }
          }
          const bool right = valid && !left;
          const uint32_t bl = __ballot_sync(0xffffffffu, left), br = __ballot_sync(0xffffffffu, right);
          if (left && nb + nl + __popc(bl & below) < ne) S.tmp[nb + nl + __popc(bl & below)] = (uint16_t)j;
          if (right && nb + ch.nleft + nr + __popc(br & below) < ne)
            S.tmp[nb + ch.nleft + nr + __popc(br & below)] = (uint16_t)j;
          nl += __popc(bl);
          nr += __popc(br);
        }
        if (nl != ch.nleft || nl == 0 || nr == 0) {
          if (lane == 0) atomicOr(status, 1u);
          failed = true;
          break;
        }
        __syncwarp();
        for (uint32_t i = nb + lane; i < ne; i += 32) S.idx[i] = S.tmp[i];
        __syncwarp();
        const uint32_t m = nb + ch.nleft;
        // children: left [nb, m) at rec + 1, right [m, ne) at rec + nleft;
        // continue with the smaller, push the larger
        const uint32_t cl[5] = {nb, m, rec + 1, level + 1, 2 * rec};
        const uint32_t cr[5] = {m, ne, rec + ch.nleft, level + 1, 2 * rec + 1};
        const bool left_small = (m - nb) <= (ne - m);
        const uint32_t* go = left_small ? cl : cr;
        const uint32_t* keep = left_small ? cr : cl;
        if (sp == kStack) {
          if (lane == 0) atomicOr(status, 2u);
          failed = true;
          break;
        }
        if (lane == 0)
          for (int q = 0; q < 5; ++q) S.stack[sp][q] = keep[q];
        ++sp;
        nb = go[0];
        ne = go[1];
        rec = go[2];
        level = go[3];
        slot = go[4];
        __syncwarp();
        continue;
      }
      if (sp == 0) break;
      --sp;
      __syncwarp();
      nb = S.stack[sp][0];
      ne = S.stack[sp][1];
      rec = S.stack[sp][2];
      level = S.stack[sp][3];
      slot = S.stack[sp][4];
      __syncwarp();
    }
    if (!failed && lane == 0) atomicMax(depth, maxlevel);
    __syncwarp();
  }
}

template <class T>
T* carve(char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += (sizeof(T) * count + 255) & ~(size_t)255;
  return r;
}

}  // namespace

int build_sah_device(fk_ctx* ctx, const float4* lo, const float4* hi, const std::vector<uint32_t>& leaves,
                     float4** out_wide, uint32_t* out_depth) {
  *out_wide = nullptr;
  *out_depth = 0;
  const uint32_t L = (uint32_t)leaves.size();
  if (L < 2) {
    *out_depth = 1;
    return FK_OK;
  }
  const uint32_t max_tasks = L / (kSmall + 1) + 1;
  const uint32_t max_chunks = L / kChunk + max_tasks + 1;
  // scratch: two index arrays, per-node accumulators / bins / splits, tasks,
  // chunks, chunk counts and offsets, two result words (carved in this order)
  const size_t parts[] = {4 * (size_t)L,
                          4 * (size_t)L,
                          4 * (size_t)max_tasks * kAccWords,
                          4 * (size_t)max_tasks * kNodeBins,
                          sizeof(Split) * (size_t)max_tasks,
                          sizeof(Task) * (size_t)max_tasks,
                          sizeof(Chunk) * (size_t)max_chunks,
                          4 * (size_t)max_chunks,
                          8 * (size_t)max_chunks,
                          8};
  size_t bytes = 0;
  for (size_t b : parts) bytes += (b + 255) & ~(size_t)255;
  char* base = nullptr;
  int rc = fk_dev_alloc(ctx, (void**)&base, bytes);
  if (rc != FK_OK) return rc;
  float4* wide = nullptr;
  rc = fk_dev_alloc(ctx, (void**)&wide, sizeof(float4) * 4 * (size_t)(L - 1));
  if (rc != FK_OK) {
    fk_dev_free(ctx, base);
    return rc;
  }
  char* p = base;
  uint32_t* perm[2] = {carve<uint32_t>(p, L), carve<uint32_t>(p, L)};
  uint32_t* acc = carve<uint32_t>(p, (size_t)max_tasks * kAccWords);
  uint32_t* bins = carve<uint32_t>(p, (size_t)max_tasks * kNodeBins);
  Split* splits = carve<Split>(p, max_tasks);
  Task* tasks = carve<Task>(p, max_tasks);
  Chunk* chunks = carve<Chunk>(p, max_chunks);
  uint32_t* chunk_left = carve<uint32_t>(p, max_chunks);
  uint32_t* offs = carve<uint32_t>(p, 2 * (size_t)max_chunks);
  uint32_t* words = carve<uint32_t>(p, 2);  // depth, status
  auto fail = [&](int code) {
    cudaStreamSynchronize(ctx->stream);
    fk_dev_free(ctx, base);
    fk_dev_free(ctx, wide);
    return code;
  };
#define FK_SAH_TRY(call)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return fail(fk_cuda_fail(ctx, e_, #call)); \
  } while (0)
  cudaStream_t st = ctx->stream;
  FK_SAH_TRY(cudaMemcpyAsync(perm[0], leaves.data(), 4 * (size_t)L, cudaMemcpyHostToDevice, st));
  FK_SAH_TRY(cudaMemsetAsync(words, 0, 8, st));

  std::vector<Task> cur, small;
  const Task root{0, L, 0, 1, kNoSlot, 0};
  if (L <= kSmall) small.push_back(root);
  else cur.push_back(root);
  int src = 0;
  std::vector<Chunk> hchunks;
  std::vector<Split> hsplits;
  std::vector<uint32_t> hleft, hoffs;
  while (!cur.empty()) {
    if (cur[0].level > kMaxOrderedDepth) {  // leaves below the ordered traversals' depth: no tree
      *out_depth = cur[0].level + 1;
      return fail(FK_OK);
    }
    const uint32_t nt = (uint32_t)cur.size();
    hchunks.clear();
    for (uint32_t t = 0; t < nt; ++t)
      for (uint32_t b = cur[t].b; b < cur[t].e; b += kChunk) hchunks.push_back({t, b, std::min(b + kChunk, cur[t].e)});
    const uint32_t nc = (uint32_t)hchunks.size();
    if (nt > max_tasks || nc > max_chunks) return fail(fk_fail(ctx, FK_ERR_DEVICE, "surface-area build: task overflow"));
    FK_SAH_TRY(cudaMemcpyAsync(tasks, cur.data(), sizeof(Task) * nt, cudaMemcpyHostToDevice, st));
    FK_SAH_TRY(cudaMemcpyAsync(chunks, hchunks.data(), sizeof(Chunk) * nc, cudaMemcpyHostToDevice, st));
    const uint32_t init_blocks = std::min<uint32_t>((uint32_t)(((size_t)nt * (kAccWords + kNodeBins) + kThreads - 1) / kThreads),
                                                    (uint32_t)ctx->sm_count * 8);
    sah_init_kernel<<<init_blocks, kThreads, 0, st>>>(acc, bins, nt);
    if ((rc = fk_after_launch(ctx, "sah init")) != FK_OK) return fail(rc);
    sah_bounds_kernel<<<nc, kThreads, 0, st>>>(chunks, perm[src], lo, hi, acc);
    if ((rc = fk_after_launch(ctx, "sah bounds")) != FK_OK) return fail(rc);
    sah_bin_kernel<<<nc, kThreads, 0, st>>>(chunks, perm[src], lo, hi, acc, bins);
    if ((rc = fk_after_launch(ctx, "sah bins")) != FK_OK) return fail(rc);
    sah_split_kernel<<<(nt * 32 + kThreads - 1) / kThreads, kThreads, 0, st>>>(tasks, nt, acc, bins, splits, wide);
    if ((rc = fk_after_launch(ctx, "sah split")) != FK_OK) return fail(rc);
    sah_count_kernel<<<nc, kThreads, 0, st>>>(chunks, tasks, perm[src], lo, hi, splits, chunk_left);
    if ((rc = fk_after_launch(ctx, "sah count")) != FK_OK) return fail(rc);
    hsplits.resize(nt);
    hleft.resize(nc);
    FK_SAH_TRY(cudaMemcpyAsync(hsplits.data(), splits, sizeof(Split) * nt, cudaMemcpyDeviceToHost, st));
    FK_SAH_TRY(cudaMemcpyAsync(hleft.data(), chunk_left, 4 * (size_t)nc, cudaMemcpyDeviceToHost, st));
    FK_SAH_TRY(cudaStreamSynchronize(st));
    hoffs.resize(2 * (size_t)nc);
    {
      uint32_t t = 0xffffffffu, l = 0, r = 0, total_left = 0;
      for (uint32_t c = 0; c < nc; ++c) {
        if (hchunks[c].task != t) {
          if (t != 0xffffffffu && l != hsplits[t].nleft) total_left = 1;  // mismatch marker
          t = hchunks[c].task;
          l = r = 0;
        }
        hoffs[2 * c] = l;
        hoffs[2 * c + 1] = r;
        l += hleft[c];
        r += (hchunks[c].e - hchunks[c].b) - hleft[c];
      }
      if (t != 0xffffffffu && l != hsplits[t].nleft) total_left = 1;
      if (total_left) return fail(fk_fail(ctx, FK_ERR_DEVICE, "surface-area build: partition disagrees with bins"));
    }
    FK_SAH_TRY(cudaMemcpyAsync(offs, hoffs.data(), 8 * (size_t)nc, cudaMemcpyHostToDevice, st));
    sah_scatter_kernel<<<nc, kThreads, 0, st>>>(chunks, tasks, perm[src], perm[src ^ 1], lo, hi, splits, offs);
    if ((rc = fk_after_launch(ctx, "sah scatter")) != FK_OK) return fail(rc);
    std::vector<Task> next;
    for (uint32_t t = 0; t < nt; ++t) {
      const Task& k = cur[t];
      const uint32_t nl = hsplits[t].nleft, m = k.b + nl;
      if (nl == 0 || m >= k.e) return fail(fk_fail(ctx, FK_ERR_DEVICE, "surface-area build: empty side"));
      const Task kids[2] = {{k.b, m, k.rec + 1, k.level + 1, 2 * k.rec, (uint32_t)(src ^ 1)},
                            {m, k.e, k.rec + nl, k.level + 1, 2 * k.rec + 1, (uint32_t)(src ^ 1)}};
      for (const Task& c : kids) (c.e - c.b > kSmall ? next : small).push_back(c);
    }
    // the next level's uploads are stream-ordered after this scatter
    cur.swap(next);
    src ^= 1;
  }
  Task* dsmall = nullptr;
  rc = fk_dev_alloc(ctx, (void**)&dsmall, sizeof(Task) * small.size());
  if (rc != FK_OK) return fail(rc);
  cudaError_t e = cudaMemcpyAsync(dsmall, small.data(), sizeof(Task) * small.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sah_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem);
  if (e != cudaSuccess) {
    fk_dev_free(ctx, dsmall);
    return fail(fk_cuda_fail(ctx, e, "surface-area build: small subtrees"));
  }
  const uint32_t ns = (uint32_t)small.size();
  const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((ns + kSmallWarps - 1) / kSmallWarps,
                                                                    (uint32_t)ctx->sm_count * 16));
  sah_small_kernel<<<blocks, kSmallWarps * 32, kSmallSmem, st>>>(dsmall, ns, perm[0], perm[1], lo, hi, wide, words,
                                                              words + 1);
  rc = fk_after_launch(ctx, "sah small subtrees");
  uint32_t hw[2] = {0, 0};
  if (rc == FK_OK) {
    e = cudaMemcpyAsync(hw, words, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fk_cuda_fail(ctx, e, "surface-area build");
  }
  fk_dev_free(ctx, dsmall);
  if (rc != FK_OK) return fail(rc);
  if (hw[1]) return fail(fk_fail(ctx, FK_ERR_DEVICE, "surface-area build: subtree check failed"));
#undef FK_SAH_TRY
  *out_depth = hw[0];
  if (hw[0] > kMaxOrderedDepth) return fail(FK_OK);  // deeper than the ordered traversals accept
  fk_dev_free(ctx, base);
  *out_wide = wide;
  return FK_OK;
}

}  // namespace fk
