// Mesh preprocessing on the device: the face, vertex and welded normal
// generators and the tangent-space generator of Src/mesh.cpp:627-768 (host
// restatement: fk_mesh.cpp) as sort-and-reduce kernels.  Results are the host
// generators' bit for bit: every sum of the reference is a sequential loop
// over the triangles in index order, so the corners are stably sorted by the
// group they add into (position, weld class or vertex) and one thread per
// group adds its corners' terms in corner order -- the same binary32
// additions in the same order (the library is built with --fmad=false and
// IEEE division and square root).
//
// Pieces:
//   * a stable LSD radix sort of (key, value) u32 pairs, 8-bit digits: per
//     tile histograms, one device-wide exclusive scan of the digit-major
//     count table, and a scatter that ranks equal digits within a tile in
//     element order (__match_any_sync per warp, warp counts in shared memory);
//   * a device-wide exclusive scan (tile sums, one-CTA scan of the sums,
//     tile scans with their offsets);
//   * the weld: positions sorted by their 96-bit key, equal neighbours form a
//     class, each class's first corner by atomicMin, classes numbered in the
//     order of their first corners by a scan of first-corner flags -- the
//     order in which the reference's std::map meets new positions.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "fk_internal.h"

namespace fk {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr uint32_t kTile = kThreads * kItems;  // elements per CTA of the sort and scan passes
constexpr int kRadix = 256;

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 mul(V3 a, float k) { return v3(a.x * k, a.y * k, a.z * k); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 normalize(V3 v) { return mul(v, 1.0f / sqrtf(dot(v, v))); }
__device__ __forceinline__ V3 load3(const float* a, size_t i) { return v3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
__device__ __forceinline__ void store3(float* a, size_t i, V3 v) {
  a[3 * i] = v.x;
  a[3 * i + 1] = v.y;
  a[3 * i + 2] = v.z;
}

// Position of corner c (triangle c / 3, slot c % 3).
__device__ __forceinline__ uint32_t corner_position(const uint32_t* verts, const uint32_t* tris, uint32_t c) {
  return verts[3 * (size_t)tris[c]];
}

// Key bits of one weld coordinate.  The reference's std::map compares
// coordinates as floats (Src/mesh.cpp:38-41), so +0 and -0 are one key; the
// host generator keys on the bits of x + 0.0f, which turns -0 into +0 and
// keeps a NaN's payload with its quiet bit set.  The same bits, by integer
// operations (the device's float add would replace the payload).
__device__ __forceinline__ uint32_t weld_bits(float x) {
  const uint32_t b = __float_as_uint(x);
  if (b == 0x80000000u) return 0u;
  if ((b & 0x7FFFFFFFu) > 0x7F800000u) return b | 0x00400000u;
  return b;
}

__device__ __forceinline__ uint32_t grid_stride() { return gridDim.x * blockDim.x; }

// ------------------------------------------------------------ scan pieces
// Exclusive scan of one value per thread over the CTA; *total gets the sum.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t before = 0, sum = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const uint32_t s = s_warp[w];
    if (w < warp) before += s;
    sum += s;
  }
  __syncthreads();  // s_warp is free again
  *total = sum;
  return before + x - v;
}

// Sum of each tile of kTile elements.
__global__ void __launch_bounds__(kThreads) scan_tiles_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                              uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_warp[kWarps];
  const size_t base = (size_t)blockIdx.x * kTile;
  uint32_t acc = 0;
  for (int k = 0; k < kItems; ++k) {
    const size_t i = base + (size_t)k * kThreads + threadIdx.x;
    if (i < n) acc += in[i];
  }
  uint32_t total;
  block_exclusive(acc, s_warp, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Exclusive scan of the m tile sums in place (one CTA); *total gets the sum.
__global__ void __launch_bounds__(1024) scan_sums_kernel(uint32_t* sums, uint32_t m, uint32_t* total) {
  __shared__ uint32_t buf[1024];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < m; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < m ? sums[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
      const uint32_t a = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
      __syncthreads();
      buf[threadIdx.x] += a;
      __syncthreads();
    }
    if (i < m) sums[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += buf[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// Exclusive scan of each tile, offset by its tile's scanned sum.  out may be
// in: every element is read and written by the same thread.
__global__ void __launch_bounds__(kThreads) scan_apply_kernel(const uint32_t* in, uint32_t n,
                                                              const uint32_t* __restrict__ sums, uint32_t* out) {
  __shared__ uint32_t s_warp[kWarps];
  const size_t base = (size_t)blockIdx.x * kTile;
  uint32_t carry = sums[blockIdx.x];
  for (int k = 0; k < kItems; ++k) {
    const size_t i = base + (size_t)k * kThreads + threadIdx.x;
    const uint32_t v = i < n ? in[i] : 0;
    uint32_t total;
    const uint32_t ex = block_exclusive(v, s_warp, &total);
    if (i < n) out[i] = carry + ex;
    carry += total;
  }
}

// ------------------------------------------------------------ radix sort pieces
// counts[d * tiles + t] = elements of tile t whose digit at `shift` is d.
__global__ void __launch_bounds__(kThreads) radix_count_kernel(const uint32_t* __restrict__ keys, uint32_t n, int shift,
                                                               uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[kRadix];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kTile;
  for (int k = 0; k < kItems; ++k) {
    const size_t i = base + (size_t)k * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  counts[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// Moves each pair to its place: offsets holds the exclusive scan of the
// count table, so offsets[d * tiles + t] is where tile t's first element of
// digit d goes; within a tile, equal digits keep their element order.
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(const uint32_t* __restrict__ keys_in,
                                                                 const uint32_t* __restrict__ vals_in, uint32_t n,
                                                                 int shift, const uint32_t* __restrict__ offsets,
                                                                 uint32_t* __restrict__ keys_out,
                                                                 uint32_t* __restrict__ vals_out) {
  __shared__ uint32_t s_next[kRadix];          // next free place per digit for this tile
  __shared__ uint32_t s_warp[kWarps][kRadix];  // per-warp digit counts, then per-warp first places
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  s_next[threadIdx.x] = offsets[(size_t)threadIdx.x * gridDim.x + blockIdx.x];
  const size_t base = (size_t)blockIdx.x * kTile;
  for (int k = 0; k < kItems; ++k) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s_warp[w][threadIdx.x] = 0;
    __syncthreads();
    const size_t i = base + (size_t)k * kThreads + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys_in[i] : 0u;
    const uint32_t val = valid ? vals_in[i] : 0u;
    const uint32_t d = valid ? (key >> shift) & (kRadix - 1) : (uint32_t)kRadix;  // kRadix: no element
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) s_warp[warp][d] = __popc(peers);
    __syncthreads();
    {
      uint32_t run = s_next[threadIdx.x];
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = s_warp[w][threadIdx.x];
        s_warp[w][threadIdx.x] = run;
        run += c;
      }
      s_next[threadIdx.x] = run;
    }
    __syncthreads();
    if (valid) {
      const uint32_t at = s_warp[warp][d] + rank;
      keys_out[at] = key;
      vals_out[at] = val;
    }
    __syncthreads();
  }
}

__global__ void iota_kernel(uint32_t* __restrict__ a, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += grid_stride()) a[i] = i;
}

__global__ void gather_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, uint32_t n,
                              uint32_t* __restrict__ dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += grid_stride()) dst[i] = src[idx[i]];
}

// Group bounds of a sorted key array: [start[g], end[g]) for each key g
// present (both arrays zeroed first, so absent groups are empty).
__global__ void bounds_kernel(const uint32_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ start,
                              uint32_t* __restrict__ end) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += grid_stride()) {
    const uint32_t g = keys[i];
    if (i == 0 || keys[i - 1] != g) start[g] = i;
    if (i + 1 == n || keys[i + 1] != g) end[g] = i + 1;
  }
}

// ------------------------------------------------------------ index checks
// bad[0] |= 1: a triangle's vertex index >= nv; 2: a vertex's position index
// >= np; 4: (tangent space only) a texcoord index >= nt or normal index >= nn.
__global__ void check_kernel(const uint32_t* __restrict__ verts, uint32_t nv, const uint32_t* __restrict__ tris,
                             uint32_t n3, uint32_t np, uint32_t nt, uint32_t nn, int tangents, uint32_t* bad) {
  uint32_t flags = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += grid_stride())
    if (tris[i] >= nv) flags |= 1u;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += grid_stride()) {
    if (verts[3 * (size_t)v] >= np) flags |= 2u;
    if (tangents && (verts[3 * (size_t)v + 1] >= nt || verts[3 * (size_t)v + 2] >= nn)) flags |= 4u;
  }
  if (flags) atomicOr(bad, flags);
}

// ------------------------------------------------------------ normals
// Src/mesh.cpp:627-648 per triangle: normalize(cross(p1 - p0, p2 - p0)).
__global__ void face_normal_kernel(const float* __restrict__ pos, const uint32_t* __restrict__ verts,
                                   const uint32_t* __restrict__ tris, uint32_t nf, float* __restrict__ fn) {
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += grid_stride()) {
    const V3 p0 = load3(pos, corner_position(verts, tris, 3 * f));
    const V3 p1 = load3(pos, corner_position(verts, tris, 3 * f + 1));
    const V3 p2 = load3(pos, corner_position(verts, tris, 3 * f + 2));
    store3(fn, f, normalize(cross(sub(p1, p0), sub(p2, p0))));
  }
}

// Face normals: a vertex keeps the last triangle that names it (the
// reference assigns in triangle order); last[v] = that triangle + 1.
__global__ void face_owner_kernel(const uint32_t* __restrict__ tris, uint32_t n3, uint32_t* __restrict__ last) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += grid_stride())
    atomicMax(&last[tris[c]], c / 3 + 1);
}
__global__ void face_assign_kernel(uint32_t* __restrict__ verts, uint32_t nv, const uint32_t* __restrict__ last) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += grid_stride())
    if (last[v]) verts[3 * (size_t)v + 2] = last[v] - 1;
}

// (group key, corner) pairs: the corner's position, or its vertex.
__global__ void corner_pairs_kernel(const uint32_t* __restrict__ verts, const uint32_t* __restrict__ tris, uint32_t n3,
                                    int by_vertex, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += grid_stride()) {
    keys[c] = by_vertex ? tris[c] : corner_position(verts, tris, c);
    vals[c] = c;
  }
}

// Src/mesh.cpp:650-678: per position, 0 + n(f) + n(f') + ... over its
// corners in corner order, then normalised (a position no triangle uses gets
// normalize(0), as in the reference).
__global__ void vertex_normal_kernel(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end,
                                     const uint32_t* __restrict__ corners, const float* __restrict__ fn, uint32_t np,
                                     float* __restrict__ out) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += grid_stride()) {
    V3 acc = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t i = start[p]; i < end[p]; ++i) acc = add(acc, load3(fn, corners[i] / 3));
    store3(out, p, normalize(acc));
  }
}
__global__ void vertex_assign_kernel(uint32_t* __restrict__ verts, uint32_t nv) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += grid_stride())
    verts[3 * (size_t)v + 2] = verts[3 * (size_t)v];
}

// Weld: the three key words of every position.
__global__ void weld_keys_kernel(const float* __restrict__ pos, uint32_t np, uint32_t* __restrict__ kx,
                                 uint32_t* __restrict__ ky, uint32_t* __restrict__ kz) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += grid_stride()) {
    kx[p] = weld_bits(pos[3 * (size_t)p]);
    ky[p] = weld_bits(pos[3 * (size_t)p + 1]);
    kz[p] = weld_bits(pos[3 * (size_t)p + 2]);
  }
}
// head[i] = 1 where sorted position i starts a new key.
__global__ void weld_heads_kernel(const uint32_t* __restrict__ order, uint32_t np, const uint32_t* __restrict__ kx,
                                  const uint32_t* __restrict__ ky, const uint32_t* __restrict__ kz,
                                  uint32_t* __restrict__ head) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += grid_stride()) {
    uint32_t h = 1;
    if (i > 0) {
      const uint32_t a = order[i], b = order[i - 1];
      h = (kx[a] != kx[b] || ky[a] != ky[b] || kz[a] != kz[b]) ? 1u : 0u;
    }
    head[i] = h;
  }
}
// cls[p] = class of position p (classes numbered in key order for now).
__global__ void weld_class_kernel(const uint32_t* __restrict__ order, uint32_t np, const uint32_t* __restrict__ head,
                                  const uint32_t* __restrict__ head_scan, uint32_t* __restrict__ cls) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += grid_stride())
    cls[order[i]] = head_scan[i] + head[i] - 1;
}
// first[class] = its first corner (first[] preset to all ones).
__global__ void weld_first_kernel(const uint32_t* __restrict__ verts, const uint32_t* __restrict__ tris, uint32_t n3,
                                  const uint32_t* __restrict__ cls, uint32_t* __restrict__ first) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += grid_stride())
    atomicMin(&first[cls[corner_position(verts, tris, c)]], c);
}
__global__ void weld_flag_kernel(const uint32_t* __restrict__ verts, const uint32_t* __restrict__ tris, uint32_t n3,
                                 const uint32_t* __restrict__ cls, const uint32_t* __restrict__ first,
                                 uint32_t* __restrict__ flag) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += grid_stride())
    flag[c] = first[cls[corner_position(verts, tris, c)]] == c ? 1u : 0u;
}
// The normal index of each corner (its class's rank among first corners),
// written to the corner's vertex (every corner of a vertex has the same
// position, so all writers agree), and the (index, corner) pairs to sort.
__global__ void weld_ids_kernel(uint32_t* __restrict__ verts, const uint32_t* __restrict__ tris, uint32_t n3,
                                const uint32_t* __restrict__ cls, const uint32_t* __restrict__ first,
                                const uint32_t* __restrict__ rank, uint32_t* __restrict__ keys,
                                uint32_t* __restrict__ vals) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += grid_stride()) {
    const uint32_t v = tris[c];
    const uint32_t id = rank[first[cls[verts[3 * (size_t)v]]]];
    keys[c] = id;
    vals[c] = c;
    verts[3 * (size_t)v + 2] = id;
  }
}
// Src/mesh.cpp:680-722: a class starts at its first corner's face normal
// and adds the others in corner order.
__global__ void weld_normal_kernel(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end,
                                   const uint32_t* __restrict__ corners, const float* __restrict__ fn, uint32_t count,
                                   float* __restrict__ out) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < count; g += grid_stride()) {
    const uint32_t s = start[g], e = end[g];
    V3 acc = load3(fn, corners[s] / 3);
    for (uint32_t i = s + 1; i < e; ++i) acc = add(acc, load3(fn, corners[i] / 3));
    store3(out, g, normalize(acc));
  }
}

// ------------------------------------------------------------ tangent space
// Src/mesh.cpp:724-768 per triangle: the texture-space s direction.
__global__ void tangent_dir_kernel(const float* __restrict__ pos, const float* __restrict__ uv,
                                   const uint32_t* __restrict__ verts, const uint32_t* __restrict__ tris, uint32_t nf,
                                   float* __restrict__ sdir) {
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += grid_stride()) {
    V3 p[3];
    float u[3][2];
    for (int k = 0; k < 3; ++k) {
      const uint32_t* v = verts + 3 * (size_t)tris[3 * (size_t)f + k];
      p[k] = load3(pos, v[0]);
      u[k][0] = uv[2 * (size_t)v[1]];
      u[k][1] = uv[2 * (size_t)v[1] + 1];
    }
    const V3 e0 = sub(p[1], p[0]), e1 = sub(p[2], p[0]);
    const float t0x = u[1][0] - u[0][0], t0y = u[1][1] - u[0][1];
    const float t1x = u[2][0] - u[0][0], t1y = u[2][1] - u[0][1];
    const float r = 1.0f / (t0x * t1y - t1x * t0y);
    store3(sdir, f, mul(sub(mul(e0, t1y), mul(e1, t0y)), r));
  }
}
// Per vertex: 0 + sdir(f) + ... in corner order, Gram-Schmidt against the
// vertex normal, bitangent = n x t.
__global__ void tangent_kernel(const uint32_t* __restrict__ start, const uint32_t* __restrict__ end,
                               const uint32_t* __restrict__ corners, const float* __restrict__ sdir,
                               const uint32_t* __restrict__ verts, const float* __restrict__ nrm, uint32_t nv,
                               float* __restrict__ tan, float* __restrict__ bit) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += grid_stride()) {
    V3 t = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t i = start[v]; i < end[v]; ++i) t = add(t, load3(sdir, corners[i] / 3));
    const V3 n = load3(nrm, verts[3 * (size_t)v + 2]);
    const V3 tt = normalize(sub(t, mul(n, dot(n, t))));
    store3(tan, v, tt);
    store3(bit, v, cross(n, tt));
  }
}

template <class T>
T* carve(char*& p, size_t count) {
  T* r = reinterpret_cast<T*>(p);
  p += (sizeof(T) * count + 255) & ~(size_t)255;
  return r;
}

uint32_t tiles_of(uint32_t n) { return (uint32_t)(((uint64_t)n + kTile - 1) / kTile); }
int bits_for(uint32_t max_key) { return max_key ? 32 - __builtin_clz(max_key) : 0; }

// One preprocessing call: device copies of the mesh, work arrays carved from
// one pool allocation, launch helpers.
struct Job {
  fk_ctx* ctx;
  cudaStream_t st;
  uint32_t grid_cap;
  char* base = nullptr;
  uint32_t* counts = nullptr;  // radix count table, kRadix x tiles
  uint32_t* sums = nullptr;    // scan tile sums (+1 word for the total)
  int rc = FK_OK;

  explicit Job(fk_ctx* c) : ctx(c), st(c->stream), grid_cap((uint32_t)std::max(c->sm_count, 1) * 16) {}
  ~Job() {
    if (base) {
      cudaStreamSynchronize(st);
      fk_dev_free(ctx, base);
    }
  }
  uint32_t grid(uint32_t n) const {
    return std::max<uint32_t>(1, std::min<uint32_t>((uint32_t)(((uint64_t)n + 255) / 256), grid_cap));
  }
  bool ok() const { return rc == FK_OK; }
  void cuda(cudaError_t e, const char* what) {
    if (rc == FK_OK && e != cudaSuccess) rc = fk_cuda_fail(ctx, e, what);
  }
  void launched(const char* what) {
    if (rc == FK_OK) rc = fk_after_launch(ctx, what);
  }
  void zero(void* p, size_t bytes, int value = 0) {
    if (ok() && bytes) cuda(cudaMemsetAsync(p, value, bytes, st), "preprocessing memset");
  }
  void up(void* dst, const void* src, size_t bytes) {
    if (ok() && bytes) cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "preprocessing upload");
  }
  void down(void* dst, const void* src, size_t bytes) {
    if (ok() && bytes) cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "preprocessing download");
  }
  void sync() {
    if (ok()) cuda(cudaStreamSynchronize(st), "preprocessing sync");
  }

  // out = exclusive scan of in (n elements; out may be in); *total (device
  // word) gets the sum when non-null.
  void scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total) {
    if (!ok()) return;
    if (n == 0) {
      zero(total, total ? 4 : 0);
      return;
    }
    const uint32_t t = tiles_of(n);
    scan_tiles_kernel<<<t, kThreads, 0, st>>>(in, n, sums);
    launched("scan_tiles_kernel");
    if (!ok()) return;
    scan_sums_kernel<<<1, 1024, 0, st>>>(sums, t, total);
    launched("scan_sums_kernel");
    if (!ok()) return;
    scan_apply_kernel<<<t, kThreads, 0, st>>>(in, n, sums, out);
    launched("scan_apply_kernel");
  }

  // Stable sort of n (key, value) pairs by the low `bits` bits of the keys;
  // the result ends in (*keys, *vals), the other pair of buffers is scratch.
  void sort(uint32_t** keys, uint32_t** vals, uint32_t** keys2, uint32_t** vals2, uint32_t n, int bits) {
    if (n <= 1) return;
    const uint32_t t = tiles_of(n);
    for (int shift = 0; shift < bits && ok(); shift += 8) {
      radix_count_kernel<<<t, kThreads, 0, st>>>(*keys, n, shift, counts);
      launched("radix_count_kernel");
      scan(counts, counts, kRadix * t, nullptr);
      if (!ok()) return;
      radix_scatter_kernel<<<t, kThreads, 0, st>>>(*keys, *vals, n, shift, counts, *keys2, *vals2);
      launched("radix_scatter_kernel");
      std::swap(*keys, *keys2);
      std::swap(*vals, *vals2);
    }
  }
};

}  // namespace
}  // namespace fk

using namespace fk;

extern "C" {

int fk_mesh_compute_normals_device(fk_ctx* ctx, fk_mesh* m, int method) {
  if (!ctx || !m || method < FK_NORMALS_FACE || method > FK_NORMALS_WELDED)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_mesh_compute_normals_device: bad arguments");
  const uint32_t np = m->position_count(), nv = m->vertex_count(), nf = m->triangle_count();
  if (3ull * nf >= 0xFFFFFFFFull || np >= 0xFFFFFFFFu)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_mesh_compute_normals_device: mesh too large for 32-bit corner indices");
  const uint32_t n3 = 3 * nf;
  const bool face = method == FK_NORMALS_FACE, vertex = method == FK_NORMALS_VERTEX, weld = method == FK_NORMALS_WELDED;
  const uint32_t N = std::max<uint32_t>(std::max(n3, np), 1);
  const uint32_t count_tiles = tiles_of(N);
  const size_t sum_words = std::max<size_t>(tiles_of(kRadix * count_tiles), tiles_of(N)) + 1;

  Job j(ctx);
  float *d_pos, *fn, *out;
  uint32_t *d_verts, *d_tris, *keys, *vals, *keys2, *vals2, *kx, *ky, *kz, *cls, *first, *flag, *scanned, *start, *end,
      *last, *words;
  auto layout = [&](char* p0) -> size_t {
    char* p = p0;
    d_pos = carve<float>(p, 3 * (size_t)np + 1);
    d_verts = carve<uint32_t>(p, 3 * (size_t)nv + 1);
    d_tris = carve<uint32_t>(p, (size_t)n3 + 1);
    fn = carve<float>(p, 3 * (size_t)nf + 1);
    out = carve<float>(p, 3 * (size_t)(face ? nf : np) + 1);
    const size_t sortn = face ? 1 : N;
    keys = carve<uint32_t>(p, sortn);
    vals = carve<uint32_t>(p, sortn);
    keys2 = carve<uint32_t>(p, sortn);
    vals2 = carve<uint32_t>(p, sortn);
    const size_t wn = weld ? N : 1;
    kx = carve<uint32_t>(p, weld ? np + 1 : 1);
    ky = carve<uint32_t>(p, weld ? np + 1 : 1);
    kz = carve<uint32_t>(p, weld ? np + 1 : 1);
    cls = carve<uint32_t>(p, weld ? np + 1 : 1);
    first = carve<uint32_t>(p, weld ? np + 1 : 1);
    flag = carve<uint32_t>(p, wn);
    scanned = carve<uint32_t>(p, wn);
    start = carve<uint32_t>(p, face ? 1 : (size_t)np + 1);
    end = carve<uint32_t>(p, face ? 1 : (size_t)np + 1);
    last = carve<uint32_t>(p, face ? (size_t)nv + 1 : 1);
    j.counts = carve<uint32_t>(p, face ? 1 : (size_t)kRadix * count_tiles);
    j.sums = carve<uint32_t>(p, sum_words);
    words = carve<uint32_t>(p, 2);  // [0] index-check flags, [1] scan total
    return (size_t)(p - p0);
  };
  {
    char probe[1];
    const size_t bytes = layout(probe);  // offsets only: nothing is written through these pointers
    int rc = fk_dev_alloc(ctx, (void**)&j.base, bytes);
    if (rc != FK_OK) return rc;
    layout(j.base);
  }
  j.up(d_pos, m->positions.data(), sizeof(float) * m->positions.size());
  j.up(d_verts, m->vertices.data(), sizeof(uint32_t) * m->vertices.size());
  j.up(d_tris, m->triangles.data(), sizeof(uint32_t) * m->triangles.size());
  j.zero(words, 8);
  if (j.ok()) {
    check_kernel<<<j.grid(std::max(n3, nv)), 256, 0, j.st>>>(d_verts, nv, d_tris, n3, np, 0, 0, 0, words);
    j.launched("check_kernel");
  }
  uint32_t bad = 0;
  j.down(&bad, words, 4);
  j.sync();
  if (!j.ok()) return j.rc;
  if (bad) return fk_fail(ctx, FK_ERR_INVALID, "fk_mesh_compute_normals_device: index out of range");

  if (nf) {
    face_normal_kernel<<<j.grid(nf), 256, 0, j.st>>>(d_pos, d_verts, d_tris, nf, fn);
    j.launched("face_normal_kernel");
  }
  uint32_t count = 0;  // normals produced
  if (face) {
    count = nf;
    j.zero(last, sizeof(uint32_t) * nv);
    if (j.ok() && n3) {
      face_owner_kernel<<<j.grid(n3), 256, 0, j.st>>>(d_tris, n3, last);
      j.launched("face_owner_kernel");
    }
    if (j.ok() && nv) {
      face_assign_kernel<<<j.grid(nv), 256, 0, j.st>>>(d_verts, nv, last);
      j.launched("face_assign_kernel");
    }
    if (j.ok() && nf) j.cuda(cudaMemcpyAsync(out, fn, sizeof(float) * 3 * nf, cudaMemcpyDeviceToDevice, j.st), "copy");
  } else if (vertex) {
    count = np;
    if (j.ok() && n3) {
      corner_pairs_kernel<<<j.grid(n3), 256, 0, j.st>>>(d_verts, d_tris, n3, 0, keys, vals);
      j.launched("corner_pairs_kernel");
    }
    j.sort(&keys, &vals, &keys2, &vals2, n3, bits_for(np ? np - 1 : 0));
    j.zero(start, sizeof(uint32_t) * np);
    j.zero(end, sizeof(uint32_t) * np);
    if (j.ok() && n3) {
      bounds_kernel<<<j.grid(n3), 256, 0, j.st>>>(keys, n3, start, end);
      j.launched("bounds_kernel");
    }
    if (j.ok() && np) {
      vertex_normal_kernel<<<j.grid(np), 256, 0, j.st>>>(start, end, vals, fn, np, out);
      j.launched("vertex_normal_kernel");
    }
    if (j.ok() && nv) {
      vertex_assign_kernel<<<j.grid(nv), 256, 0, j.st>>>(d_verts, nv);
      j.launched("vertex_assign_kernel");
    }
  } else if (n3) {  // welded; no triangles, no normals
    // positions sorted by (x, y, z) key words: three stable passes, z first
    weld_keys_kernel<<<j.grid(np), 256, 0, j.st>>>(d_pos, np, kx, ky, kz);
    j.launched("weld_keys_kernel");
    if (j.ok()) {
      iota_kernel<<<j.grid(np), 256, 0, j.st>>>(vals, np);
      j.launched("iota_kernel");
    }
    const uint32_t* word[3] = {kz, ky, kx};
    for (int w = 0; w < 3 && j.ok(); ++w) {
      gather_kernel<<<j.grid(np), 256, 0, j.st>>>(word[w], vals, np, keys);
      j.launched("gather_kernel");
      j.sort(&keys, &vals, &keys2, &vals2, np, 32);
    }
    if (j.ok()) {
      weld_heads_kernel<<<j.grid(np), 256, 0, j.st>>>(vals, np, kx, ky, kz, flag);
      j.launched("weld_heads_kernel");
    }
    j.scan(flag, scanned, np, nullptr);
    if (j.ok()) {
      weld_class_kernel<<<j.grid(np), 256, 0, j.st>>>(vals, np, flag, scanned, cls);
      j.launched("weld_class_kernel");
    }
    j.zero(first, sizeof(uint32_t) * np, 0xFF);
    if (j.ok()) {
      weld_first_kernel<<<j.grid(n3), 256, 0, j.st>>>(d_verts, d_tris, n3, cls, first);
      j.launched("weld_first_kernel");
    }
    if (j.ok()) {
      weld_flag_kernel<<<j.grid(n3), 256, 0, j.st>>>(d_verts, d_tris, n3, cls, first, flag);
      j.launched("weld_flag_kernel");
    }
    j.scan(flag, scanned, n3, words + 1);
    j.down(&count, words + 1, 4);
    j.sync();
    if (!j.ok()) return j.rc;
    if (count == 0 || count > np) return fk_fail(ctx, FK_ERR_DEVICE, "fk_mesh_compute_normals_device: weld count");
    weld_ids_kernel<<<j.grid(n3), 256, 0, j.st>>>(d_verts, d_tris, n3, cls, first, scanned, keys, vals);
    j.launched("weld_ids_kernel");
    j.sort(&keys, &vals, &keys2, &vals2, n3, bits_for(count - 1));
    j.zero(start, sizeof(uint32_t) * count);
    j.zero(end, sizeof(uint32_t) * count);
    if (j.ok()) {
      bounds_kernel<<<j.grid(n3), 256, 0, j.st>>>(keys, n3, start, end);
      j.launched("bounds_kernel");
    }
    if (j.ok()) {
      weld_normal_kernel<<<j.grid(count), 256, 0, j.st>>>(start, end, vals, fn, count, out);
      j.launched("weld_normal_kernel");
    }
  }
  std::vector<float> normals(3 * (size_t)count);
  std::vector<uint32_t> verts(m->vertices.size());
  j.down(normals.data(), out, sizeof(float) * normals.size());
  j.down(verts.data(), d_verts, sizeof(uint32_t) * verts.size());
  j.sync();
  if (!j.ok()) return j.rc;
  m->normals.swap(normals);
  m->vertices.swap(verts);
  return FK_OK;
}

int fk_mesh_compute_tangent_space_device(fk_ctx* ctx, fk_mesh* m) {
  if (!ctx || !m) return fk_fail(ctx, FK_ERR_INVALID, "fk_mesh_compute_tangent_space_device: bad arguments");
  const uint32_t np = m->position_count(), nv = m->vertex_count(), nf = m->triangle_count();
  const uint32_t nt = (uint32_t)(m->texcoords.size() / 2), nn = (uint32_t)(m->normals.size() / 3);
  if (3ull * nf >= 0xFFFFFFFFull)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_mesh_compute_tangent_space_device: mesh too large for 32-bit corner indices");
  const uint32_t n3 = 3 * nf;
  const uint32_t N = std::max<uint32_t>(n3, 1);
  const uint32_t count_tiles = tiles_of(N);
  const size_t sum_words = std::max<size_t>(tiles_of(kRadix * count_tiles), tiles_of(N)) + 1;

  Job j(ctx);
  float *d_pos, *d_uv, *d_nrm, *sdir, *tan, *bit;
  uint32_t *d_verts, *d_tris, *keys, *vals, *keys2, *vals2, *start, *end, *words;
  auto layout = [&](char* p0) -> size_t {
    char* p = p0;
    d_pos = carve<float>(p, 3 * (size_t)np + 1);
    d_uv = carve<float>(p, 2 * (size_t)nt + 1);
    d_nrm = carve<float>(p, 3 * (size_t)nn + 1);
    d_verts = carve<uint32_t>(p, 3 * (size_t)nv + 1);
    d_tris = carve<uint32_t>(p, (size_t)n3 + 1);
    sdir = carve<float>(p, 3 * (size_t)nf + 1);
    tan = carve<float>(p, 3 * (size_t)nv + 1);
    bit = carve<float>(p, 3 * (size_t)nv + 1);
    keys = carve<uint32_t>(p, N);
    vals = carve<uint32_t>(p, N);
    keys2 = carve<uint32_t>(p, N);
    vals2 = carve<uint32_t>(p, N);
    start = carve<uint32_t>(p, (size_t)nv + 1);
    end = carve<uint32_t>(p, (size_t)nv + 1);
    j.counts = carve<uint32_t>(p, (size_t)kRadix * count_tiles);
    j.sums = carve<uint32_t>(p, sum_words);
    words = carve<uint32_t>(p, 2);
    return (size_t)(p - p0);
  };
  {
    char probe[1];
    const size_t bytes = layout(probe);  // offsets only: nothing is written through these pointers
    int rc = fk_dev_alloc(ctx, (void**)&j.base, bytes);
    if (rc != FK_OK) return rc;
    layout(j.base);
  }
  j.up(d_pos, m->positions.data(), sizeof(float) * m->positions.size());
  j.up(d_uv, m->texcoords.data(), sizeof(float) * 2 * (size_t)nt);
  j.up(d_nrm, m->normals.data(), sizeof(float) * 3 * (size_t)nn);
  j.up(d_verts, m->vertices.data(), sizeof(uint32_t) * m->vertices.size());
  j.up(d_tris, m->triangles.data(), sizeof(uint32_t) * m->triangles.size());
  j.zero(words, 8);
  if (j.ok()) {
    check_kernel<<<j.grid(std::max(n3, nv)), 256, 0, j.st>>>(d_verts, nv, d_tris, n3, np, nt, nn, 1, words);
    j.launched("check_kernel");
  }
  uint32_t bad = 0;
  j.down(&bad, words, 4);
  j.sync();
  if (!j.ok()) return j.rc;
  if (bad) return fk_fail(ctx, FK_ERR_INVALID, "fk_mesh_compute_tangent_space_device: index out of range");

  if (nf) {
    tangent_dir_kernel<<<j.grid(nf), 256, 0, j.st>>>(d_pos, d_uv, d_verts, d_tris, nf, sdir);
    j.launched("tangent_dir_kernel");
    if (j.ok()) {
      corner_pairs_kernel<<<j.grid(n3), 256, 0, j.st>>>(d_verts, d_tris, n3, 1, keys, vals);
      j.launched("corner_pairs_kernel");
    }
    j.sort(&keys, &vals, &keys2, &vals2, n3, bits_for(nv ? nv - 1 : 0));
  }
  j.zero(start, sizeof(uint32_t) * nv);
  j.zero(end, sizeof(uint32_t) * nv);
  if (j.ok() && n3) {
    bounds_kernel<<<j.grid(n3), 256, 0, j.st>>>(keys, n3, start, end);
    j.launched("bounds_kernel");
  }
  if (j.ok() && nv) {
    tangent_kernel<<<j.grid(nv), 256, 0, j.st>>>(start, end, vals, sdir, d_verts, d_nrm, nv, tan, bit);
    j.launched("tangent_kernel");
  }
  std::vector<float> t(3 * (size_t)nv), b(3 * (size_t)nv);
  j.down(t.data(), tan, sizeof(float) * t.size());
  j.down(b.data(), bit, sizeof(float) * b.size());
  j.sync();
  if (!j.ok()) return j.rc;
  m->tangents.swap(t);
  m->bitangents.swap(b);
  return FK_OK;
}

}  // extern "C"
