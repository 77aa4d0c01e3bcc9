// UV-space rasterisation of the low-poly mesh and compaction of the covered
// texels, on the device: MapUV::fromMesh / fromMeshes / fromMeshes_Hybrid
// (Src/compute.cpp:75-370) and CompressedMapUV (Src/compute.cpp:372-416).
//
// The reference loops over triangles in order and lets later triangles
// overwrite earlier ones.  Here pass 1 (one CTA per triangle, threads over its
// texel box) records, per texel, the largest key (triangle + 1, loop position)
// whose barycentric test passed: that is exactly the last write of the
// reference's loop nest.  Pass 2 recomputes the winning write's attributes
// with the same float operations, flags texels with dot(dir, dir) > 0.5,
// scans the flags in row-major order and writes the compressed rows.
#include <cmath>
#include <cstring>
#include <vector>

#include "fk_device.cuh"
#include "fk_internal.h"

namespace fk {

struct RasterTri {
  float p[3][3], n[3][3], d[3][3], t[3][3], b[3][3];
  float u[3][2];
  uint32_t x0, y0, x1, y1;
};

struct RasterArgs {
  const RasterTri* tris;
  uint32_t ntri, w, h;
  int hybrid;
  float edge;
  float pixx, pixy, halfx, halfy;
  uint32_t key_stride;  // > every texel x a triangle box reaches
  unsigned long long* owner;
};

__device__ __forceinline__ f3 ld(const float* v) { return mk3(v[0], v[1], v[2]); }

// Barycentric of Src/math.h:250-259 (reciprocal form).
__device__ __forceinline__ f3 bary2(float px, float py, const float u[3][2]) {
  float v0x = __fsub_rn(u[1][0], u[0][0]), v0y = __fsub_rn(u[1][1], u[0][1]);
  float v1x = __fsub_rn(u[2][0], u[0][0]), v1y = __fsub_rn(u[2][1], u[0][1]);
  float v2x = __fsub_rn(px, u[0][0]), v2y = __fsub_rn(py, u[0][1]);
  float s = __fdiv_rn(1.0f, __fsub_rn(__fmul_rn(v0x, v1y), __fmul_rn(v1x, v0y)));
  float i = __fmul_rn(__fsub_rn(__fmul_rn(v2x, v1y), __fmul_rn(v1x, v2y)), s);
  float j = __fmul_rn(__fsub_rn(__fmul_rn(v0x, v2y), __fmul_rn(v2x, v0y)), s);
  return mk3(__fsub_rn(__fsub_rn(1.0f, i), j), i, j);
}

__device__ __forceinline__ bool inside(f3 w) {
  return w.x >= -0.001f && w.x <= 1.0f && w.y >= -0.001f && w.y <= 1.0f && w.z >= -0.001f && w.z <= 1.0f;
}

__device__ __forceinline__ f3 texel_bary(const RasterArgs& a, const RasterTri& T, uint32_t x, uint32_t y) {
  float px = __fadd_rn(__fmul_rn((float)x, a.pixx), a.halfx);
  float py = __fadd_rn(__fmul_rn((float)y, a.pixy), a.halfy);
  return bary2(px, py, T.u);
}

__global__ void raster_owner_kernel(RasterArgs a) {
  const RasterTri& T = a.tris[blockIdx.x];
  uint32_t bw = T.x1 - T.x0 + 1;
  uint64_t area = (uint64_t)bw * (uint64_t)(T.y1 - T.y0 + 1);
  uint64_t total = (uint64_t)a.w * a.h;
  unsigned long long tri_key = (unsigned long long)(blockIdx.x + 1) << 32;
  for (uint64_t q = threadIdx.x; q < area; q += blockDim.x) {
    uint32_t x = T.x0 + (uint32_t)(q % bw), y = T.y0 + (uint32_t)(q / bw);
    if (!inside(texel_bary(a, T, x, y))) continue;
    uint32_t i = y * a.w + x;  // 32-bit index arithmetic of Src/compute.cpp:147
    if ((uint64_t)i >= total) continue;
    unsigned long long key = tri_key | (unsigned long long)(y * a.key_stride + x);
    atomicMax(a.owner + i, key);
  }
}

struct Attr {
  f3 p, d, n, t, b;
};

__device__ __forceinline__ float edge_dist(f3 e0, f3 e1, f3 p) {
  f3 v = sub(p, e0), e = sub(e1, e0);
  float t = __fdiv_rn(dot(v, e), dot(e, e));
  f3 q = add(e0, scale(e, t));
  f3 r = sub(q, p);
  return __fsqrt_rn(dot(r, r));
}

// Attributes written for texel (x, y) by triangle T (Src/compute.cpp:146-154
// and, for the hybrid mapping, :286-306).
__device__ __forceinline__ Attr texel_attr(const RasterArgs& a, const RasterTri& T, uint32_t x, uint32_t y) {
  f3 w = texel_bary(a, T, x, y);
  Attr r;
  r.p = blend3(ld(T.p[0]), ld(T.p[1]), ld(T.p[2]), w.x, w.y, w.z);
  r.n = normalize(blend3(ld(T.n[0]), ld(T.n[1]), ld(T.n[2]), w.x, w.y, w.z));
  f3 ds = normalize(blend3(ld(T.d[0]), ld(T.d[1]), ld(T.d[2]), w.x, w.y, w.z));
  if (a.hybrid) {
    f3 p0 = ld(T.p[0]), p1 = ld(T.p[1]), p2 = ld(T.p[2]);
    float e = fminf(edge_dist(p0, p1, r.p), fminf(edge_dist(p0, p2, r.p), edge_dist(p1, p2, r.p)));
    float k = fminf(__fdiv_rn(e, a.edge), 1.0f);
    r.d = normalize(add(scale(ds, __fsub_rn(1.0f, k)), scale(r.n, k)));
  } else {
    r.d = ds;
  }
  r.t = normalize(blend3(ld(T.t[0]), ld(T.t[1]), ld(T.t[2]), w.x, w.y, w.z));
  r.b = normalize(blend3(ld(T.b[0]), ld(T.b[1]), ld(T.b[2]), w.x, w.y, w.z));
  return r;
}

__device__ __forceinline__ bool texel_attr_of(const RasterArgs& a, uint32_t i, Attr& r) {
  unsigned long long k = a.owner[i];
  if (k == 0ull) return false;
  uint32_t tri = (uint32_t)(k >> 32) - 1u;
  uint32_t pos = (uint32_t)(k & 0xFFFFFFFFull);
  uint32_t y = pos / a.key_stride, x = pos % a.key_stride;
  r = texel_attr(a, a.tris[tri], x, y);
  return dot(r.d, r.d) > 0.5f;  // Src/compute.cpp:380
}

static constexpr int kScanBlock = 256;
static constexpr int kScanItems = 4;  // texels per thread
static constexpr int kScanTile = kScanBlock * kScanItems;

__global__ void __launch_bounds__(kScanBlock) raster_count_kernel(RasterArgs a, uint32_t* __restrict__ counts) {
  __shared__ uint32_t warp_sum[kScanBlock / 32];
  uint64_t total = (uint64_t)a.w * a.h;
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  uint32_t c = 0;
  for (int k = 0; k < kScanItems; ++k) {
    uint64_t i = base + (uint64_t)k * kScanBlock + threadIdx.x;
    Attr r;
    if (i < total && texel_attr_of(a, (uint32_t)i, r)) ++c;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int w = 0; w < kScanBlock / 32; ++w) s += warp_sum[w];
    counts[blockIdx.x] = s;
  }
}

// Exclusive scan of the per-tile counts (one CTA; tiles processed in chunks).
__global__ void __launch_bounds__(1024) scan_counts_kernel(uint32_t* counts, uint32_t n, uint32_t* total) {
  __shared__ uint32_t buf[1024];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < n; base += 1024) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < n ? counts[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
      uint32_t add_v = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
      __syncthreads();
      buf[threadIdx.x] += add_v;
      __syncthreads();
    }
    if (i < n) counts[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += buf[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanBlock) raster_write_kernel(RasterArgs a, const uint32_t* __restrict__ offsets,
                                                                   float4* __restrict__ pix, float4* __restrict__ pixt,
                                                                   uint32_t* __restrict__ idx) {
  __shared__ uint32_t warp_sum[kScanBlock / 32];
  __shared__ uint32_t round_base;
  uint64_t total = (uint64_t)a.w * a.h;
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  if (threadIdx.x == 0) round_base = offsets[blockIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < kScanItems; ++k) {
    uint64_t i = base + (uint64_t)k * kScanBlock + threadIdx.x;
    Attr r;
    bool f = i < total && texel_attr_of(a, (uint32_t)i, r);
    unsigned m = __ballot_sync(0xFFFFFFFFu, f);
    if (lane == 0) warp_sum[warp] = __popc(m);
    __syncthreads();
    uint32_t before = round_base;
    for (int w = 0; w < warp; ++w) before += warp_sum[w];
    before += __popc(m & ((1u << lane) - 1u));
    if (f) {
      pix[2 * (size_t)before] = make_float4(r.p.x, r.p.y, r.p.z, 0.0f);
      pix[2 * (size_t)before + 1] = make_float4(r.d.x, r.d.y, r.d.z, 0.0f);
      pixt[3 * (size_t)before] = make_float4(r.n.x, r.n.y, r.n.z, 0.0f);
      pixt[3 * (size_t)before + 1] = make_float4(r.t.x, r.t.y, r.t.z, 0.0f);
      pixt[3 * (size_t)before + 2] = make_float4(r.b.x, r.b.y, r.b.z, 0.0f);
      idx[before] = (uint32_t)i;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t s = 0;
      for (int w = 0; w < kScanBlock / 32; ++w) s += warp_sum[w];
      round_base += s;
    }
    __syncthreads();
  }
}

}  // namespace fk

namespace {

// (uint32_t)roundf(x) as the reference's x86-64 build performs it: through a
// signed 64-bit truncation, so negative values wrap (Src/compute.cpp:136-139).
inline uint32_t to_u32(float f) {
  if (!(f > -9.2e18f && f < 9.2e18f)) return 0u;
  return (uint32_t)(uint64_t)(int64_t)f;
}

}  // namespace

extern "C" int fk_raster_uv(fk_ctx* ctx, const fk_mesh* m, const fk_mesh* dirs, uint32_t W, uint32_t H, int mode,
                            float edge, fk_texel_map** out) {
  using fk::RasterTri;
  if (!ctx || !m || !out || W == 0 || H == 0 || (uint64_t)W * H > 0xFFFFFFFFull || mode < 0 || mode > 2)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: bad arguments");
  if (mode != FK_MAP_LOWPOLY_NORMALS && (!dirs || dirs->vertex_count() != m->vertex_count()))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: this mapping mode needs a direction mesh with the same vertices");
  const uint32_t nf = m->triangle_count();
  const uint32_t np = m->position_count(), nt = (uint32_t)(m->texcoords.size() / 2);
  const uint32_t nn = (uint32_t)(m->normals.size() / 3), nv = m->vertex_count();
  const bool has_tan = !m->tangents.empty();
  std::vector<RasterTri> tris(nf);
  const float scale_x = (float)W, scale_y = (float)H;
  const float pixx = 1.0f / scale_x, pixy = 1.0f / scale_y;
  const float halfx = pixx * 0.5f, halfy = pixy * 0.5f;
  uint64_t work = 0;
  uint64_t stride = (uint64_t)W + 1, max_y = H;
  for (uint32_t f = 0; f < nf; ++f) {
    RasterTri& T = tris[f];
    float sx[3], sy[3];
    for (int k = 0; k < 3; ++k) {
      uint32_t vi = m->triangles[3 * (size_t)f + k];
      const uint32_t* v = &m->vertices[3 * (size_t)vi];
      if (v[1] == 0xFFFFFFFFu || v[2] == 0xFFFFFFFFu)
        return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: low-poly mesh lacks texture coordinates or normals");
      if (v[0] >= np || v[1] >= nt || v[2] >= nn) return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: index out of range");
      for (int a = 0; a < 3; ++a) {
        T.p[k][a] = m->positions[3 * (size_t)v[0] + a];
        T.n[k][a] = m->normals[3 * (size_t)v[2] + a];
      }
      T.u[k][0] = m->texcoords[2 * (size_t)v[1]];
      T.u[k][1] = m->texcoords[2 * (size_t)v[1] + 1];
      if (mode == FK_MAP_LOWPOLY_NORMALS) {
        for (int a = 0; a < 3; ++a) T.d[k][a] = T.n[k][a];
      } else {
        uint32_t dn = dirs->vertices[3 * (size_t)vi + 2];
        if (dn >= dirs->normals.size() / 3) return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: direction index out of range");
        for (int a = 0; a < 3; ++a) T.d[k][a] = dirs->normals[3 * (size_t)dn + a];
      }
      // Tangent frames are read per vertex (Src/compute.cpp:109-114), by
      // normal index in the hybrid raster (Src/compute.cpp:248-253).
      uint32_t ti = mode == FK_MAP_HYBRID ? v[2] : vi;
      for (int a = 0; a < 3; ++a) {
        bool ok = has_tan && ti < nv;
        T.t[k][a] = ok ? m->tangents[3 * (size_t)ti + a] : 0.0f;
        T.b[k][a] = ok ? m->bitangents[3 * (size_t)ti + a] : 0.0f;
      }
      sx[k] = (T.u[k][0] - halfx) * scale_x;
      sy[k] = (T.u[k][1] - halfy) * scale_y;
    }
    float fx0 = std::roundf(std::fmin(sx[0], std::fmin(sx[1], sx[2])));
    float fy0 = std::roundf(std::fmin(sy[0], std::fmin(sy[1], sy[2])));
    float fx1 = std::roundf(std::fmax(sx[0], std::fmax(sx[1], sx[2])));
    float fy1 = std::roundf(std::fmax(sy[0], std::fmax(sy[1], sy[2])));
    if (mode == FK_MAP_HYBRID) {
      T.x0 = to_u32(std::fmax(fx0, 0.0f)); T.y0 = to_u32(std::fmax(fy0, 0.0f));
      T.x1 = to_u32(std::fmax(fx1, 0.0f)); T.y1 = to_u32(std::fmax(fy1, 0.0f));
    } else {
      T.x0 = std::min(to_u32(fx0), W); T.y0 = std::min(to_u32(fy0), H);
      T.x1 = std::min(to_u32(fx1), W); T.y1 = std::min(to_u32(fy1), H);
    }
    if (T.x0 > T.x1 || T.y0 > T.y1) {  // the reference's loops run zero times
      T.x0 = 1; T.x1 = 0; T.y0 = 1; T.y1 = 0;
      continue;
    }
    uint64_t area = (uint64_t)(T.x1 - T.x0 + 1) * (uint64_t)(T.y1 - T.y0 + 1);
    if (T.x1 >= 0xFFFFFFFEu || T.y1 >= 0xFFFFFFFEu || area > 4ull * W * H + 4096)
      return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: triangle " + std::to_string(f) + " spans too many texels");
    work += area;
    stride = std::max<uint64_t>(stride, (uint64_t)T.x1 + 1);
    max_y = std::max<uint64_t>(max_y, T.y1);
  }
  (void)work;
  if ((max_y + 1) * stride > 0xFFFFFFFFull)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_raster_uv: texel boxes exceed the 32-bit key range");
  const uint64_t total = (uint64_t)W * H;
  const uint32_t tiles = (uint32_t)((total + fk::kScanTile - 1) / fk::kScanTile);
  fk::RasterTri* dtris = nullptr;
  unsigned long long* owner = nullptr;
  uint32_t* counts = nullptr;
  uint32_t* dcount = nullptr;
  int rc = fk_dev_alloc(ctx, (void**)&dtris, sizeof(RasterTri) * (size_t)(nf ? nf : 1));
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&owner, 8 * total);
  if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&counts, 4 * (size_t)(tiles + 1));
  fk_texel_map* map = nullptr;
  uint32_t count = 0;
  auto cleanup = [&]() {
    cudaStreamSynchronize(ctx->stream);
    fk_dev_free(ctx, dtris);
    fk_dev_free(ctx, owner);
    fk_dev_free(ctx, counts);
  };
  auto cuda_ok = [&](cudaError_t e, const char* what) {
    if (rc == FK_OK && e != cudaSuccess) rc = fk_cuda_fail(ctx, e, what);
  };
  if (rc == FK_OK) {
    dcount = counts + tiles;
    if (nf) cuda_ok(cudaMemcpyAsync(dtris, tris.data(), sizeof(RasterTri) * nf, cudaMemcpyHostToDevice, ctx->stream), "raster upload");
    cuda_ok(cudaMemsetAsync(owner, 0, 8 * total, ctx->stream), "raster clear");
  }
  fk::RasterArgs a;
  a.tris = dtris;
  a.ntri = nf;
  a.w = W;
  a.h = H;
  a.hybrid = mode == FK_MAP_HYBRID;
  a.edge = edge;
  a.pixx = pixx;
  a.pixy = pixy;
  a.halfx = halfx;
  a.halfy = halfy;
  a.key_stride = (uint32_t)stride;
  a.owner = owner;
  if (rc == FK_OK && nf) {
    fk::raster_owner_kernel<<<nf, 256, 0, ctx->stream>>>(a);
    rc = fk_after_launch(ctx, "raster_owner_kernel");
  }
  if (rc == FK_OK) {
    fk::raster_count_kernel<<<tiles, fk::kScanBlock, 0, ctx->stream>>>(a, counts);
    rc = fk_after_launch(ctx, "raster_count_kernel");
  }
  if (rc == FK_OK) {
    fk::scan_counts_kernel<<<1, 1024, 0, ctx->stream>>>(counts, tiles, dcount);
    rc = fk_after_launch(ctx, "scan_counts_kernel");
  }
  if (rc == FK_OK) {
    cuda_ok(cudaMemcpyAsync(&count, dcount, 4, cudaMemcpyDeviceToHost, ctx->stream), "raster count");
    cuda_ok(cudaStreamSynchronize(ctx->stream), "raster sync");
  }
  if (rc == FK_OK) {
    map = new (std::nothrow) fk_texel_map();
    if (!map) rc = FK_ERR_NOMEM;
  }
  if (rc == FK_OK) {
    map->ctx = ctx;
    map->width = W;
    map->height = H;
    map->count = count;
    ctx->maps.insert(map);
    rc = fk_dev_alloc(ctx, (void**)&map->pix, 32 * (size_t)count);
    if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&map->pixt, 48 * (size_t)count);
    if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&map->indices, 4 * (size_t)count);
  }
  if (rc == FK_OK && count) {
    fk::raster_write_kernel<<<tiles, fk::kScanBlock, 0, ctx->stream>>>(a, counts, map->pix, map->pixt, map->indices);
    rc = fk_after_launch(ctx, "raster_write_kernel");
  }
  cleanup();
  if (rc != FK_OK) {
    if (map) fk_texel_map_free(ctx, map);
    return rc;
  }
  *out = map;
  return FK_OK;
}
