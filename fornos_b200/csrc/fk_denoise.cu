// Learned per-texel denoiser (no counterpart in the reference): an MLP
// 250 -> 64 -> 64 -> 4 with tanh-form GELU, BF16 weights and activations on
// the tensor cores (mma.sync m16n8k16, FP32 accumulation), over a 5 x 5 texel
// neighbourhood of 10 features per texel:
//   AO (1), bent normal as 2-D octahedral (2), position relative to the centre
//   texel in units of the centre's texel spacing (3), interpolated normal as
//   octahedral (2), mapping hit distance / max distance (1), coverage (1).
// Neighbours outside the texture or without a mapping hit contribute zeros.
// The input width is padded from 250 to 256 with zero columns.
//
// Kernels: the dense feature image, input-row assembly, the fused training
// step (forward, MSE loss, backward, per-CTA weight-gradient partials), the
// deterministic gradient reduction + Adam update, and inference fused with
// the neighbourhood gather.  Per-tile verification helpers serve the
// denoised bake, which re-bakes a tile at full sample count when the network
// disagrees with a full-count subsample there.
#include <cuda_bf16.h>

#include "fk_device.cuh"
#include "fk_internal.h"

namespace fk {
namespace {

using dn::kHidden;
using dn::kK1;
using dn::kOut;
using dn::kRows;

constexpr int XS = kK1 + 8;     // bf16 row stride of an input tile in shared memory
constexpr int HS = kHidden + 8; // bf16 row stride of a hidden-width tile
constexpr int TS = kRows + 8;   // bf16 row stride of a transposed (unit x row) tile
constexpr uint32_t kNoTexel = 0xFFFFFFFFu;

__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Two floats rounded to bf16 (nearest even), the lower column in the low half.
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t pack_u16(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<uint16_t*>(&h);
}

// tanh-form GELU and its derivative.
__device__ __forceinline__ float gelu(float z, float& dz) {
  const float k0 = 0.7978845608028654f, k1 = 0.044715f;
  const float z2 = z * z;
  const float u = k0 * (z + k1 * (z2 * z));
  const float th = tanhf(u);
  dz = 0.5f * (1.0f + th) + (0.5f * z) * ((1.0f - th * th) * (k0 * (1.0f + (3.0f * k1) * z2)));
  return (0.5f * z) * (1.0f + th);
}

// Octahedral encoding of a direction (zero or non-finite vectors map to 0).
__device__ __forceinline__ float2 oct_encode(float x, float y, float z) {
  const float s = (fabsf(x) + fabsf(y)) + fabsf(z);
  if (!(s > 0.0f) || !isfinite(s)) return make_float2(0.0f, 0.0f);
  float px = x / s, py = y / s;
  if (z < 0.0f) {
    const float qx = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f);
    const float qy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
    px = qx;
    py = qy;
  }
  return make_float2(px, py);
}

__device__ __forceinline__ float clamp4(float v) { return fminf(fmaxf(v, -4.0f), 4.0f); }

// The 10 features of neighbour j (< 25, row-major over the 5 x 5 window) of
// the texel at pixel p; zeros outside the texture, without a mapping hit, or
// for p = kNoTexel.
__device__ __forceinline__ void neighbour_features(const float4* __restrict__ f0, const float4* __restrict__ f1,
                                                   const float4* __restrict__ f2, uint32_t w, uint32_t h, uint32_t p,
                                                   int j, float (&v)[10]) {
#pragma unroll
  for (int k = 0; k < 10; ++k) v[k] = 0.0f;
  if (p == kNoTexel) return;
  const int cx = (int)(p % w), cy = (int)(p / w);
  const int x = cx + j % 5 - 2, y = cy + j / 5 - 2;
  if (x < 0 || y < 0 || x >= (int)w || y >= (int)h) return;
  const uint32_t q = (uint32_t)y * w + (uint32_t)x;
  const float4 a = __ldg(f0 + q);
  if (!(a.w > 0.0f)) return;
  const float4 c = __ldg(f1 + p), b = __ldg(f1 + q), n = __ldg(f2 + q);
  const float sp = __ldg(f2 + p).z;  // centre texel spacing
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  if (sp > 0.0f) {
    v[3] = clamp4((b.x - c.x) / sp);
    v[4] = clamp4((b.y - c.y) / sp);
    v[5] = clamp4((b.z - c.z) / sp);
  }
  v[6] = n.x;
  v[7] = n.y;
  v[8] = b.w;
  v[9] = 1.0f;
}

// One input row (256 bf16 = 128 words) for the texel at pixel p, written by a
// whole warp: lane j < 25 writes neighbour j's 10 features, lane 25 the pad.
__device__ __forceinline__ void assemble_row(const float4* __restrict__ f0, const float4* __restrict__ f1,
                                             const float4* __restrict__ f2, uint32_t w, uint32_t h, uint32_t p,
                                             int lane, uint32_t* dst) {
  if (lane < 25) {
    float v[10];
    neighbour_features(f0, f1, f2, w, h, p, lane, v);
#pragma unroll
    for (int k = 0; k < 5; ++k) dst[5 * lane + k] = pack2(v[2 * k], v[2 * k + 1]);
  } else if (lane == 25) {
    dst[125] = 0u;
    dst[126] = 0u;
    dst[127] = 0u;
  }
}

struct Smem {
  __nv_bfloat16* x;    // [kRows][XS]
  __nv_bfloat16* w1;   // [64][XS]
  __nv_bfloat16* w2;   // [64][HS]  (out, in)
  __nv_bfloat16* w3;   // [8][HS]   rows 4..7 zero
};

__device__ __forceinline__ void copy_words(uint32_t* dst, int dst_stride_w, const uint32_t* src, int src_stride_w,
                                           int rows, int words) {
  for (int i = threadIdx.x; i < rows * words; i += blockDim.x) {
    const int r = i / words, c = i % words;
    dst[r * dst_stride_w + c] = __ldg(src + r * src_stride_w + c);
  }
}

__device__ __forceinline__ void load_forward_weights(const Smem& s, const DnWeights& wt) {
  copy_words((uint32_t*)s.w1, XS / 2, (const uint32_t*)wt.w1, kK1 / 2, kHidden, kK1 / 2);
  copy_words((uint32_t*)s.w2, HS / 2, (const uint32_t*)wt.w2, kHidden / 2, kHidden, kHidden / 2);
  copy_words((uint32_t*)s.w3, HS / 2, (const uint32_t*)wt.w3, kHidden / 2, 8, kHidden / 2);
}

// Forward pass of one warp's 16 rows (rows r0 .. r0+15 of the tile in s.x).
// y: network outputs in the C-fragment layout (column 2t + (c & 1), row
// g + 8 (c >> 1)); only columns 0..3 are meaningful.  TRAIN keeps the GELU
// derivatives and the bf16 activations for the backward pass.
template <bool TRAIN>
__device__ __forceinline__ void forward16(const Smem& s, const float* __restrict__ bias, int r0, float (&y)[4],
                                          float (&d1)[8][4], float (&d2)[8][4], uint32_t (&a1)[4][4],
                                          uint32_t (&a2)[4][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[j][c] = 0.0f;
  const uint32_t* xr = (const uint32_t*)(s.x + (r0 + g) * XS);
  const uint32_t* xr8 = (const uint32_t*)(s.x + (r0 + g + 8) * XS);
#pragma unroll 4
  for (int kk = 0; kk < kK1 / 16; ++kk) {
    const uint32_t x0 = xr[8 * kk + t], x1 = xr8[8 * kk + t], x2 = xr[8 * kk + 4 + t], x3 = xr8[8 * kk + 4 + t];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t* wr = (const uint32_t*)(s.w1 + (8 * j + g) * XS);
      mma16816(acc[j], x0, x1, x2, x3, wr[8 * kk + t], wr[8 * kk + 4 + t]);
    }
  }
  // layer 1 epilogue: bias, GELU, bf16 A fragments of layer 2
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float dz;
      a[c] = gelu(acc[j][c] + __ldg(bias + dn::kB1 + 8 * j + 2 * t + (c & 1)), dz);
      if (TRAIN) d1[j][c] = dz;
    }
    a1[j >> 1][(j & 1) * 2 + 0] = pack2(a[0], a[1]);
    a1[j >> 1][(j & 1) * 2 + 1] = pack2(a[2], a[3]);
  }
  // a1[kk][0] = row g, units 16kk + 2t; [1] = row g+8; [2] = units + 8, row g; [3] = row g+8, units + 8
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[j][c] = 0.0f;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t* wr = (const uint32_t*)(s.w2 + (8 * j + g) * HS);
      mma16816(acc[j], a1[kk][0], a1[kk][1], a1[kk][2], a1[kk][3], wr[8 * kk + t], wr[8 * kk + 4 + t]);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float dz;
      a[c] = gelu(acc[j][c] + __ldg(bias + dn::kB2 + 8 * j + 2 * t + (c & 1)), dz);
      if (TRAIN) d2[j][c] = dz;
    }
    a2[j >> 1][(j & 1) * 2 + 0] = pack2(a[0], a[1]);
    a2[j >> 1][(j & 1) * 2 + 1] = pack2(a[2], a[3]);
  }
  float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const uint32_t* wr = (const uint32_t*)(s.w3 + g * HS);
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) mma16816(o, a2[kk][0], a2[kk][1], a2[kk][2], a2[kk][3], wr[8 * kk + t], wr[8 * kk + 4 + t]);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int col = 2 * t + (c & 1);
    y[c] = col < kOut ? o[c] + __ldg(bias + dn::kB3 + col) : 0.0f;
  }
}

// ------------------------------------------------------------------ features
__global__ void dn_features_kernel(uint32_t n, uint32_t w, uint32_t h, const uint32_t* __restrict__ indices,
                                   const uint32_t* __restrict__ tidx, const float4* __restrict__ coords,
                                   const float* __restrict__ ao, const float* __restrict__ bn3,
                                   const float* __restrict__ pos3, const float* __restrict__ nrm3, float max_d,
                                   float4* f0, float4* f1, float4* f2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = __ldg(indices + i);
  if (p >= w * h || __ldg(tidx + i) == kMiss) return;  // stays zero: no coverage
  float bx = __ldg(bn3 + 3 * (size_t)i), by = __ldg(bn3 + 3 * (size_t)i + 1), bz = __ldg(bn3 + 3 * (size_t)i + 2);
  const float2 ob = oct_encode(bx, by, bz);
  const float2 on = oct_encode(__ldg(nrm3 + 3 * (size_t)i), __ldg(nrm3 + 3 * (size_t)i + 1),
                               __ldg(nrm3 + 3 * (size_t)i + 2));
  f0[p] = make_float4(__ldg(ao + i), ob.x, ob.y, 1.0f);
  f1[p] = make_float4(__ldg(pos3 + 3 * (size_t)i) / max_d, __ldg(pos3 + 3 * (size_t)i + 1) / max_d,
                      __ldg(pos3 + 3 * (size_t)i + 2) / max_d, __ldg(coords + i).x / max_d);
  f2[p] = make_float4(on.x, on.y, 0.0f, 0.0f);
}

// Texel spacing of each covered pixel: the mean distance (in position / max
// distance units) to its covered 4-neighbours, right, left, down, up; 0 when
// none is covered.  Stored in plane 2's z.
__global__ void dn_spacing_kernel(uint32_t n, uint32_t w, uint32_t h, const uint32_t* __restrict__ indices,
                                  const float4* __restrict__ f0, const float4* __restrict__ f1, float4* f2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = __ldg(indices + i);
  if (p >= w * h || !(__ldg(f0 + p).w > 0.0f)) return;
  const int x = (int)(p % w), y = (int)(p / w);
  const int nx[4] = {x + 1, x - 1, x, x}, ny[4] = {y, y, y + 1, y - 1};
  const float4 c = __ldg(f1 + p);
  float sum = 0.0f;
  int k = 0;
  for (int j = 0; j < 4; ++j) {
    if (nx[j] < 0 || ny[j] < 0 || nx[j] >= (int)w || ny[j] >= (int)h) continue;
    const uint32_t q = (uint32_t)ny[j] * w + (uint32_t)nx[j];
    if (!(__ldg(f0 + q).w > 0.0f)) continue;
    const float4 b = __ldg(f1 + q);
    const float dx = b.x - c.x, dy = b.y - c.y, dz = b.z - c.z;
    sum += sqrtf((dx * dx + dy * dy) + dz * dz);
    ++k;
  }
  f2[p].z = k ? sum / (float)k : 0.0f;
}

// Input rows for a list of pixels (kNoTexel or out-of-image: an all-zero row).
__global__ void dn_rows_kernel(const float4* __restrict__ f0, const float4* __restrict__ f1,
                               const float4* __restrict__ f2, uint32_t w, uint32_t h,
                               const uint32_t* __restrict__ pixels, uint32_t n, uint32_t* rows) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  uint32_t p = __ldg(pixels + warp);
  if (p >= w * h) p = kNoTexel;
  assemble_row(f0, f1, f2, w, h, p, lane, rows + (size_t)warp * (kK1 / 2));
}

// ------------------------------------------------------------------ training
struct TrainArgs {
  const uint32_t* rows;     // [nrows][128 words] bf16 inputs
  const float4* targets;    // [nrows] (dAO, dBN.xyz) residual targets
  const uint32_t* row_ids;  // batch row -> dataset row (null: identity from offset)
  uint32_t nrows, offset;
  float scale;              // 2 / (4 x batch): d(mean squared error)/dy
  DnWeights wt;
  float* partials;          // [tiles][kParams]
  float* loss;              // [tiles] sum of squared errors
  int* status;
};

__global__ void __launch_bounds__(256, 1) dn_train_kernel(TrainArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* base = (__nv_bfloat16*)smem_raw;
  Smem s;
  s.x = base;
  s.w1 = s.x + kRows * XS;
  s.w2 = s.w1 + kHidden * XS;
  s.w3 = s.w2 + kHidden * HS;
  __nv_bfloat16* w2t = s.w3 + 8 * HS;     // [64][HS] (in, out)
  __nv_bfloat16* w3t = w2t + kHidden * HS; // [64][8]  (unit, out)
  __nv_bfloat16* a1s = w3t + kHidden * 8;  // [kRows][HS]
  __nv_bfloat16* a2s = a1s + kRows * HS;   // [kRows][HS]
  __nv_bfloat16* dz1t = a2s + kRows * HS;  // [64][TS]
  __nv_bfloat16* dz2t = dz1t + kHidden * TS;
  __nv_bfloat16* dyt = dz2t + kHidden * TS;  // [16][TS], rows 4..15 zero
  float* bsum = (float*)(dyt + 16 * TS);     // [8 warps][64 + 64 + 4]
  float* lsum = bsum + 8 * 132;              // [8]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  load_forward_weights(s, p.wt);
  copy_words((uint32_t*)w2t, HS / 2, (const uint32_t*)p.wt.w2t, kHidden / 2, kHidden, kHidden / 2);
  copy_words((uint32_t*)w3t, 4, (const uint32_t*)p.wt.w3t, 4, kHidden, 4);
  for (int i = tid; i < 16 * TS / 2; i += blockDim.x) ((uint32_t*)dyt)[i] = 0u;
  // this warp's 16 rows of the tile
  const int r0 = warp * 16;
  uint32_t rid[2] = {0, 0};
  bool rok[2] = {false, false};
  for (int rr = 0; rr < 16; ++rr) {
    const uint32_t b = p.offset + blockIdx.x * kRows + r0 + rr;
    uint32_t r = p.row_ids ? __ldg(p.row_ids + b) : b;
    const bool ok = r < p.nrows;
    if (!ok && lane == 0) atomicOr(p.status, 8);
    const uint4 v = ok ? __ldg((const uint4*)(p.rows + (size_t)r * (kK1 / 2)) + lane) : make_uint4(0, 0, 0, 0);
    *((uint4*)(s.x + (r0 + rr) * XS) + lane) = v;
    if (rr == g) { rid[0] = r; rok[0] = ok; }
    if (rr == g + 8) { rid[1] = r; rok[1] = ok; }
  }
  __syncthreads();

  float y[4], d1[8][4], d2[8][4];
  uint32_t a1[4][4], a2[4][4];
  forward16<true>(s, p.wt.params, r0, y, d1, d2, a1, a2);

  // loss and dY (C layout, columns 0..3 valid)
  float dy[4], se = 0.0f;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int col = 2 * t + (c & 1), h = c >> 1;
    dy[c] = 0.0f;
    if (col < kOut && rok[h]) {
      const float4 tv = __ldg(p.targets + rid[h]);
      const float tc = col == 0 ? tv.x : (col == 1 ? tv.y : (col == 2 ? tv.z : tv.w));
      const float d = y[c] - tc;
      se += d * d;
      dy[c] = p.scale * d;
    }
  }
  // dA2 = dY W3  (K = 8 outputs padded to 16)
  const uint32_t dya0 = pack2(dy[0], dy[1]), dya1 = pack2(dy[2], dy[3]);
  float da[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
#pragma unroll
    for (int c = 0; c < 4; ++c) da[j][c] = 0.0f;
    const uint32_t b0 = ((const uint32_t*)(w3t + (8 * j + g) * 8))[t];
    mma16816(da[j], dya0, dya1, 0u, 0u, b0, 0u);
  }
  // dZ2 = dA2 * GELU'(Z2); dA1 = dZ2 W2
  uint32_t dz2a[4][4];
  float dz2[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
#pragma unroll
    for (int c = 0; c < 4; ++c) dz2[j][c] = da[j][c] * d2[j][c];
    dz2a[j >> 1][(j & 1) * 2 + 0] = pack2(dz2[j][0], dz2[j][1]);
    dz2a[j >> 1][(j & 1) * 2 + 1] = pack2(dz2[j][2], dz2[j][3]);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int c = 0; c < 4; ++c) da[j][c] = 0.0f;
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t* wr = (const uint32_t*)(w2t + (8 * j + g) * HS);
      mma16816(da[j], dz2a[kk][0], dz2a[kk][1], dz2a[kk][2], dz2a[kk][3], wr[8 * kk + t], wr[8 * kk + 4 + t]);
    }
  }
  // stage transposed gradients and activations for the weight gradients
#pragma unroll
  for (int j = 0; j < 8; ++j) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int unit = 8 * j + 2 * t + (c & 1), row = r0 + g + 8 * (c >> 1);
      const float dz1 = da[j][c] * d1[j][c];
      da[j][c] = dz1;
      ((uint16_t*)dz1t)[unit * TS + row] = bf16_bits(dz1);
      ((uint16_t*)dz2t)[unit * TS + row] = bf16_bits(dz2[j][c]);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int col = 2 * t + (c & 1), row = r0 + g + 8 * (c >> 1);
    if (col < kOut) ((uint16_t*)dyt)[col * TS + row] = bf16_bits(dy[c]);
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    uint32_t* r1 = (uint32_t*)(a1s + (r0 + g) * HS);
    uint32_t* r18 = (uint32_t*)(a1s + (r0 + g + 8) * HS);
    uint32_t* r2 = (uint32_t*)(a2s + (r0 + g) * HS);
    uint32_t* r28 = (uint32_t*)(a2s + (r0 + g + 8) * HS);
    r1[8 * kk + t] = a1[kk][0];
    r18[8 * kk + t] = a1[kk][1];
    r1[8 * kk + 4 + t] = a1[kk][2];
    r18[8 * kk + 4 + t] = a1[kk][3];
    r2[8 * kk + t] = a2[kk][0];
    r28[8 * kk + t] = a2[kk][1];
    r2[8 * kk + 4 + t] = a2[kk][2];
    r28[8 * kk + 4 + t] = a2[kk][3];
  }
  // bias gradients: column sums over this warp's rows in fixed order
#pragma unroll
  for (int j = 0; j < 8; ++j) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      float s1 = da[j][q] + da[j][q + 2], s2 = dz2[j][q] + dz2[j][q + 2];
      for (int off = 4; off < 32; off <<= 1) {
        s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, off);
        s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, off);
      }
      if (g == 0) {
        bsum[warp * 132 + 8 * j + 2 * t + q] = s1;
        bsum[warp * 132 + 64 + 8 * j + 2 * t + q] = s2;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    float s3 = dy[q] + dy[q + 2];
    for (int off = 4; off < 32; off <<= 1) s3 += __shfl_xor_sync(0xFFFFFFFFu, s3, off);
    if (g == 0 && 2 * t + q < kOut) bsum[warp * 132 + 128 + 2 * t + q] = s3;
  }
  for (int off = 1; off < 32; off <<= 1) se += __shfl_xor_sync(0xFFFFFFFFu, se, off);
  if (lane == 0) lsum[warp] = se;
  __syncthreads();

  float* part = p.partials + (size_t)blockIdx.x * dn::kParams;
  const uint16_t* xs16 = (const uint16_t*)s.x;
  // dW1 = dZ1^T X: 64 units x 256 inputs, K = 128 rows; warp w: inputs 32w .. 32w+31
  {
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[i][jj][c] = 0.0f;
#pragma unroll 2
    for (int kk = 0; kk < kRows / 16; ++kk) {
      uint32_t af[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const uint32_t* ar = (const uint32_t*)(dz1t + (16 * i + g) * TS);
        const uint32_t* ar8 = (const uint32_t*)(dz1t + (16 * i + g + 8) * TS);
        af[i][0] = ar[8 * kk + t];
        af[i][1] = ar8[8 * kk + t];
        af[i][2] = ar[8 * kk + 4 + t];
        af[i][3] = ar8[8 * kk + 4 + t];
      }
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int f = 32 * warp + 8 * jj + g, k0 = 16 * kk + 2 * t;
        const uint32_t b0 = pack_u16(xs16[k0 * XS + f], xs16[(k0 + 1) * XS + f]);
        const uint32_t b1 = pack_u16(xs16[(k0 + 8) * XS + f], xs16[(k0 + 9) * XS + f]);
#pragma unroll
        for (int i = 0; i < 4; ++i) mma16816(acc[i][jj], af[i][0], af[i][1], af[i][2], af[i][3], b0, b1);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int unit = 16 * i + g + 8 * (c >> 1), f = 32 * warp + 8 * jj + 2 * t + (c & 1);
          part[dn::kW1 + unit * kK1 + f] = acc[i][jj][c];
        }
  }
  // dW2 = dZ2^T A1 (64 x 64) and dW3 = dY^T A2 (4 x 64); warp w: input units 8w .. 8w+7
  {
    float acc[4][4], acc3[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][c] = 0.0f;
    const uint16_t* a1h = (const uint16_t*)a1s;
    const uint16_t* a2h = (const uint16_t*)a2s;
#pragma unroll 2
    for (int kk = 0; kk < kRows / 16; ++kk) {
      const int u = 8 * warp + g, k0 = 16 * kk + 2 * t;
      const uint32_t b0 = pack_u16(a1h[k0 * HS + u], a1h[(k0 + 1) * HS + u]);
      const uint32_t b1 = pack_u16(a1h[(k0 + 8) * HS + u], a1h[(k0 + 9) * HS + u]);
      const uint32_t c0 = pack_u16(a2h[k0 * HS + u], a2h[(k0 + 1) * HS + u]);
      const uint32_t c1 = pack_u16(a2h[(k0 + 8) * HS + u], a2h[(k0 + 9) * HS + u]);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const uint32_t* ar = (const uint32_t*)(dz2t + (16 * i + g) * TS);
        const uint32_t* ar8 = (const uint32_t*)(dz2t + (16 * i + g + 8) * TS);
        mma16816(acc[i], ar[8 * kk + t], ar8[8 * kk + t], ar[8 * kk + 4 + t], ar8[8 * kk + 4 + t], b0, b1);
      }
      const uint32_t* yr = (const uint32_t*)(dyt + g * TS);
      const uint32_t* yr8 = (const uint32_t*)(dyt + (g + 8) * TS);
      mma16816(acc3, yr[8 * kk + t], yr8[8 * kk + t], yr[8 * kk + 4 + t], yr8[8 * kk + 4 + t], c0, c1);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int o = 16 * i + g + 8 * (c >> 1), u = 8 * warp + 2 * t + (c & 1);
        part[dn::kW2 + o * kHidden + u] = acc[i][c];
      }
#pragma unroll
    for (int c = 0; c < 2; ++c) {  // rows g < 4 only (c >> 1 == 0)
      const int u = 8 * warp + 2 * t + c;
      if (g < kOut) part[dn::kW3 + g * kHidden + u] = acc3[c];
    }
  }
  if (tid < kHidden) {
    float s1 = 0.0f, s2 = 0.0f;
    for (int w = 0; w < 8; ++w) {
      s1 += bsum[w * 132 + tid];
      s2 += bsum[w * 132 + 64 + tid];
    }
    part[dn::kB1 + tid] = s1;
    part[dn::kB2 + tid] = s2;
  }
  if (tid < kOut) {
    float s3 = 0.0f;
    for (int w = 0; w < 8; ++w) s3 += bsum[w * 132 + 128 + tid];
    part[dn::kB3 + tid] = s3;
  }
  if (tid == 0) {
    float l = 0.0f;
    for (int w = 0; w < 8; ++w) l += lsum[w];
    p.loss[blockIdx.x] = l;
  }
}

// Sums the per-tile partial gradients in tile order and applies one Adam
// step (or only reports the gradient when `update` is 0).  Refreshes the
// bf16 working copies of the weights.
struct AdamArgs {
  const float* partials;
  uint32_t tiles;
  float* params;
  float* m;
  float* v;
  float* grad_out;  // optional
  int update;
  float lr, beta1, beta2, eps, c1, c2;  // c1 = 1 / (1 - beta1^t), c2 = 1 / (1 - beta2^t)
  __nv_bfloat16 *w1, *w2, *w2t, *w3, *w3t;
};

__global__ void dn_adam_kernel(AdamArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint32_t)dn::kParams) return;
  float gsum = 0.0f;
  for (uint32_t c = 0; c < a.tiles; ++c) gsum += a.partials[(size_t)c * dn::kParams + i];
  if (a.grad_out) a.grad_out[i] = gsum;
  if (!a.update) return;
  static_assert(dn::kW1 == 0, "W1 leads the parameter block");
  if (i < (uint32_t)dn::kB1 && i % kK1 >= (uint32_t)dn::kInputs) return;  // W1's zero pad columns
  const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * gsum;
  const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * (gsum * gsum);
  a.m[i] = m;
  a.v[i] = v;
  const float mh = m * a.c1, vh = v * a.c2;
  const float w = a.params[i] - a.lr * mh / (sqrtf(vh) + a.eps);
  a.params[i] = w;
  const __nv_bfloat16 b = __float2bfloat16_rn(w);
  if (i < (uint32_t)dn::kB1) {
    a.w1[i] = b;
  } else if (i >= (uint32_t)dn::kW2 && i < (uint32_t)dn::kB2) {
    const uint32_t o = (i - dn::kW2) / kHidden, u = (i - dn::kW2) % kHidden;
    a.w2[o * kHidden + u] = b;
    a.w2t[u * kHidden + o] = b;
  } else if (i >= (uint32_t)dn::kW3 && i < (uint32_t)dn::kB3) {
    const uint32_t o = (i - dn::kW3) / kHidden, u = (i - dn::kW3) % kHidden;
    a.w3[o * kHidden + u] = b;
    a.w3t[u * 8 + o] = b;
  }
}

// bf16 working copies from the fp32 parameters (after a host upload).
__global__ void dn_refresh_kernel(const float* params, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w2t,
                                  __nv_bfloat16* w3, __nv_bfloat16* w3t) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (uint32_t)(kHidden * kK1)) w1[i] = __float2bfloat16_rn(params[dn::kW1 + i]);
  if (i < (uint32_t)(kHidden * kHidden)) {
    const uint32_t o = i / kHidden, u = i % kHidden;
    const __nv_bfloat16 b = __float2bfloat16_rn(params[dn::kW2 + i]);
    w2[i] = b;
    w2t[u * kHidden + o] = b;
  }
  if (i < (uint32_t)(8 * kHidden)) {
    const uint32_t o = i / kHidden, u = i % kHidden;
    const __nv_bfloat16 b = o < (uint32_t)kOut ? __float2bfloat16_rn(params[dn::kW3 + i]) : __float2bfloat16_rn(0.0f);
    w3[i] = b;
    w3t[u * 8 + o] = b;
  }
}

// ------------------------------------------------------------------ inference
struct ApplyArgs {
  const float4 *f0, *f1, *f2;
  uint32_t w, h;
  const uint32_t* indices;  // texel -> pixel
  const uint32_t* tidx;
  const float* ao_in;
  const float* bn_in;
  uint32_t offset, count;
  DnWeights wt;
  float* ao_out;  // null: raw network outputs to y_out
  float* bn_out;
  float4* y_out;
  const uint32_t* rows;  // raw mode over given input rows instead of the feature image
};

__global__ void __launch_bounds__(256, 2) dn_apply_kernel(ApplyArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem s;
  s.x = (__nv_bfloat16*)smem_raw;
  s.w1 = s.x + kRows * XS;
  s.w2 = s.w1 + kHidden * XS;
  s.w3 = s.w2 + kHidden * HS;
  load_forward_weights(s, a.wt);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = warp * 16;
  const uint32_t tiles = (a.count + kRows - 1) / kRows;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t first = a.offset + tile * kRows + r0;
    const uint32_t end = a.offset + a.count;
    for (int rr = 0; rr < 16; ++rr) {
      const uint32_t i = first + rr;
      uint32_t* dst = (uint32_t*)(s.x + (r0 + rr) * XS);
      if (a.rows) {
        const uint4 v = i < end ? __ldg((const uint4*)(a.rows + (size_t)i * (kK1 / 2)) + lane) : make_uint4(0, 0, 0, 0);
        ((uint4*)dst)[lane] = v;
      } else {
        const uint32_t px = i < end ? __ldg(a.indices + i) : kNoTexel;
        assemble_row(a.f0, a.f1, a.f2, a.w, a.h, px < a.w * a.h ? px : kNoTexel, lane, dst);
      }
    }
    __syncwarp();
    float y[4], d1[8][4], d2[8][4];
    uint32_t a1[4][4], a2[4][4];
    forward16<false>(s, a.wt.params, r0, y, d1, d2, a1, a2);
    // lanes t = 0 gather columns 2, 3 from lane t = 1
    const float y2 = __shfl_down_sync(0xFFFFFFFFu, y[0], 1), y3 = __shfl_down_sync(0xFFFFFFFFu, y[1], 1);
    const float y6 = __shfl_down_sync(0xFFFFFFFFu, y[2], 1), y7 = __shfl_down_sync(0xFFFFFFFFu, y[3], 1);
    if (t == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t i = first + g + 8 * h;
        if (i >= end) continue;
        const float o0 = h ? y[2] : y[0], o1 = h ? y[3] : y[1], o2 = h ? y6 : y2, o3 = h ? y7 : y3;
        if (!a.ao_out) {
          a.y_out[i] = make_float4(o0, o1, o2, o3);
          continue;
        }
        float ao = 1.0f, bx = 0.0f, by = 0.0f, bz = 0.0f;
        if (__ldg(a.tidx + i) != kMiss) {
          float cx = __ldg(a.bn_in + 3 * (size_t)i), cy = __ldg(a.bn_in + 3 * (size_t)i + 1),
                cz = __ldg(a.bn_in + 3 * (size_t)i + 2);
          if (!isfinite(cx) || !isfinite(cy) || !isfinite(cz)) cx = cy = cz = 0.0f;
          ao = fminf(fmaxf(__ldg(a.ao_in + i) + o0, 0.0f), 1.0f);
          const float vx = cx + o1, vy = cy + o2, vz = cz + o3;
          const float d = (vx * vx + vy * vy) + vz * vz;
          if (d > 0.0f) {
            const float inv = 1.0f / sqrtf(d);
            bx = vx * inv;
            by = vy * inv;
            bz = vz * inv;
          }
        }
        a.ao_out[i] = ao;
        a.bn_out[3 * (size_t)i] = bx;
        a.bn_out[3 * (size_t)i + 1] = by;
        a.bn_out[3 * (size_t)i + 2] = bz;
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------ inference on tcgen05
// The same network on sm_100's fifth-generation tensor cores: a CTA of one
// warpgroup (128 threads) owns a 128-texel tile; the tile's input rows and the
// weights sit in shared memory in the no-swizzle K-major core-matrix layout
// (8 rows x 16 bytes per core matrix, core matrices 128 bytes apart along K
// and SBO bytes apart along the rows), one elected thread issues
// tcgen05.mma (kind::f16, BF16 operands, FP32 accumulation) for each layer
// into tensor memory, and every thread reads its own row back with
// tcgen05.ld (TMEM lane = tile row) for the bias / GELU epilogue, which writes
// the next layer's operand.  Completion is tracked by an mbarrier that
// tcgen05.commit arrives on; every wait on it is bounded and a timeout stops
// the kernel with status bit 16 after freeing its tensor memory.
namespace tc {
// 16 warps: all gather input rows; for the epilogues, warps w, w + 4, w + 8 and
// w + 12 share TMEM lane quarter w % 4 (the only lanes a warp may read) and
// split its 64 accumulator columns 16 each.
constexpr uint32_t kThreads = 512;
constexpr uint32_t kTmemCols = 128;  // layer 1 / 3 accumulators at column 0, layer 2 at column 64
constexpr uint32_t kA1 = 0;                  // 128 x 256 bf16
constexpr uint32_t kW1 = kA1 + 128 * 256 * 2;  // 64 x 256
constexpr uint32_t kA2 = kW1 + 64 * 256 * 2;   // 128 x 64
constexpr uint32_t kA3 = kA2 + 128 * 64 * 2;   // 128 x 64
constexpr uint32_t kW2 = kA3 + 128 * 64 * 2;   // 64 x 64
constexpr uint32_t kW3 = kW2 + 64 * 64 * 2;    // 16 x 64, rows 4..15 zero
constexpr uint32_t kBar = kW3 + 16 * 64 * 2;   // mbarrier (8 bytes)
constexpr uint32_t kSlot = kBar + 8;           // allocated TMEM address
constexpr uint32_t kBytes = kSlot + 8;
constexpr uint32_t kWaitLimit = 1u << 22;

// Byte offset of element (r, k) in a K-major core-matrix tile whose rows hold
// `kdim` elements: core matrices of 8 rows x 8 elements, 128 bytes each,
// consecutive along K; row groups of 8 are kdim / 8 x 128 bytes apart.
__device__ __forceinline__ uint32_t core_off(uint32_t r, uint32_t k, uint32_t kdim) {
  return (r >> 3) * (kdim * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (row-group) byte offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it)
    if (try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor cores' reads
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// all threads: tensor-core work before this point is ordered before the barrier,
// and work after it after the barrier
__device__ __forceinline__ void sync_all() {
  fence_before();
  __syncthreads();
  fence_after();
}

__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Bias + GELU of 16 accumulator columns (c0 .. c0 + 15) of this thread's row,
// written into the row of the next layer's operand tile (K = 64).
__device__ __forceinline__ void hidden_epilogue(uint32_t taddr, uint32_t c0, const float* __restrict__ bias,
                                                uint8_t* dst, uint32_t row) {
  float v[16];
  ld16(taddr + c0, v);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t w4[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float dz;
      const uint32_t c = c0 + 8 * h + 2 * e;
      const float a0 = gelu(v[8 * h + 2 * e] + __ldg(bias + c), dz);
      const float a1 = gelu(v[8 * h + 2 * e + 1] + __ldg(bias + c + 1), dz);
      w4[e] = pack2(a0, a1);
    }
    *(uint4*)(dst + core_off(row, c0 + 8 * h, 64)) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
  }
}
}  // namespace tc

__global__ void __launch_bounds__(tc::kThreads, 1) dn_apply_tc_kernel(ApplyArgs a, int* status) {
  extern __shared__ __align__(128) unsigned char sm[];
  const uint32_t sb = (uint32_t)__cvta_generic_to_shared(sm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t quarter = warp & 3;          // TMEM lanes 32 quarter .. + 31
  const uint32_t cols = 16 * (warp >> 2);     // this warp's accumulator columns in an epilogue
  const uint32_t row = 32 * quarter + lane;   // tile row = TMEM lane of this thread
  // weights into the core-matrix layout (16-byte chunks of 8 elements)
  for (uint32_t i = threadIdx.x; i < 64 * 32; i += tc::kThreads) {
    const uint32_t n = i / 32, kg = i % 32;
    *(uint4*)(sm + tc::kW1 + tc::core_off(n, 8 * kg, 256)) = __ldg((const uint4*)a.wt.w1 + n * 32 + kg);
  }
  for (uint32_t i = threadIdx.x; i < 64 * 8; i += tc::kThreads) {
    const uint32_t n = i / 8, kg = i % 8;
    *(uint4*)(sm + tc::kW2 + tc::core_off(n, 8 * kg, 64)) = __ldg((const uint4*)a.wt.w2 + n * 8 + kg);
  }
  for (uint32_t i = threadIdx.x; i < 16 * 8; i += tc::kThreads) {
    const uint32_t n = i / 8, kg = i % 8;
    *(uint4*)(sm + tc::kW3 + tc::core_off(n, 8 * kg, 64)) =
        n < 8 ? __ldg((const uint4*)a.wt.w3 + n * 8 + kg) : make_uint4(0, 0, 0, 0);
  }
  const uint32_t bar = sb + tc::kBar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sb + tc::kSlot),
                 "r"(tc::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc::fence_proxy();
  tc::sync_all();
  const uint32_t tmem = *(volatile uint32_t*)(sm + tc::kSlot);
  const uint32_t my_lanes = tmem + ((32 * quarter) << 16);  // this warp's 32 TMEM lanes
  const uint64_t dA1 = tc::smem_desc(sb + tc::kA1, 128, 4096), dW1 = tc::smem_desc(sb + tc::kW1, 128, 4096);
  const uint64_t dA2 = tc::smem_desc(sb + tc::kA2, 128, 1024), dA3 = tc::smem_desc(sb + tc::kA3, 128, 1024);
  const uint64_t dW2 = tc::smem_desc(sb + tc::kW2, 128, 1024), dW3 = tc::smem_desc(sb + tc::kW3, 128, 1024);
  // a descriptor's start address advances 256 bytes (16 elements of K) per MMA: 16 in 16-byte units
  const uint32_t end = a.offset + a.count;
  const uint32_t tiles = (a.count + dn::kRows - 1) / dn::kRows;
  uint32_t parity = 0;
  bool failed = false;  // a bounded wait ran out (agreed by all threads)
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t first = a.offset + tile * dn::kRows;
    // input rows: warp w assembles rows 8w .. 8w + 7
    for (int rr = 0; rr < 8; ++rr) {
      const uint32_t r = (uint32_t)(warp * 8 + rr), i = first + r;
      if (a.rows) {
        const uint4 v = i < end ? __ldg((const uint4*)(a.rows + (size_t)i * (dn::kK1 / 2)) + lane)
                                : make_uint4(0, 0, 0, 0);
        *(uint4*)(sm + tc::kA1 + tc::core_off(r, 8 * lane, 256)) = v;
      } else {
        uint32_t px = i < end ? __ldg(a.indices + i) : kNoTexel;
        if (px >= a.w * a.h) px = kNoTexel;
        if (lane < 25) {
          float v[10];
          neighbour_features(a.f0, a.f1, a.f2, a.w, a.h, px, lane, v);
#pragma unroll
          for (int k = 0; k < 5; ++k)
            *(uint32_t*)(sm + tc::kA1 + tc::core_off(r, 10 * lane + 2 * k, 256)) = pack2(v[2 * k], v[2 * k + 1]);
        } else if (lane == 25) {
          for (int k = 250; k < 256; k += 2) *(uint32_t*)(sm + tc::kA1 + tc::core_off(r, k, 256)) = 0u;
        }
      }
    }
    tc::fence_proxy();
    tc::sync_all();
    // layer 1: D[:, 0..63] = X W1^T over K = 256
    if (threadIdx.x == 0) {
      for (uint32_t s = 0; s < 16; ++s) tc::mma(tmem, dA1 + 16 * s, dW1 + 16 * s, tc::instr_desc(64), s > 0);
      tc::commit(bar);
    }
    parity ^= 1;
    if (!__syncthreads_and(tc::wait(bar, parity ^ 1))) {
      failed = true;
      break;
    }
    tc::fence_after();
    tc::hidden_epilogue(my_lanes, cols, a.wt.params + dn::kB1, sm + tc::kA2, row);
    tc::fence_proxy();
    tc::sync_all();
    // layer 2: D[:, 64..127] = A1 W2^T over K = 64
    if (threadIdx.x == 0) {
      for (uint32_t s = 0; s < 4; ++s) tc::mma(tmem + 64, dA2 + 16 * s, dW2 + 16 * s, tc::instr_desc(64), s > 0);
      tc::commit(bar);
    }
    parity ^= 1;
    if (!__syncthreads_and(tc::wait(bar, parity ^ 1))) {
      failed = true;
      break;
    }
    tc::fence_after();
    tc::hidden_epilogue(my_lanes + 64, cols, a.wt.params + dn::kB2, sm + tc::kA3, row);
    tc::fence_proxy();
    tc::sync_all();
    // layer 3: D[:, 0..15] = A2 W3^T over K = 64 (outputs 4..15 are zero rows of W3)
    if (threadIdx.x == 0) {
      for (uint32_t s = 0; s < 4; ++s) tc::mma(tmem, dA3 + 16 * s, dW3 + 16 * s, tc::instr_desc(16), s > 0);
      tc::commit(bar);
    }
    parity ^= 1;
    if (!__syncthreads_and(tc::wait(bar, parity ^ 1))) {
      failed = true;
      break;
    }
    tc::fence_after();
    float y[16];
    if (cols == 0) tc::ld16(my_lanes, y);  // the output columns: one warp per lane quarter
    const uint32_t i = first + row;
    if (cols == 0 && i < end) {
      const float o0 = y[0] + __ldg(a.wt.params + dn::kB3), o1 = y[1] + __ldg(a.wt.params + dn::kB3 + 1);
      const float o2 = y[2] + __ldg(a.wt.params + dn::kB3 + 2), o3 = y[3] + __ldg(a.wt.params + dn::kB3 + 3);
      if (!a.ao_out) {
        a.y_out[i] = make_float4(o0, o1, o2, o3);
      } else {
        float ao = 1.0f, bx = 0.0f, by = 0.0f, bz = 0.0f;
        if (__ldg(a.tidx + i) != kMiss) {
          float cx = __ldg(a.bn_in + 3 * (size_t)i), cy = __ldg(a.bn_in + 3 * (size_t)i + 1),
                cz = __ldg(a.bn_in + 3 * (size_t)i + 2);
          if (!isfinite(cx) || !isfinite(cy) || !isfinite(cz)) cx = cy = cz = 0.0f;
          ao = fminf(fmaxf(__ldg(a.ao_in + i) + o0, 0.0f), 1.0f);
          const float vx = cx + o1, vy = cy + o2, vz = cz + o3;
          const float d = (vx * vx + vy * vy) + vz * vz;
          if (d > 0.0f) {
            const float inv = 1.0f / sqrtf(d);
            bx = vx * inv;
            by = vy * inv;
            bz = vz * inv;
          }
        }
        a.ao_out[i] = ao;
        a.bn_out[3 * (size_t)i] = bx;
        a.bn_out[3 * (size_t)i + 1] = by;
        a.bn_out[3 * (size_t)i + 2] = bz;
      }
    }
    tc::sync_all();  // the next tile overwrites the operand tiles and the accumulators
  }
  if (failed) {
    if (threadIdx.x == 0) atomicOr(status, 16);
    // let the committed group that timed out drain before the memory is freed
    tc::wait(bar, parity ^ 1);
  }
  tc::sync_all();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kTmemCols) : "memory");
}

// ------------------------------------------------------------------ per-tile verification
__global__ void dn_inverse_kernel(uint32_t n, const uint32_t* __restrict__ indices, uint32_t pixels, uint32_t* inv) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = __ldg(indices + i);
  if (p < pixels) inv[p] = i;
}

// Slot (tile, cell): the first texel with a mapping hit, in row-major order,
// of cell `cell` of a cells x cells grid over the tile; kNoTexel if none.
__global__ void dn_verify_slots_kernel(uint32_t w, uint32_t h, uint32_t tile, uint32_t cells, uint32_t tiles_x,
                                       uint32_t tiles, const uint32_t* __restrict__ inv,
                                       const uint32_t* __restrict__ tidx, uint32_t* slots) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t per = cells * cells;
  if (s >= tiles * per) return;
  const uint32_t tl = s / per, c = s % per;
  const uint32_t cs = (tile + cells - 1) / cells;
  const uint32_t x0 = (tl % tiles_x) * tile + (c % cells) * cs, y0 = (tl / tiles_x) * tile + (c / cells) * cs;
  const uint32_t x1 = min(min(x0 + cs, (tl % tiles_x) * tile + tile), w);
  const uint32_t y1 = min(min(y0 + cs, (tl / tiles_x) * tile + tile), h);
  uint32_t found = kNoTexel;
  for (uint32_t y = y0; y < y1 && found == kNoTexel; ++y)
    for (uint32_t x = x0; x < x1; ++x) {
      const uint32_t i = __ldg(inv + y * w + x);
      if (i != kNoTexel && __ldg(tidx + i) != kMiss) {
        found = i;
        break;
      }
    }
  slots[s] = found;
}

// Per tile: the larger of the AO error and the mean bent-normal component
// error between the denoised values and the full-count values over the tile's
// slots, in slot order; -1 for a tile without slots.
__global__ void dn_tile_error_kernel(uint32_t tiles, uint32_t per, const uint32_t* __restrict__ slots,
                                     const float* __restrict__ ao_d, const float* __restrict__ bn_d,
                                     const float* __restrict__ ao_v, const float* __restrict__ bn_v, float* err) {
  const uint32_t tl = blockIdx.x * blockDim.x + threadIdx.x;
  if (tl >= tiles) return;
  float ea = 0.0f, eb = 0.0f;
  uint32_t k = 0;
  for (uint32_t c = 0; c < per; ++c) {
    const uint32_t i = __ldg(slots + tl * per + c);
    if (i == kNoTexel) continue;
    ++k;
    ea += fabsf(__ldg(ao_d + i) - __ldg(ao_v + i));
    float e = 0.0f;
    for (int q = 0; q < 3; ++q) e += fabsf(__ldg(bn_d + 3 * (size_t)i + q) - __ldg(bn_v + 3 * (size_t)i + q));
    eb += e / 3.0f;
  }
  err[tl] = k ? fmaxf(ea / (float)k, eb / (float)k) : -1.0f;
}

// Texels (with a mapping hit) of the failed tiles, appended in any order.
__global__ void dn_fallback_list_kernel(uint32_t n, uint32_t w, uint32_t tile, uint32_t tiles_x,
                                        const uint32_t* __restrict__ indices, const uint32_t* __restrict__ tidx,
                                        const uint8_t* __restrict__ failed, uint32_t* list, uint32_t* count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = __ldg(indices + i);
  const uint32_t tl = (p / w / tile) * tiles_x + (p % w) / tile;
  if (__ldg(failed + tl) && __ldg(tidx + i) != kMiss) list[atomicAdd(count, 1u)] = i;
}

}  // namespace

// ------------------------------------------------------------------ launchers
namespace dn {

size_t train_smem_bytes() {
  return 2 * ((size_t)kRows * XS + (size_t)kHidden * XS + (size_t)kHidden * HS + 8 * HS + (size_t)kHidden * HS +
              (size_t)kHidden * 8 + 2 * (size_t)kRows * HS + 2 * (size_t)kHidden * TS + 16 * (size_t)TS) +
         4 * (8 * 132 + 8);
}
size_t apply_smem_bytes() { return 2 * ((size_t)kRows * XS + (size_t)kHidden * XS + (size_t)kHidden * HS + 8 * HS); }

cudaError_t launch_features(cudaStream_t st, uint32_t n, uint32_t w, uint32_t h, const uint32_t* indices,
                            const uint32_t* tidx, const float4* coords, const float* ao, const float* bn3,
                            const float* pos3, const float* nrm3, float max_d, float4* image) {
  const size_t px = (size_t)w * h;
  cudaError_t e = cudaMemsetAsync(image, 0, 3 * px * sizeof(float4), st);
  if (e != cudaSuccess || n == 0) return e;
  dn_features_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, w, h, indices, tidx, coords, ao, bn3, pos3, nrm3, max_d,
                                                       image, image + px, image + 2 * px);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  dn_spacing_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, w, h, indices, image, image + px, image + 2 * px);
  return cudaGetLastError();
}

cudaError_t launch_rows(cudaStream_t st, const float4* image, uint32_t w, uint32_t h, const uint32_t* pixels,
                        uint32_t n, uint32_t* rows) {
  if (n == 0) return cudaSuccess;
  const size_t px = (size_t)w * h;
  dn_rows_kernel<<<(uint32_t)(((size_t)n * 32 + 255) / 256), 256, 0, st>>>(image, image + px, image + 2 * px, w, h,
                                                                            pixels, n, rows);
  return cudaGetLastError();
}

cudaError_t launch_train(cudaStream_t st, const uint32_t* rows, const float4* targets, const uint32_t* row_ids,
                         uint32_t nrows, uint32_t offset, uint32_t batch, const DnWeights& wt, float* partials,
                         float* loss, int* status) {
  const size_t smem = train_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(dn_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  TrainArgs p;
  p.rows = rows;
  p.targets = targets;
  p.row_ids = row_ids;
  p.nrows = nrows;
  p.offset = offset;
  p.scale = 2.0f / (4.0f * (float)batch);
  p.wt = wt;
  p.partials = partials;
  p.loss = loss;
  p.status = status;
  dn_train_kernel<<<batch / kRows, 256, smem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_adam(cudaStream_t st, const float* partials, uint32_t tiles, float* params, float* m, float* v,
                        float* grad_out, int update, float lr, float beta1, float beta2, float eps, float c1, float c2,
                        const DnWeights& wt) {
  AdamArgs a;
  a.partials = partials;
  a.tiles = tiles;
  a.params = params;
  a.m = m;
  a.v = v;
  a.grad_out = grad_out;
  a.update = update;
  a.lr = lr;
  a.beta1 = beta1;
  a.beta2 = beta2;
  a.eps = eps;
  a.c1 = c1;
  a.c2 = c2;
  a.w1 = (__nv_bfloat16*)wt.w1;
  a.w2 = (__nv_bfloat16*)wt.w2;
  a.w2t = (__nv_bfloat16*)wt.w2t;
  a.w3 = (__nv_bfloat16*)wt.w3;
  a.w3t = (__nv_bfloat16*)wt.w3t;
  dn_adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_refresh(cudaStream_t st, const DnWeights& wt) {
  dn_refresh_kernel<<<(kHidden * kK1 + 255) / 256, 256, 0, st>>>(
      wt.params, (__nv_bfloat16*)wt.w1, (__nv_bfloat16*)wt.w2, (__nv_bfloat16*)wt.w2t, (__nv_bfloat16*)wt.w3,
      (__nv_bfloat16*)wt.w3t);
  return cudaGetLastError();
}

cudaError_t launch_apply(cudaStream_t st, int sm_count, const float4* image, uint32_t w, uint32_t h,
                         const uint32_t* indices, const uint32_t* tidx, const float* ao_in, const float* bn_in,
                         uint32_t offset, uint32_t count, const DnWeights& wt, float* ao_out, float* bn_out,
                         const uint32_t* rows, float4* y_out) {
  const size_t smem = apply_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(dn_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (count == 0) return cudaSuccess;
  ApplyArgs a;
  const size_t px = (size_t)w * h;
  a.f0 = image;
  a.f1 = image ? image + px : nullptr;
  a.f2 = image ? image + 2 * px : nullptr;
  a.w = w;
  a.h = h;
  a.indices = indices;
  a.tidx = tidx;
  a.ao_in = ao_in;
  a.bn_in = bn_in;
  a.offset = offset;
  a.count = count;
  a.wt = wt;
  a.ao_out = ao_out;
  a.bn_out = bn_out;
  a.y_out = y_out;
  a.rows = rows;
  const uint32_t tiles = (count + kRows - 1) / kRows;
  const uint32_t blocks = std::min<uint32_t>(tiles, (uint32_t)sm_count * 2);
  dn_apply_kernel<<<blocks, 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_apply_tc(cudaStream_t st, int sm_count, const float4* image, uint32_t w, uint32_t h,
                            const uint32_t* indices, const uint32_t* tidx, const float* ao_in, const float* bn_in,
                            uint32_t offset, uint32_t count, const DnWeights& wt, float* ao_out, float* bn_out,
                            const uint32_t* rows, float4* y_out, int* status) {
  cudaError_t e = cudaFuncSetAttribute(dn_apply_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::kBytes);
  if (e != cudaSuccess) return e;
  if (count == 0) return cudaSuccess;
  ApplyArgs a;
  const size_t px = (size_t)w * h;
  a.f0 = image;
  a.f1 = image ? image + px : nullptr;
  a.f2 = image ? image + 2 * px : nullptr;
  a.w = w;
  a.h = h;
  a.indices = indices;
  a.tidx = tidx;
  a.ao_in = ao_in;
  a.bn_in = bn_in;
  a.offset = offset;
  a.count = count;
  a.wt = wt;
  a.ao_out = ao_out;
  a.bn_out = bn_out;
  a.y_out = y_out;
  a.rows = rows;
  const uint32_t tiles = (count + kRows - 1) / kRows;
  const uint32_t blocks = std::min<uint32_t>(tiles, (uint32_t)sm_count);  // one CTA per SM (141 KB of shared memory)
  dn_apply_tc_kernel<<<blocks, tc::kThreads, tc::kBytes, st>>>(a, status);
  return cudaGetLastError();
}

cudaError_t launch_inverse(cudaStream_t st, uint32_t n, const uint32_t* indices, uint32_t pixels, uint32_t* inv) {
  cudaError_t e = cudaMemsetAsync(inv, 0xFF, (size_t)pixels * 4, st);
  if (e != cudaSuccess || n == 0) return e;
  dn_inverse_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, indices, pixels, inv);
  return cudaGetLastError();
}

cudaError_t launch_verify_slots(cudaStream_t st, uint32_t w, uint32_t h, uint32_t tile, uint32_t cells,
                                const uint32_t* inv, const uint32_t* tidx, uint32_t* slots) {
  const uint32_t tx = (w + tile - 1) / tile, ty = (h + tile - 1) / tile;
  const uint32_t n = tx * ty * cells * cells;
  dn_verify_slots_kernel<<<(n + 255) / 256, 256, 0, st>>>(w, h, tile, cells, tx, tx * ty, inv, tidx, slots);
  return cudaGetLastError();
}

cudaError_t launch_tile_error(cudaStream_t st, uint32_t tiles, uint32_t per, const uint32_t* slots, const float* ao_d,
                              const float* bn_d, const float* ao_v, const float* bn_v, float* err) {
  dn_tile_error_kernel<<<(tiles + 255) / 256, 256, 0, st>>>(tiles, per, slots, ao_d, bn_d, ao_v, bn_v, err);
  return cudaGetLastError();
}

cudaError_t launch_fallback_list(cudaStream_t st, uint32_t n, uint32_t w, uint32_t tile, const uint32_t* indices,
                                 const uint32_t* tidx, const uint8_t* failed, uint32_t* list, uint32_t* count) {
  const uint32_t tx = (w + tile - 1) / tile;
  cudaError_t e = cudaMemsetAsync(count, 0, 4, st);
  if (e != cudaSuccess || n == 0) return e;
  dn_fallback_list_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, w, tile, tx, indices, tidx, failed, list, count);
  return cudaGetLastError();
}

}  // namespace dn
}  // namespace fk
