// Image export of Src/image.cpp:22-405 on the device: the compressed texel
// values scattered into the W x H image the reference writes (rows flipped:
// texel (x, y) lands in row h - y - 1), filtered and normalised, quantised to
// RGB8 or kept as float planes, and, for RGB8, dilated.
//
// Dilation (dilateRGB, Src/image.cpp:127-182) visits the pixels in row order
// and reads sources that earlier pixels may have filled.  Which source centre
// a pixel takes depends only on the table of valid pixels, so it is computed
// for every pixel at once; the value is then resolved by following the chain
// of chosen centres that are themselves uncovered and were visited earlier
// (scan index strictly decreasing, so the chain ends), reading the image as it
// was before dilation.  The result is the sequential scan's, pixel for pixel.
#include <algorithm>
#include <cstring>

#include "fk_bvh_rules.h"
#include "fk_internal.h"

namespace fk {
namespace {

constexpr int kThreads = 256;

// (uint8_t) of a float as x86-64 code converts it: truncation to int32
// (0x80000000 for NaN and out-of-range values), low byte kept.
__device__ __forceinline__ uint8_t u8_of(float v) {
  if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
  return (uint8_t)(int32_t)v;
}

// Order-preserving key of a float with the two zeros merged.
__host__ __device__ __forceinline__ uint32_t zkey(float f) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  std::memcpy(&u, &f, 4);
#endif
  if ((u << 1) == 0) u = 0;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// getMinMax (Src/image.cpp:33-43): min / max folds (fk_bvh_rules.h), as keys
// (zeros merged) plus -0 flags: w[0] min key, w[1] max key, w[2] flags.
__global__ void __launch_bounds__(kThreads) export_minmax_kernel(const float* __restrict__ data, uint32_t n,
                                                                 uint32_t* w) {
  float mn = FLT_MAX, mx = -FLT_MAX;
  for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    const float v = data[i];
    mn = bvh::fmin(mn, v);
    mx = bvh::fmax(mx, v);
  }
  for (int d = 16; d > 0; d >>= 1) {
    mn = bvh::fmin(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, d));
    mx = bvh::fmax(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, d));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(w, zkey(mn));
    atomicMax(w + 1, zkey(mx));
    const uint32_t f = (__float_as_uint(mn) == 0x80000000u ? 1u : 0u) | (__float_as_uint(mx) == 0x80000000u ? 2u : 0u);
    if (f) atomicOr(w + 2, f);
  }
}

struct Scatter {
  const float* data;  // 1 or 3 floats per texel
  const uint32_t* idx;
  uint32_t count, w, h;
  int mode;
  int filter, normalize;
  float flo, fhi, scale, bias;
  uint8_t* rgb;    // RGB8 modes
  float* planes;   // float modes: 1 or 3 planes of w x h
};

// exportFloatImage / exportNormalImage / exportVectorImage, per texel.
__global__ void export_scatter_kernel(Scatter a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.count) return;
  const uint32_t id = a.idx[i];
  const size_t x = id % a.w, y = id / a.w;
  if (y >= a.h) return;  // an id outside the map: nothing to write
  const size_t px = (a.h - y - 1) * a.w + x;
  if (a.mode == FK_EXPORT_FLOAT_RGB8) {
    const float d = a.data[i];
    const float df = a.filter && (d < a.flo || d > a.fhi) ? 0.0f : d;
    const float t = __fadd_rn(__fmul_rn(df, a.scale), a.bias);
    const float lo = t < 0.0f ? 0.0f : t;   // std::max(t, 0.0f)
    const float cl = 1.0f < lo ? 1.0f : lo;  // std::min(., 1.0f)
    const uint8_t c = u8_of(__fmul_rn(cl, 255.0f));
    a.rgb[3 * px] = a.rgb[3 * px + 1] = a.rgb[3 * px + 2] = c;
  } else if (a.mode == FK_EXPORT_FLOAT_F32) {
    const float d = a.data[i];
    const float df = a.filter ? bvh::fmin(bvh::fmax(d, a.flo), a.fhi) : d;
    a.planes[px] = a.normalize ? __fadd_rn(__fmul_rn(df, a.scale), a.bias) : df;
  } else if (a.mode == FK_EXPORT_NORMAL_RGB8) {
    for (int k = 0; k < 3; ++k) {
      const float n = __fadd_rn(__fmul_rn(a.data[3 * (size_t)i + k], 0.5f), 0.5f);
      a.rgb[3 * px + k] = u8_of(__fmul_rn(n, 255.0f));
    }
  } else {  // FK_EXPORT_VECTOR_F32: planes B (z), G (y), R (x)
    const size_t plane = (size_t)a.w * a.h;
    a.planes[px] = a.data[3 * (size_t)i + 2];
    a.planes[plane + px] = a.data[3 * (size_t)i + 1];
    a.planes[2 * plane + px] = a.data[3 * (size_t)i];
  }
}

// Valid-pixel tables (Src/image.cpp:83-125), indexed by unflipped x + y w:
// the map's texels, or (normal maps) the texels whose bytes are not all zero,
// with the row taken as index / h as the reference does.
__global__ void export_valid_kernel(const uint32_t* idx, uint32_t count, uint32_t w, uint32_t h, int by_bytes,
                                    const uint8_t* rgb, uint8_t* valid) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t id = idx[i];
  if ((size_t)id >= (size_t)w * h) return;  // outside the map: nothing to mark
  if (!by_bytes) {
    valid[id] = 1;
    return;
  }
  const size_t x = id % w, y = id / h;
  if (y >= h) return;
  const size_t p = 3 * ((h - y - 1) * (size_t)w + x);
  valid[id] = (rgb[p] | rgb[p + 1] | rgb[p + 2]) != 0;
}

// Source centre of each uncovered pixel: the first of the reference's search
// order (distance 1 .. max_dist - 1, 8 directions) strictly inside the image
// with all 8 neighbours valid; -1 when none.
__global__ void export_choice_kernel(const uint8_t* valid, uint32_t w, uint32_t h, int max_dist, int32_t* choice) {
  const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (p >= (size_t)w * h) return;
  int32_t c = -1;
  if (!valid[p]) {
    const int off[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    const int x = (int)(p % w), y = (int)(p / w), W = (int)w, H = (int)h;
    for (int dist = 1; dist < max_dist && c < 0; ++dist)
      for (int k = 0; k < 8; ++k) {
        const int cx = x + off[k][0] * dist, cy = y + off[k][1] * dist;
        if (!(cx > 0 && cy > 0 && cx < W - 1 && cy < H - 1)) continue;
        bool ok = true;
        for (int q = 0; q < 8 && ok; ++q) ok = valid[(size_t)(cx + off[q][0]) + (size_t)(cy + off[q][1]) * w] != 0;
        if (ok) {
          c = cy * W + cx;
          break;
        }
      }
  }
  choice[p] = c;
}

// Dilated value of each uncovered pixel: follows chosen centres that are
// themselves uncovered and earlier in the scan; copies from the image as it
// was before dilation (`src`) into `dst`.
__global__ void export_resolve_kernel(const uint8_t* valid, const int32_t* choice, uint32_t w, uint32_t h,
                                      const uint8_t* src, uint8_t* dst) {
  const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t n = (size_t)w * h;
  if (p >= n || valid[p] || choice[p] < 0) return;
  size_t t = p, s = (size_t)choice[p];
  for (size_t guard = 0; guard < n; ++guard) {  // the scan index strictly decreases along the chain
    if (valid[s] || s > t) break;             // its value at t: unchanged since the start
    const int32_t c = choice[s];
    if (c < 0) break;                         // an earlier pixel with no source kept its value
    t = s;
    s = (size_t)c;
  }
  const size_t a = 3 * ((h - 1 - s / w) * (size_t)w + s % w), b = 3 * ((h - 1 - p / w) * (size_t)w + p % w);
  dst[b] = src[a];
  dst[b + 1] = src[a + 1];
  dst[b + 2] = src[a + 2];
}

float zval(uint32_t k, bool neg_zero) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  std::memcpy(&f, &u, 4);
  return (f == 0.0f && neg_zero) ? -0.0f : f;
}

}  // namespace
}  // namespace fk

extern "C" int fk_export_image(fk_ctx* ctx, const fk_texel_map* map, const fk_buf* data, const fk_export_params* p,
                               fk_buf* image, float* minmax) {
  using namespace fk;
  if (!ctx || !map || !data || !p || !image) return fk_fail(ctx, FK_ERR_INVALID, "fk_export_image: null argument");
  const uint32_t w = map->width, h = map->height, n = map->count;
  const int mode = p->mode;
  if (mode < FK_EXPORT_FLOAT_RGB8 || mode > FK_EXPORT_VECTOR_F32)
    return fk_fail(ctx, FK_ERR_INVALID, "fk_export_image: unknown mode");
  const bool vec3 = mode == FK_EXPORT_NORMAL_RGB8 || mode == FK_EXPORT_VECTOR_F32;
  const bool rgb8 = mode == FK_EXPORT_FLOAT_RGB8 || mode == FK_EXPORT_NORMAL_RGB8;
  const size_t pixels = (size_t)w * h;
  const size_t need = rgb8 ? 3 * pixels : (mode == FK_EXPORT_VECTOR_F32 ? 3 : 1) * pixels * sizeof(float);
  if (data->bytes < (size_t)n * (vec3 ? 12 : 4))
    return fk_fail(ctx, FK_ERR_INVALID, "fk_export_image: data buffer smaller than the texel count");
  if (image->bytes < need) return fk_fail(ctx, FK_ERR_INVALID, "fk_export_image: image buffer too small");
  if (p->dilate > 0 && !rgb8) return fk_fail(ctx, FK_ERR_INVALID, "fk_export_image: dilation needs an RGB8 mode");
  cudaStream_t st = ctx->stream;
  int rc = FK_OK;
  Scatter a{};
  a.data = (const float*)data->ptr;
  a.idx = map->indices;
  a.count = n;
  a.w = w;
  a.h = h;
  a.mode = mode;
  a.filter = p->filter_hi > p->filter_lo;
  a.normalize = p->normalize != 0;
  a.flo = p->filter_lo;
  a.fhi = p->filter_hi;
  a.scale = 1.0f;
  a.bias = 0.0f;
  if (mode == FK_EXPORT_FLOAT_RGB8 || mode == FK_EXPORT_FLOAT_F32) {
    uint32_t* words = nullptr;
    if ((rc = fk_dev_alloc(ctx, (void**)&words, 16)) != FK_OK) return rc;
    const uint32_t init[3] = {zkey(FLT_MAX), zkey(-FLT_MAX), 0};
    uint32_t got[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(words, init, 12, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n) {
      export_minmax_kernel<<<std::min<uint32_t>((n + kThreads - 1) / kThreads, (uint32_t)ctx->sm_count * 4),
                             kThreads, 0, st>>>((const float*)data->ptr, n, words);
      rc = fk_after_launch(ctx, "export min / max");
    }
    if (rc == FK_OK && e == cudaSuccess) e = cudaMemcpyAsync(got, words, 12, cudaMemcpyDeviceToHost, st);
    if (rc == FK_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    fk_dev_free(ctx, words);
    if (rc != FK_OK) return rc;
    if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "export min / max");
    float mn = zval(got[0], got[2] & 1u), mx = zval(got[1], (got[2] & 2u) != 0);
    if (a.filter) {  // Src/image.cpp:201-206
      mn = bvh::fmax(mn, a.flo);
      mx = bvh::fmin(mx, a.fhi);
    }
    if (minmax) {
      minmax[0] = mn;
      minmax[1] = mx;
    }
    if (a.normalize && mn != FLT_MAX && mx != -FLT_MAX) {  // computeScaleBias (Src/image.cpp:59-67)
      a.scale = 1.0f / (mx - mn);
      a.bias = -mn * a.scale;
    }
  }
  FK_CUDA(ctx, cudaMemsetAsync(image->ptr, 0, need, st));
  a.rgb = rgb8 ? (uint8_t*)image->ptr : nullptr;
  a.planes = rgb8 ? nullptr : (float*)image->ptr;
  if (n) {
    export_scatter_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(a);
    if ((rc = fk_after_launch(ctx, "export scatter")) != FK_OK) return rc;
  }
  if (p->dilate > 0 && pixels > 0) {
    uint8_t *valid = nullptr, *before = nullptr;
    int32_t* choice = nullptr;
    rc = fk_dev_alloc(ctx, (void**)&valid, pixels);
    if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&choice, 4 * pixels);
    if (rc == FK_OK) rc = fk_dev_alloc(ctx, (void**)&before, 3 * pixels);
    cudaError_t e = cudaSuccess;
    if (rc == FK_OK) e = cudaMemsetAsync(valid, 0, pixels, st);
    if (rc == FK_OK && e == cudaSuccess) e = cudaMemcpyAsync(before, image->ptr, 3 * pixels, cudaMemcpyDeviceToDevice, st);
    if (rc == FK_OK && e == cudaSuccess && n) {
      export_valid_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(
          map->indices, n, w, h, mode == FK_EXPORT_NORMAL_RGB8, before, valid);
      rc = fk_after_launch(ctx, "export valid pixels");
    }
    const uint32_t blocks = (uint32_t)((pixels + kThreads - 1) / kThreads);
    if (rc == FK_OK && e == cudaSuccess) {
      export_choice_kernel<<<blocks, kThreads, 0, st>>>(valid, w, h, p->dilate, choice);
      rc = fk_after_launch(ctx, "export dilation sources");
    }
    if (rc == FK_OK && e == cudaSuccess) {
      export_resolve_kernel<<<blocks, kThreads, 0, st>>>(valid, choice, w, h, before, (uint8_t*)image->ptr);
      rc = fk_after_launch(ctx, "export dilation");
    }
    if (rc == FK_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);  // before the scratch goes back
    fk_dev_free(ctx, valid);
    fk_dev_free(ctx, choice);
    fk_dev_free(ctx, before);
    if (rc != FK_OK) return rc;
    if (e != cudaSuccess) return fk_cuda_fail(ctx, e, "export dilation");
  }
  return FK_OK;
}
