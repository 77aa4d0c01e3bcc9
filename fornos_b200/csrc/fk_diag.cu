// FP32 throughput probe: the denominator of the traversal roofline.  The ray
// kernels run separately-rounded add / multiply / min / compare instructions
// (no FMA), so the peak they can reach is one such instruction per lane per
// clock; this kernel issues independent chains of exactly those.
#include "fk_internal.h"

namespace fk {

static constexpr int kChains = 8;
static constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) fp32_peak_kernel(float seed, float* sink) {
  float a[kChains], b[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    a[c] = seed + threadIdx.x * 1e-7f + c;
    b[c] = 1.0f + c * 1e-6f;
  }
  for (int i = 0; i < kIters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      a[c] = __fadd_rn(a[c], b[c]);      // 1 op
      b[c] = __fmul_rn(b[c], 0.999999f); // 1 op
      a[c] = fminf(a[c], 1e30f);         // 1 op
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += a[c] + b[c];
  if (s == 12345.678f) *sink = s;  // keeps the chains live
}

}  // namespace fk

extern "C" int fk_diag_fp32_peak(fk_ctx* ctx, double* ops) {
  if (!ctx || !ops) return fk_fail(ctx, FK_ERR_INVALID, "fk_diag_fp32_peak: null");
  float* sink = nullptr;
  int rc = fk_dev_alloc(ctx, (void**)&sink, sizeof(float));
  if (rc != FK_OK) return rc;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fk::fp32_peak_kernel, 256, 0);
  if (per_sm < 1) per_sm = 1;
  const int blocks = ctx->sm_count * per_sm * 4;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    fk::fp32_peak_kernel<<<blocks, 256, 0, ctx->stream>>>(1.0f, sink);
    cudaEventRecord(e1, ctx->stream);
    rc = fk_after_launch(ctx, "fp32_peak_kernel");
    if (rc != FK_OK) break;
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_ms) best_ms = ms;  // first launch is warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  fk_dev_free(ctx, sink);
  if (rc != FK_OK) return rc;
  double total = (double)blocks * 256.0 * fk::kIters * fk::kChains * 3.0;
  *ops = total / (best_ms * 1e-3);
  return FK_OK;
}
