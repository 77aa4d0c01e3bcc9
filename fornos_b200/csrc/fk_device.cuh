// Device-side arithmetic for the bake kernels.
//
// Hit identity must match the reference's shaders bit for bit, so every
// parity-relevant operation is an explicit IEEE-rounded intrinsic: no FMA
// contraction (the build also passes --fmad=false), correctly rounded division
// and square root, fminf / fmaxf (a NaN operand loses), dot products summed
// left to right, normalize(v) = v * (1 / sqrt(dot(v, v))) (Src/math.h:110-113).
#pragma once
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace fk {

static constexpr uint32_t kMiss = 0xFFFFFFFFu;

struct f3 {
  float x, y, z;
};

__device__ __forceinline__ f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ f3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ f3 neg(f3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ f3 scale(f3 a, float k) { return mk3(__fmul_rn(a.x, k), __fmul_rn(a.y, k), __fmul_rn(a.z, k)); }
__device__ __forceinline__ f3 divv(f3 a, f3 b) { return mk3(__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y), __fdiv_rn(a.z, b.z)); }
__device__ __forceinline__ float dot(f3 a, f3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return mk3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
             __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ f3 normalize(f3 v) { return scale(v, __fdiv_rn(1.0f, __fsqrt_rn(dot(v, v)))); }
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return mk3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return mk3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
// a*w.x + b*w.y + c*w.z, evaluated ((a*wx + b*wy) + c*wz) as the shaders write it
__device__ __forceinline__ f3 blend3(f3 a, f3 b, f3 c, float wx, float wy, float wz) {
  return add(add(scale(a, wx), scale(b, wy)), scale(c, wz));
}

// RayAABB of Shaders/ao_step1.comp:43-52 (same in every shader): entry distance
// when the slab interval is non-empty and not behind the origin, else FLT_MAX.
__device__ __forceinline__ float ray_box(f3 o, f3 d, f3 lo, f3 hi) {
  f3 t1 = divv(sub(lo, o), d);
  f3 t2 = divv(sub(hi, o), d);
  f3 tn = vmin(t1, t2), tx = vmax(t1, t2);
  float a = fmaxf(tn.x, fmaxf(tn.y, tn.z));
  float b = fminf(tx.x, fminf(tx.y, tx.z));
  return (b >= 0.0f && a <= b) ? a : FLT_MAX;
}

// Filtered form of ray_box for a ray traced many times against boxes: the
// six slab quotients q = fl(num / d) are replaced by q' = fl(num * fl(1 / d)).
// For d != 0 with |d| >= 2^-100 and |num| < 2^26, |q' - q| <= 2^-22 |q'| +
// 2^-125 (two roundings of relative size 2^-24 each, one more for q itself,
// and an absolute term for subnormal quotients); for d = 0 both forms give
// the same +-inf or NaN.  min / max keep that bound for the entry and exit
// distances a, b.  A decision (b >= 0, a <= b, a < thr) is taken from a', b'
// only when it holds with those margins; otherwise the exact quotients decide.
// The outcome is therefore always that of ray_box(o, d, lo, hi) < thr.
struct RayPre {
  f3 o, d, inv;
  f3 ol, oh;        // box_near: per-axis offsets of the near and far faces
  bool exact_only;  // the filtered decision's premises fail: always divide
};

__device__ __forceinline__ RayPre ray_pre(f3 o, f3 d) {
  RayPre r;
  r.o = o;
  r.d = d;
  r.inv = mk3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
  const float tiny = 7.8886091e-31f;  // 2^-100
  r.exact_only = (d.x != 0.0f && fabsf(d.x) < tiny) || (d.y != 0.0f && fabsf(d.y) < tiny) ||
                 (d.z != 0.0f && fabsf(d.z) < tiny);
  r.ol = mk3(FLT_MAX, FLT_MAX, FLT_MAX);
  r.oh = mk3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  return r;
}

// Terms of box_near on one axis, for origin o, direction d and a scene whose
// boxes lie within [lo, hi] on this axis (the root box).  Let M bound |o| and
// every face coordinate f, and inv = fl(1 / d).  The slab value box_near
// computes, fl(f * inv - fl(fl(o * inv) +- m)), and the reference's,
// fl(fl(f - o) / d), both lie within 2 |Q| u + |o inv| u (+ subnormal terms)
// of the real Q = (f - o) / d, with |Q| <= 2 M |inv| (1 + u) and u = 2^-24;
// their difference is therefore below 10.02 u M |inv| + 2^-149, and so is
// the rounding of ol / oh themselves.  The margin m = 2^-20 M |inv| +
// 2^-126 (16 u per unit, rounded) covers that, so the near face's value,
// shifted by -m, is at most the reference's, and the far face's, shifted by
// +m, at least.  The products stay below 2^124 when M |inv| < 2^120.  An axis
// where that fails, or where |d| < 2^-100 (including d = 0), is left
// unconstrained (slab values -FLT_MAX / +FLT_MAX: the box's other axes
// decide), and the ray then takes the exact quotients in box_hit.  M below
// 2^24 is box_hit's premise (|f - o| < 2^26) as well.
__device__ __forceinline__ void near_far_axis(float o, float d, float lo, float hi, float& inv, float& ol, float& oh,
                                              bool& exact) {
  const float rc = __frcp_rn(d);
  const float M = fmaxf(fmaxf(fabsf(lo), fabsf(hi)), fabsf(o));
  const float span = __fmul_rn(M, fabsf(rc));
  const bool ok = fabsf(d) >= 7.8886091e-31f && M < 16777216.0f && span < 1.32922800e36f;  // 2^-100, 2^24, 2^120
  const float m = __fmaf_rn(span, 9.53674316e-07f, 1.17549435e-38f);                         // 2^-20, 2^-126
  const float oi = __fmul_rn(o, rc);
  const float sm = rc < 0.0f ? -m : m;
  inv = ok ? rc : 0.0f;
  ol = ok ? __fadd_rn(oi, sm) : FLT_MAX;
  oh = ok ? __fsub_rn(oi, sm) : -FLT_MAX;
  exact = exact || !ok;
}

// Ray terms for both box tests (box_hit, box_near) over a scene with root box
// [L, H] whose coordinates are all below 2^24 in magnitude.
__device__ __forceinline__ RayPre ray_pre_bounded(f3 o, f3 d, f3 L, f3 H) {
  RayPre r;
  r.o = o;
  r.d = d;
  r.exact_only = false;
  near_far_axis(o.x, d.x, L.x, H.x, r.inv.x, r.ol.x, r.oh.x, r.exact_only);
  near_far_axis(o.y, d.y, L.y, H.y, r.inv.y, r.ol.y, r.oh.y, r.exact_only);
  near_far_axis(o.z, d.z, L.z, H.z, r.inv.z, r.ol.z, r.oh.z, r.exact_only);
  return r;
}

// Margins around a filtered slab value v: below(v) <= v - 2^-22 |v| - 2^-125
// and above(v) >= v + 2^-22 |v| + 2^-125, each in two roundings (one fused
// multiply-add with 2^-21, whose rounding costs at most 2^-24 |v|, then the
// absolute term, which survives the rounding exactly where it matters: for
// subnormal v).  For an infinite or NaN v both are NaN, so every comparison
// with them fails and the exact quotients decide.
__device__ __forceinline__ float below(float v) {
  return __fsub_rn(__fmaf_rn(fabsf(v), -4.76837158e-07f, v), 2.3509887e-38f);
}
__device__ __forceinline__ float above(float v) {
  return __fadd_rn(__fmaf_rn(fabsf(v), 4.76837158e-07f, v), 2.3509887e-38f);
}

// Returns ray_box(o, d, lo, hi) < thr exactly, and in `entry` the filtered
// entry distance (for ordering / deferred culling only).  o and d are the
// ray's (kept outside `r` where registers are short); r supplies 1 / d.
__device__ __forceinline__ bool box_hit(const RayPre& r, f3 o, f3 d, f3 lo, f3 hi, float thr, float& entry) {
  f3 n1 = sub(lo, o), n2 = sub(hi, o);
  if (!r.exact_only) {
    f3 t1 = mk3(__fmul_rn(n1.x, r.inv.x), __fmul_rn(n1.y, r.inv.y), __fmul_rn(n1.z, r.inv.z));
    f3 t2 = mk3(__fmul_rn(n2.x, r.inv.x), __fmul_rn(n2.y, r.inv.y), __fmul_rn(n2.z, r.inv.z));
    f3 tn = vmin(t1, t2), tx = vmax(t1, t2);
    float a = fmaxf(tn.x, fmaxf(tn.y, tn.z));
    float b = fminf(tx.x, fminf(tx.y, tx.z));
    entry = a;
    const float a_lo = below(a), b_hi = above(b);
    // certain rejections
    if (b_hi < 0.0f || a_lo > b_hi || a_lo >= thr) return false;
    // certain acceptance (never from a NaN margin)
    const float a_hi = above(a), b_lo = below(b);
    if (b_lo >= 0.0f && a_hi <= b_lo && a_hi < thr) return true;
  }
  f3 t1 = divv(n1, d), t2 = divv(n2, d);
  f3 tn = vmin(t1, t2), tx = vmax(t1, t2);
  float a = fmaxf(tn.x, fmaxf(tn.y, tn.z));
  float b = fminf(tx.x, fminf(tx.y, tx.z));
  entry = a;
  return ((b >= 0.0f && a <= b) ? a : FLT_MAX) < thr;
}
__device__ __forceinline__ bool box_hit(const RayPre& r, f3 lo, f3 hi, float thr, float& entry) {
  return box_hit(r, r.o, r.d, lo, hi, thr, entry);
}

// Conservative test for boxes that only prune (inner records), on the terms
// of ray_pre_bounded: one fused multiply-add per slab value, margins folded
// into the offsets.  The near value of each axis is at most the reference's
// and the far value at least (near_far_axis), min / max keep those bounds,
// so a <= the reference's entry and b >= its exit: whenever
// ray_box(o, d, lo, hi) < thr holds (exit >= 0, entry <= exit, entry < thr)
// this holds too.  `entry` = a is a lower bound of the reference's entry
// distance, for ordering and for culling deferred records (entry < thr).  The
// box must lie within the root box the terms were made for.
__device__ __forceinline__ bool box_near(const RayPre& r, f3 lo, f3 hi, float thr, float& entry) {
  const float t1x = __fmaf_rn(lo.x, r.inv.x, -r.ol.x), t2x = __fmaf_rn(hi.x, r.inv.x, -r.oh.x);
  const float t1y = __fmaf_rn(lo.y, r.inv.y, -r.ol.y), t2y = __fmaf_rn(hi.y, r.inv.y, -r.oh.y);
  const float t1z = __fmaf_rn(lo.z, r.inv.z, -r.ol.z), t2z = __fmaf_rn(hi.z, r.inv.z, -r.oh.z);
  const float a = fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fminf(t1z, t2z));
  const float b = fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fmaxf(t1z, t2z));
  entry = a;
  return fmaxf(a, 0.0f) <= b && a < thr;
}

// Binary64 barycentric of Shaders/meshmapping_nobackfaces.comp:48-62.
__device__ __forceinline__ f3 bary_f64(f3 p, f3 a, f3 b, f3 c) {
  double ax = a.x, ay = a.y, az = a.z;
  double v0x = __dsub_rn((double)b.x, ax), v0y = __dsub_rn((double)b.y, ay), v0z = __dsub_rn((double)b.z, az);
  double v1x = __dsub_rn((double)c.x, ax), v1y = __dsub_rn((double)c.y, ay), v1z = __dsub_rn((double)c.z, az);
  double v2x = __dsub_rn((double)p.x, ax), v2y = __dsub_rn((double)p.y, ay), v2z = __dsub_rn((double)p.z, az);
#define FK_DDOT(ax_, ay_, az_, bx_, by_, bz_) \
  __dadd_rn(__dadd_rn(__dmul_rn(ax_, bx_), __dmul_rn(ay_, by_)), __dmul_rn(az_, bz_))
  double d00 = FK_DDOT(v0x, v0y, v0z, v0x, v0y, v0z);
  double d01 = FK_DDOT(v0x, v0y, v0z, v1x, v1y, v1z);
  double d11 = FK_DDOT(v1x, v1y, v1z, v1x, v1y, v1z);
  double d20 = FK_DDOT(v2x, v2y, v2z, v0x, v0y, v0z);
  double d21 = FK_DDOT(v2x, v2y, v2z, v1x, v1y, v1z);
#undef FK_DDOT
  double den = __dsub_rn(__dmul_rn(d00, d11), __dmul_rn(d01, d01));
  double y = __ddiv_rn(__dsub_rn(__dmul_rn(d11, d20), __dmul_rn(d01, d21)), den);
  double z = __ddiv_rn(__dsub_rn(__dmul_rn(d00, d21), __dmul_rn(d01, d20)), den);
  return mk3(__double2float_rn(__dsub_rn(__dsub_rn(1.0, y), z)), __double2float_rn(y), __double2float_rn(z));
}

}  // namespace fk
