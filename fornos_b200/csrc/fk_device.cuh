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
  bool exact_only;  // some |d| is nonzero but below 2^-100: always divide
};

__device__ __forceinline__ RayPre ray_pre(f3 o, f3 d) {
  RayPre r;
  r.o = o;
  r.d = d;
  r.inv = mk3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
  const float tiny = 7.8886091e-31f;  // 2^-100
  r.exact_only = (d.x != 0.0f && fabsf(d.x) < tiny) || (d.y != 0.0f && fabsf(d.y) < tiny) ||
                 (d.z != 0.0f && fabsf(d.z) < tiny);
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
// entry distance (for ordering / deferred culling only).
__device__ __forceinline__ bool box_hit(const RayPre& r, f3 lo, f3 hi, float thr, float& entry) {
  f3 n1 = sub(lo, r.o), n2 = sub(hi, r.o);
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
  f3 t1 = divv(n1, r.d), t2 = divv(n2, r.d);
  f3 tn = vmin(t1, t2), tx = vmax(t1, t2);
  float a = fmaxf(tn.x, fmaxf(tn.y, tn.z));
  float b = fminf(tx.x, fminf(tx.y, tx.z));
  entry = a;
  return ((b >= 0.0f && a <= b) ? a : FLT_MAX) < thr;
}

// Conservative form for boxes that only prune (inner nodes): false only when
// ray_box(o, d, lo, hi) < thr certainly fails, true when it holds or is
// uncertain.  `entry` is the filtered entry distance.  An infinite entry or a
// minus-infinite exit (a direction component of exactly 0 with the origin
// outside that slab) is a certain miss of the exact test as well; rejecting it
// here matters for speed, since its margins are NaN and the box would
// otherwise be accepted, and with it every box below.  For the rare ray whose
// direction has a component in (0, 2^-100) (exact_only) every box is
// accepted, with entry -FLT_MAX so that deferred culling keeps it: its leaf
// boxes are still tested exactly, so results are unchanged, and the test
// stays free of branches.
__device__ __forceinline__ bool box_maybe(const RayPre& r, f3 lo, f3 hi, float thr, float& entry) {
  f3 n1 = sub(lo, r.o), n2 = sub(hi, r.o);
  f3 t1 = mk3(__fmul_rn(n1.x, r.inv.x), __fmul_rn(n1.y, r.inv.y), __fmul_rn(n1.z, r.inv.z));
  f3 t2 = mk3(__fmul_rn(n2.x, r.inv.x), __fmul_rn(n2.y, r.inv.y), __fmul_rn(n2.z, r.inv.z));
  f3 tn = vmin(t1, t2), tx = vmax(t1, t2);
  float a = fmaxf(tn.x, fmaxf(tn.y, tn.z));
  float b = fminf(tx.x, fminf(tx.y, tx.z));
  const float inf = __int_as_float(0x7f800000);
  const float a_lo = below(a), b_hi = above(b);
  const bool reject = !(a < inf) || !(b > -inf) || b_hi < 0.0f || a_lo > b_hi || a_lo >= thr;
  entry = r.exact_only ? -FLT_MAX : a;
  return r.exact_only || !reject;
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
