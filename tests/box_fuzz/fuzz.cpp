// Fuzzer of the traversal's box tests, compiled for the host from the device
// source itself (fornos_b200/csrc/fk_device.cuh, through the stand-in
// cuda_runtime.h beside this file).  For random and adversarial rays and
// boxes inside a root box it checks, against the reference's ray_box
// (Shaders/ao_step1.comp:43-52):
//   * box_near never rejects a box the reference accepts (entry < thr), and
//     its entry is then at most the reference's;
//   * box_hit takes exactly the reference's decision.
// Prints the counts: cases, reference acceptances, violations of the first
// rule, mismatches of the second, and the boxes box_near accepts beyond the
// reference's (all rays; rays with every axis constrained).
//
//   fuzz <seed> <cases>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../fornos_b200/csrc/fk_device.cuh"

using namespace fk;

namespace {

std::mt19937_64 rng;

float uni(float a, float b) { return std::uniform_real_distribution<float>(a, b)(rng); }
int pick(int n) { return (int)(rng() % (uint64_t)n); }

// a coordinate in [lo, hi], often exactly on a bound or at zero
float coord(float lo, float hi) {
  switch (pick(8)) {
    case 0: return lo;
    case 1: return hi;
    case 2: return (lo <= 0.0f && hi >= 0.0f) ? 0.0f : lo;
    default: return uni(lo, hi);
  }
}

f3 direction() {
  f3 d = mk3(uni(-1.0f, 1.0f), uni(-1.0f, 1.0f), uni(-1.0f, 1.0f));
  switch (pick(10)) {  // components exactly zero, tiny, or subnormal
    case 0: d.x = 0.0f; break;
    case 1: d.y = 0.0f; d.z = -0.0f; break;
    case 2: d.z = 1e-35f; break;
    case 3: d.x = 1e-42f; break;
    case 4: d.y = 3e-30f; break;
    default: break;
  }
  if (d.x == 0.0f && d.y == 0.0f && d.z == 0.0f) d.z = 1.0f;
  const f3 n = normalize(d);
  // keep deliberately tiny components (normalising a mostly-unit vector keeps them)
  return n;
}

}  // namespace

int main(int argc, char** argv) {
  const unsigned long long seed = argc > 1 ? strtoull(argv[1], nullptr, 10) : 1;
  const long cases = argc > 2 ? atol(argv[2]) : 1000000;
  rng.seed(seed);
  long near_violations = 0, hit_mismatches = 0, near_extra = 0, ref_accepts = 0, regular = 0, regular_extra = 0;
  const float scales[] = {1e-3f, 1.0f, 37.5f, 1e3f, 1e6f};
  for (long i = 0; i < cases; ++i) {
    const float sc = scales[pick(5)];
    const float off = pick(3) == 0 ? 0.0f : uni(-2.0f, 2.0f) * sc;  // root box off the origin
    const f3 L = mk3(off - sc * uni(0.1f, 1.0f), off - sc * uni(0.1f, 1.0f), -sc * uni(0.0f, 1.0f));
    const f3 H = mk3(off + sc * uni(0.1f, 1.0f), off + sc * uni(0.1f, 1.0f), sc * uni(0.0f, 1.0f));
    // a child box inside the root box, sometimes flat on an axis
    f3 a = mk3(coord(L.x, H.x), coord(L.y, H.y), coord(L.z, H.z));
    f3 b = mk3(coord(L.x, H.x), coord(L.y, H.y), coord(L.z, H.z));
    if (pick(6) == 0) b.z = a.z;
    const f3 lo = vmin(a, b), hi = vmax(a, b);
    // the origin in the root box, sometimes on a face of the child box
    f3 o = mk3(coord(L.x, H.x), coord(L.y, H.y), coord(L.z, H.z));
    switch (pick(6)) {
      case 0: o.x = lo.x; break;
      case 1: o.y = hi.y; break;
      case 2: o = lo; break;
      default: break;
    }
    const f3 d = direction();
    float thr;
    switch (pick(4)) {
      case 0: thr = FLT_MAX; break;
      case 1: thr = uni(0.0f, 3.0f) * sc; break;
      case 2: thr = uni(0.0f, 1e-4f) * sc; break;
      default: thr = 0.3f * sc; break;
    }
    const float ref_entry = ray_box(o, d, lo, hi);
    const bool ref = ref_entry < thr;
    ref_accepts += ref;
    const RayPre rp = ray_pre_bounded(o, d, L, H);
    float near_entry = 0.0f;
    const bool near = box_near(rp, lo, hi, thr, near_entry);
    if (ref && (!near || !(near_entry <= ref_entry))) {
      if (near_violations < 10)
        printf("near violation: o (%.9g %.9g %.9g) d (%.9g %.9g %.9g) lo (%.9g %.9g %.9g) hi (%.9g %.9g %.9g) "
               "thr %.9g ref %.9g near %d %.9g\n",
               o.x, o.y, o.z, d.x, d.y, d.z, lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, thr, ref_entry, (int)near,
               near_entry);
      ++near_violations;
    }
    near_extra += near && !ref;
    if (!rp.exact_only) {  // every axis constrained: the margins alone make the difference
      ++regular;
      regular_extra += near && !ref;
    }
    float hit_entry = 0.0f;
    const bool hit = box_hit(rp, o, d, lo, hi, thr, hit_entry);
    if (hit != ref) {
      if (hit_mismatches < 10)
        printf("hit mismatch: o (%.9g %.9g %.9g) d (%.9g %.9g %.9g) thr %.9g ref %d\n", o.x, o.y, o.z, d.x, d.y,
               d.z, thr, (int)ref);
      ++hit_mismatches;
    }
  }
  printf("cases %ld ref_accepts %ld near_violations %ld hit_mismatches %ld near_extra %ld regular %ld "
         "regular_extra %ld\n",
         cases, ref_accepts, near_violations, hit_mismatches, near_extra, regular, regular_extra);
  return near_violations || hit_mismatches ? 1 : 0;
}
