// mixed.cuh -- shared pieces of the mixed-precision non-local sum.
//
// Far field in FP32 with the cancellation-free form of the segment formula.  For a
// segment from A to B = A + d seen from x, with r = A - x and e = r + d = B - x, the
// reference's term (timestep.f90:162-169)
//   Gamma/(2 pi) (r x d)/(4ac - b^2) ((2c+b)/sqrt(a+b+c) - b/sqrt(a))
// (a = |r|^2, b = 2 r.d, c = |d|^2) equals
//   Gamma/(4 pi) (r x d) (|r| + |e|) / (|r| |e| (|r| |e| + r.e)),
// which subtracts nothing when the target is far from the segment (r.e ~ +|r||e|), so FP32
// keeps ~1e-7 relative accuracy where the original form loses digits to 4ac - b^2 and to
// the bracket.  The near field (leaves or segments closer than near_radius) and the terms
// FP32 would evaluate badly run in FP64: the reference's own arithmetic decides whether a term
// is skipped (4ac - b^2 against its threshold), and its value comes from the same
// cancellation-free form in FP64 (term64_stable), equal to the reference's to ~1e-15.
#pragma once

#include "common.cuh"

// The denominator |r||e| + r.e cancels when the segment subtends nearly 180 degrees at the
// target (r.e ~ -|r||e|).  Since (|r||e| + r.e)(|r||e| - r.e) = |r x e|^2 = |r x d|^2, it is
// taken as |r x d|^2 / (|r||e| - r.e) when r.e < 0, which subtracts nothing either.
//
// Conditioning guards of the FP32 segment term: a far term is evaluated in FP64 when
//   |r||e| + r.e < angle |r||e|         (the segment subtends more than ~154 degrees at the
//                                        target for angle 0.1: the target is close to a long
//                                        segment, where r x circ keeps only ~1e-6 of its
//                                        digits in FP32 and the term is large),
//   |r x circ|^2 < line |circ|^2 min(|r|^2, |e|^2)   (the target lies near the segment's line),
//   |e|^2 < end max(|r|^2, |circ|^2)    (the target lies near the far end: e = r + circ loses
//                                        digits).
struct Fp32Guards {
  float angle = 0.1f, line = 1e-3f, end = 1e-2f;
};

// FP64 reciprocal and reciprocal square root by Newton's iteration (y <- y + y(1 - x y) and
// y <- y + y(1 - x y^2)/2), each started from the FP32 hardware approximation (relative error
// ~1e-7) and iterated twice: the error squares at every step, so two steps reach the FP64
// rounding level.  Arguments outside the FP32 exponent range take the IEEE operation.
__device__ __forceinline__ double rcp64(double x) {
  const double ax = fabs(x);
  if (!(ax > 1e-30 && ax < 1e30)) return 1.0 / x;
  double y = (double)__fdividef(1.f, (float)x);
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ double rsqrt64(double x) {
  if (!(x > 1e-30 && x < 1e30)) return 1.0 / sqrt(x);
  double y = (double)rsqrtf((float)x);
  double e = fma(-x * y, y, 1.0);
  y = fma(0.5 * y, e, y);
  e = fma(-x * y, y, 1.0);
  return fma(0.5 * y, e, y);
}

// One segment term in FP64 from the cancellation-free form above:
//   gq (r x d)(1/|r| + 1/|e|) / (|r||e| + r.e),  e = r + d, gq = Gamma/(4 pi),
// given rr = |r|^2.  Agrees with the reference's expression (timestep.f90:162-169) to a few
// FP64 roundings; the caller takes the reference's decision whether to skip the term.
__device__ __forceinline__ void term64_stable(const double r[3], const double d[3], double rr, double gq,
                                              double out[3]) {
  const double e[3] = {r[0] + d[0], r[1] + d[1], r[2] + d[2]};
  const double ee = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
  const double re = r[0] * e[0] + r[1] * e[1] + r[2] * e[2];
  const double cr[3] = {r[1] * d[2] - r[2] * d[1], r[2] * d[0] - r[0] * d[2], r[0] * d[1] - r[1] * d[0]};
  const double ia = rsqrt64(rr), ib = rsqrt64(ee);
  const double pp = (rr * ia) * (ee * ib);
  double f;
  if (re >= 0.0) {
    f = gq * (ia + ib) * rcp64(pp + re);
  } else {
    const double cr2 = cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2];
    f = gq * (ia + ib) * (pp - re) * rcp64(cr2);
  }
  out[0] = f * cr[0];
  out[1] = f * cr[1];
  out[2] = f * cr[2];
}

// One node as the mixed walk reads it: 64 bytes, four 16-byte loads.
struct __align__(16) WalkNode {
  float4 a;  // centre (FP32 high part), accept threshold t1^2 rounded to FP32
  float4 b;  // centre (FP32 low part: centre - high part), |circ|^2 in FP32
  float4 c;  // circulation in FP32, the line guard's threshold (Fp32Guards::line x |circ|^2)
  int4 d;    // pcount, first child, next sibling, first member's infront
};

struct MixedNodes {  // per tree node, built after the FP64 node sums
  double4 *C = nullptr;  // cent.xyz, accept threshold t1^2 (dist^2 > t1^2 opens nothing)
  double2 *G = nullptr;  // geo^2, t0^2 for the dist <= geo branch (theta0 > 2/sqrt(3) only)
  WalkNode *W = nullptr;
};

// Kahan-compensated FP32 accumulation of one tile's partial sum into (s, comp).
__device__ __forceinline__ void kahan_add(float &s, float &comp, float v) {
  const float y = v - comp;
  const float t = s + y;
  comp = (t - s) - y;
  s = t;
}
