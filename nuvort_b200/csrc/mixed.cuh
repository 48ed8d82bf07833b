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
// the bracket.  The near field (leaves or segments closer than near_radius) is evaluated in
// FP64 with the reference's own expression, so those terms equal the plain path's.
#pragma once

#include "common.cuh"

// Conditioning guards of the FP32 segment term: a far term is evaluated in FP64 when
//   |r||e| + r.e < angle |r||e|         (the segment subtends nearly 180 degrees at the target),
//   |r x circ|^2 < line |circ|^2 min(|r|^2, |e|^2)   (the target lies near the segment's line),
//   |e|^2 < end max(|r|^2, |circ|^2)    (the target lies near the far end),
// where FP32 cancellation would cost digits.
struct Fp32Guards {
  float angle = 0.1f, line = 1e-3f, end = 1e-2f;
};

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
