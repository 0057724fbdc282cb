// device_lists.cuh -- certified geometric tests of the pair lists and of
// the tile classification: a pair's shadow rays all lie in its capsule (the
// centroid segment grown by R = max(rad_i, rad_j) plus a margin), and a box
// or triangle farther than the capsule's radius (plus the rounding margin of
// the reference's test) is never reached or hit by any of them.
#pragma once

#include "device_trace.cuh"

namespace rvf {

// Separation of the centroid segment (a, b) and the triangle (p0, p1, p2)
// along w, in FP32: true when the gap exceeds rm |w|.  Squares avoid the
// square root (rm > 0).
__device__ __forceinline__ bool axis_separates(const float* a, const float* b, const float4& p0, const float4& p1,
                                               const float4& p2, float wx, float wy, float wz, float rm) {
  const float sa = fmaf(a[0], wx, fmaf(a[1], wy, a[2] * wz)), sb = fmaf(b[0], wx, fmaf(b[1], wy, b[2] * wz));
  const float q0 = fmaf(p0.x, wx, fmaf(p0.y, wy, p0.z * wz));
  const float q1 = fmaf(p1.x, wx, fmaf(p1.y, wy, p1.z * wz));
  const float q2 = fmaf(p2.x, wx, fmaf(p2.y, wy, p2.z * wz));
  const float gap = fmaxf(fminf(q0, fminf(q1, q2)) - fmaxf(sa, sb), fminf(sa, sb) - fmaxf(q0, fmaxf(q1, q2)));
  return gap > 0.0f && gap * gap > rm * rm * fmaf(wx, wx, fmaf(wy, wy, wz * wz));
}

// True when no ray of the pair (segments within R of the centroid segment
// a -> b, direction d) can be a hit of the reference's test of the triangle
// with corners p0, p1, p2 (FP32) and rounding margin p0.w.  em absorbs the
// FP32 rounding of the corners and of this test (a few 2^-24 of the
// coordinates' magnitude, against em = S 2^-16).
__device__ __forceinline__ bool pair_misses_tri(const float* a, const float* b, const float* d, float R, float em,
                                                const float4& p0, const float4& p1, const float4& p2) {
  const float rm = R + p0.w + em;
  const float f1[3] = {p1.x - p0.x, p1.y - p0.y, p1.z - p0.z};
  const float f2[3] = {p2.x - p0.x, p2.y - p0.y, p2.z - p0.z};
  const float f3[3] = {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z};
  // the segment direction crossed with each edge, then the triangle's normal
  if (axis_separates(a, b, p0, p1, p2, d[1] * f1[2] - d[2] * f1[1], d[2] * f1[0] - d[0] * f1[2],
                     d[0] * f1[1] - d[1] * f1[0], rm))
    return true;
  if (axis_separates(a, b, p0, p1, p2, d[1] * f2[2] - d[2] * f2[1], d[2] * f2[0] - d[0] * f2[2],
                     d[0] * f2[1] - d[1] * f2[0], rm))
    return true;
  if (axis_separates(a, b, p0, p1, p2, d[1] * f3[2] - d[2] * f3[1], d[2] * f3[0] - d[0] * f3[2],
                     d[0] * f3[1] - d[1] * f3[0], rm))
    return true;
  return axis_separates(a, b, p0, p1, p2, f1[1] * f2[2] - f1[2] * f2[1], f1[2] * f2[0] - f1[0] * f2[2],
                        f1[0] * f2[1] - f1[1] * f2[0], rm);
}

// The same test over more separating axes: the coordinate axes first (the
// cheapest and, for the long thin triangles the reference's transposed read
// produces, often enough), then the segment direction crossed with each
// edge, the normal, and each coordinate axis crossed with each edge.  Each
// axis is a valid separation on its own (the capsule projects onto w as its
// centroid segment widened by rm |w|), so more axes only drop more.
__device__ __forceinline__ bool pair_misses_tri_full(const float* a, const float* b, const float* d, float R,
                                                     float em, const float4& p0, const float4& p1,
                                                     const float4& p2) {
  const float rm = R + p0.w + em;
  {
    const float ax[3] = {a[0], a[1], a[2]}, bx[3] = {b[0], b[1], b[2]};
    const float q0[3] = {p0.x, p0.y, p0.z}, q1[3] = {p1.x, p1.y, p1.z}, q2[3] = {p2.x, p2.y, p2.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float tlo = fminf(q0[k], fminf(q1[k], q2[k])), thi = fmaxf(q0[k], fmaxf(q1[k], q2[k]));
      const float slo = fminf(ax[k], bx[k]), shi = fmaxf(ax[k], bx[k]);
      if (tlo - shi > rm || slo - thi > rm) return true;
    }
  }
  if (pair_misses_tri(a, b, d, R, em, p0, p1, p2)) return true;
  const float f[3][3] = {{p1.x - p0.x, p1.y - p0.y, p1.z - p0.z},
                         {p2.x - p0.x, p2.y - p0.y, p2.z - p0.z},
                         {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z}};
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float w[3] = {0.f, 0.f, 0.f};  // e_k x f_m
      w[(k + 1) % 3] = -f[m][(k + 2) % 3];
      w[(k + 2) % 3] = f[m][(k + 1) % 3];
      if (axis_separates(a, b, p0, p1, p2, w[0], w[1], w[2], rm)) return true;
    }
  return false;
}

// The pair's capsule for the list walk, in FP32: the centroid segment's
// start A and direction reciprocals (from FP64, rounded once), and the radius
// grown by em.  A box test in FP32 (capsule_misses_box) then only reports a
// miss when the FP64 test with the ungrown radius would: every rounding of
// the test (the nodes' and A's FP32 copies, the subtraction, 1/d) moves a
// slab parameter by a few 2^-24 S |1/d|, the growth by em = 2^-16 S moves it
// by em |1/d|.  Components of d that are exactly zero use the containment
// test, as pair_misses_box does.
struct CapsuleF {
  float A[3], inv[3];
  bool zero[3];
  float R;
};

__device__ __forceinline__ bool capsule_misses_box(const CapsuleF& c, const NodeF& nd) {
  float te = 0.0f, tx = 1.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float lo = nd.lo[k] - c.R, hi = nd.hi[k] + c.R;
    if (c.zero[k]) {
      if (c.A[k] < lo || c.A[k] > hi) return true;
      continue;
    }
    const float t1 = (lo - c.A[k]) * c.inv[k], t2 = (hi - c.A[k]) * c.inv[k];
    te = fmaxf(te, fminf(t1, t2));
    tx = fminf(tx, fmaxf(t1, t2));
  }
  return te > tx;
}

}  // namespace rvf
