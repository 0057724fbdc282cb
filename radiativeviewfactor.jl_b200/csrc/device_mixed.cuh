// device_mixed.cuh -- FP32 shadow-ray primitives with certified decisions.
//
// Every FP32 slab or Moller-Trumbore decision comes with a forward error
// bound against the FP64 computation the reference performs (src/GPUBVH.jl:
// 219-269).  A decision is taken in FP32 only when the FP32 value clears its
// threshold by more than the bound; otherwise the lane is marked uncertain and
// its whole ray is traced again in FP64 with the reference's arithmetic.  The
// bounds are deliberately loose (relative terms 2^-16 .. 2^-18 against FP32
// rounding of ~2^-22 for these expressions): a loose bound only costs re-tests.
#pragma once

#include "device_common.cuh"

namespace rvf {

// relative error allowances
constexpr float kRho = 9.5367431640625e-07f;  // 2^-20: direction, 1/direction, segment length
constexpr float kE0 = 1.52587890625e-05f;     // 2^-16: Moller-Trumbore terms
constexpr float kMinDir = 1e-4f;              // smaller direction components go to FP64

struct RayF {
  float o[3];
  float d[3];
  float inv[3];
  float tmax;
  float k0;     // absolute slab-parameter error: 2 delta max|inv|
  float delta;  // absolute position error of origin / node / vertex coordinates
};

enum : int { kMiss = 0, kHit = 1, kUnsure = 2 };

// Approximate reciprocal (one MUFU op, at most 1 ulp = 2^-23 relative error):
// every quantity it feeds has an error allowance of 2^-20 or more.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// FP32 ray from origin xo (absolute, rounded) along r = (rx,ry,rz), |r|^2 = r2.
// Returns false when a direction component is too small for a certified FP32
// traversal (the ray then goes to FP64).
__device__ __forceinline__ bool make_ray_f(const float* xo, float rx, float ry, float rz, float r2, float delta,
                                           RayF& R) {
  float ir = rsqrtf(r2);
  R.o[0] = xo[0]; R.o[1] = xo[1]; R.o[2] = xo[2];
  R.d[0] = rx * ir; R.d[1] = ry * ir; R.d[2] = rz * ir;
  R.tmax = r2 * ir;
  if (fabsf(R.d[0]) < kMinDir || fabsf(R.d[1]) < kMinDir || fabsf(R.d[2]) < kMinDir) return false;
  R.inv[0] = rcp_approx(R.d[0]); R.inv[1] = rcp_approx(R.d[1]); R.inv[2] = rcp_approx(R.d[2]);
  float mi = fmaxf(fmaxf(fabsf(R.inv[0]), fabsf(R.inv[1])), fabsf(R.inv[2]));
  R.delta = delta;
  R.k0 = 2.0f * delta * mi;
  return true;
}

// Slab test with a certified outcome (kHit / kMiss / kUnsure).
//
// The box is hit iff the four parameter intervals X, Y, Z (one per slab) and
// S = [0, t_max] share a point, i.e. (1-D Helly) iff every pair of different
// intervals overlaps: the comparison te <= tx of the reference.  An interval
// never needs a margin against itself -- in particular the two ends of a
// slab of zero thickness (lo == hi, as for the leaves of a flat face) are the
// same number in FP32 and in FP64 -- so when te and tx are within the error
// band the six pairs are checked one by one with margins.
__device__ __forceinline__ int slab_f(const NodeF& nd, const RayF& R) {
  float t1x = (nd.lo[0] - R.o[0]) * R.inv[0], t2x = (nd.hi[0] - R.o[0]) * R.inv[0];
  float t1y = (nd.lo[1] - R.o[1]) * R.inv[1], t2y = (nd.hi[1] - R.o[1]) * R.inv[1];
  float t1z = (nd.lo[2] - R.o[2]) * R.inv[2], t2z = (nd.hi[2] - R.o[2]) * R.inv[2];
  const float lx = fminf(t1x, t2x), hx = fmaxf(t1x, t2x);
  const float ly = fminf(t1y, t2y), hy = fmaxf(t1y, t2y);
  const float lz = fminf(t1z, t2z), hz = fmaxf(t1z, t2z);
  float te = fmaxf(fmaxf(fmaxf(lx, ly), lz), 0.0f);
  float tx = fminf(fminf(fminf(hx, hy), hz), R.tmax);
  float m = R.k0 + 2.0f * kRho * (fabsf(te) + fabsf(tx) + R.tmax);
  if (te + m < tx) return kHit;
  if (te > tx + m) return kMiss;
  // pairwise overlaps of different intervals
  const float lo[4] = {lx, ly, lz, 0.0f}, hi[4] = {hx, hy, hz, R.tmax};
  bool unsure = false;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      if (u == v) continue;
      if (lo[u] > hi[v] + m) return kMiss;
      if (!(lo[u] + m < hi[v])) unsure = true;
    }
  return unsure ? kUnsure : kHit;
}

// Moller-Trumbore with certified outcome; the triangle stores |e1|, |e2|
// (rounded up) in n1, n2.
__device__ __forceinline__ int mt_f(const TriF& t, const RayF& R) {
  const float n1 = __int_as_float(t.pad0), n2 = __int_as_float(t.pad1);
  float hx = fmaf(R.d[1], t.e2[2], -R.d[2] * t.e2[1]);
  float hy = fmaf(R.d[2], t.e2[0], -R.d[0] * t.e2[2]);
  float hz = fmaf(R.d[0], t.e2[1], -R.d[1] * t.e2[0]);
  float a = fmaf(t.e1[0], hx, fmaf(t.e1[1], hy, t.e1[2] * hz));
  const float na = n1 * n2;
  const float Ea = kE0 * na;
  const float aa = fabsf(a);
  if (aa + Ea < 1e-10f) return kMiss;
  if (aa - Ea < 1e-10f) return kUnsure;
  const float f = rcp_approx(a);
  const float ia = fabsf(f);
  float sx = R.o[0] - t.v0[0], sy = R.o[1] - t.v0[1], sz = R.o[2] - t.v0[2];
  const float ns = fabsf(sx) + fabsf(sy) + fabsf(sz) + 2.0f * R.delta;
  const float d2 = 2.0f * R.delta;
  float u = f * fmaf(sx, hx, fmaf(sy, hy, sz * hz));
  float Eu = fmaf(fabsf(u), Ea, (kE0 * ns + d2) * n2) * ia + kE0 * fabsf(u);
  if (u < -Eu || u > 1.0f + Eu) return kMiss;
  float qx = fmaf(sy, t.e1[2], -sz * t.e1[1]);
  float qy = fmaf(sz, t.e1[0], -sx * t.e1[2]);
  float qz = fmaf(sx, t.e1[1], -sy * t.e1[0]);
  float v = f * fmaf(R.d[0], qx, fmaf(R.d[1], qy, R.d[2] * qz));
  float Ev = fmaf(fabsf(v), Ea, (kE0 * ns + 2.0f * d2) * n1) * ia + kE0 * fabsf(v);
  if (v < -Ev || u + v > 1.0f + Eu + Ev + 1e-6f) return kMiss;
  float tt = f * fmaf(t.e2[0], qx, fmaf(t.e2[1], qy, t.e2[2] * qz));
  float Et = fmaf(fabsf(tt), Ea, (kE0 * ns + 2.0f * d2) * na) * ia + kE0 * fabsf(tt);
  const float Etm = Et + 2.0f * kRho * R.tmax;
  if (tt < (float)kTEps - Et || tt > R.tmax + Etm) return kMiss;
  const bool inside = (u > Eu && u < 1.0f - Eu) && (v > Ev && u + v < 1.0f - Eu - Ev - 1e-6f);
  if (inside && tt > (float)kTEps + Et && tt < R.tmax - Etm) return kHit;
  return kUnsure;
}

// Warp-coherent FP32 any-hit traversal (same walk as packet_any_hit) with
// certified decisions.  A lane leaves the walk at its first uncertain
// decision (unsure = true); its ray must then be traced in FP64.
template <typename LeafF>
__device__ __forceinline__ bool packet_any_hit_f(bool alive, const NodeF* __restrict__ nodes, int n_nodes,
                                                 const RayF& R, LeafF leaf, bool& unsure, TravCount& cnt) {
  bool hit = false;
  unsure = false;
  int wake = 0, node = 0;
  if (!__any_sync(kFull, alive)) return false;
  while (node < n_nodes) {
    const NodeF nd = nodes[node];
    const bool live = alive && !hit && !unsure;
    bool act = live && node >= wake;
    unsigned am = __ballot_sync(kFull, act);
    if (am == 0) {
      node = __reduce_min_sync(kFull, live ? wake : n_nodes);
      continue;
    }
    cnt.nodes += act ? 1 : 0;
    int s = act ? slab_f(nd, R) : kMiss;
    if (s == kUnsure) {
      unsure = true;
      ++cnt.unsure_slab;
    }
    bool sh = (s == kHit);
    unsigned hm = __ballot_sync(kFull, sh);
    const int cntp = nd.ab & 15, first = nd.ab >> 4;
    if (cntp > 0) {
      if (hm) {
        for (int k = first; k < first + cntp; ++k) {
          int r = leaf(k, sh && !hit && !unsure);
          if (r == kHit) hit = true;
          else if (r == kUnsure) {
            unsure = true;
            ++cnt.unsure_prim;
          }
        }
      }
      node = nd.miss;
    } else {
      if (hm) {
        if (act && s == kMiss) wake = nd.miss;
        node = node + 1;
      } else {
        node = nd.miss;
      }
    }
    if (!__any_sync(kFull, alive && !hit && !unsure)) break;
  }
  return hit;
}

}  // namespace rvf
