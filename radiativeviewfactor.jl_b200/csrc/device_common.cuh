// device_common.cuh -- device primitives shared by the librvf_b200 kernels.
//
// The library is compiled with --fmad=false: a plain expression is evaluated
// exactly in the order written with IEEE rounding (double '/' and sqrt are
// correctly rounded), which reproduces the reference's Float64 arithmetic bit
// for bit.  Fast paths request fused multiply-adds explicitly with fma().
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rvf_host.h"

namespace rvf {

constexpr double kPiD = 3.141592653589793;        // Float64(pi)
constexpr double kTEps = 9.999999974752427e-07;   // Float64(1f-6), src/GPUBVH.jl:200
constexpr unsigned kFull = 0xffffffffu;


// ---------------------------------------------------------------------------
// reciprocal: hardware seed (rcp.approx.ftz.f64) refined by two Newton-Raphson
// steps r <- r + r(1 - x r) (the classical iteration for 1/x); relative error
// below 1 ulp for normal x.  Used only where the result feeds a sum checked to
// a tolerance, never where a decision must match the reference bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  return r;
}

// ---------------------------------------------------------------------------
// shape functions, src/GPUKernels.jl:51-176 and src/Geometry.jl:247-334,
// written in the reference's evaluation order
// ---------------------------------------------------------------------------
__device__ __forceinline__ int fam_nodes(int f) {
  return f == 0 ? 8 : f == 1 ? 6 : f == 2 ? 4 : f == 3 ? 3 : f == 4 ? 3 : 2;
}
__device__ __forceinline__ bool is_quad_fam(int f) { return f == 0 || f == 2; }
__device__ __forceinline__ bool is_line_fam(int f) { return f == 4 || f == 5; }

__device__ __forceinline__ void shape_surface(int f, double x, double e, double* N, double* dx, double* de) {
  if (f == 0) {
    N[0] = ((0.25 * (1 - x)) * (1 - e)) * (((-x) - e) - 1);
    N[1] = ((0.25 * (1 + x)) * (1 - e)) * ((x - e) - 1);
    N[2] = ((0.25 * (1 + x)) * (1 + e)) * ((x + e) - 1);
    N[3] = ((0.25 * (1 - x)) * (1 + e)) * (((-x) + e) - 1);
    N[4] = (0.5 * (1 - x * x)) * (1 - e);
    N[5] = (0.5 * (1 + x)) * (1 - e * e);
    N[6] = (0.5 * (1 - x * x)) * (1 + e);
    N[7] = (0.5 * (1 - x)) * (1 - e * e);
    dx[0] = (0.25 * (1 - e)) * (2 * x + e);
    dx[1] = (0.25 * (1 - e)) * (2 * x - e);
    dx[2] = (0.25 * (1 + e)) * (2 * x + e);
    dx[3] = (0.25 * (1 + e)) * (2 * x - e);
    dx[4] = (-x) * (1 - e);
    dx[5] = 0.5 * (1 - e * e);
    dx[6] = (-x) * (1 + e);
    dx[7] = (-0.5) * (1 - e * e);
    de[0] = (0.25 * (1 - x)) * (x + 2 * e);
    de[1] = (0.25 * (1 + x)) * ((-x) + 2 * e);
    de[2] = (0.25 * (1 + x)) * (x + 2 * e);
    de[3] = (0.25 * (1 - x)) * ((-x) + 2 * e);
    de[4] = (-0.5) * (1 - x * x);
    de[5] = (-(1 + x)) * e;
    de[6] = 0.5 * (1 - x * x);
    de[7] = (-(1 - x)) * e;
  } else if (f == 1) {
    double L1 = (1 - x) - e, L2 = x, L3 = e;
    N[0] = L1 * (2 * L1 - 1); N[1] = L2 * (2 * L2 - 1); N[2] = L3 * (2 * L3 - 1);
    N[3] = (4 * L1) * L2; N[4] = (4 * L2) * L3; N[5] = (4 * L1) * L3;
    dx[0] = (4 * L1 - 1) * (-1.0); dx[1] = 4 * L2 - 1; dx[2] = 0.0;
    dx[3] = 4 * (L2 * (-1.0) + L1); dx[4] = 4 * L3; dx[5] = (4 * L3) * (-1.0);
    de[0] = (4 * L1 - 1) * (-1.0); de[1] = 0.0; de[2] = 4 * L3 - 1;
    de[3] = (4 * L2) * (-1.0); de[4] = 4 * L2; de[5] = 4 * (L3 * (-1.0) + L1);
  } else if (f == 2) {
    N[0] = (0.25 * (1 - x)) * (1 - e); N[1] = (0.25 * (1 + x)) * (1 - e);
    N[2] = (0.25 * (1 + x)) * (1 + e); N[3] = (0.25 * (1 - x)) * (1 + e);
    dx[0] = (-0.25) * (1 - e); dx[1] = 0.25 * (1 - e); dx[2] = 0.25 * (1 + e); dx[3] = (-0.25) * (1 + e);
    de[0] = (-0.25) * (1 - x); de[1] = (-0.25) * (1 + x); de[2] = 0.25 * (1 + x); de[3] = 0.25 * (1 - x);
  } else {
    N[0] = (1 - x) - e; N[1] = x; N[2] = e;
    dx[0] = -1.0; dx[1] = 1.0; dx[2] = 0.0;
    de[0] = -1.0; de[1] = 0.0; de[2] = 1.0;
  }
}

// x, n = c/|c|, dA = |c| with |c| = sqrt(dot(c,c))  (src/GPUKernels.jl:95-110)
__device__ __forceinline__ void eval_surface(const double* __restrict__ coords, const int32_t* en, int f,
                                             double xi, double eta, double* x, double* n, double* dA) {
  double N[8], dX[8], dE[8];
  shape_surface(f, xi, eta, N, dX, dE);
  int nn = fam_nodes(f);
  double px = 0.0, py = 0.0, pz = 0.0, ax = 0.0, ay = 0.0, az = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
  for (int k = 0; k < nn; ++k) {
    const double* xa = coords + 3 * (int64_t)en[k];
    double cx = xa[0], cy = xa[1], cz = xa[2];
    px = px + N[k] * cx; py = py + N[k] * cy; pz = pz + N[k] * cz;
    ax = ax + dX[k] * cx; ay = ay + dX[k] * cy; az = az + dX[k] * cz;
    bx = bx + dE[k] * cx; by = by + dE[k] * cy; bz = bz + dE[k] * cz;
  }
  double cx = ay * bz - az * by;
  double cy = az * bx - ax * bz;
  double cz = ax * by - ay * bx;
  double d = sqrt((cx * cx + cy * cy) + cz * cz);
  x[0] = px; x[1] = py; x[2] = pz;
  n[0] = cx / d; n[1] = cy / d; n[2] = cz / d;
  *dA = d;
}

// Line3 / Line2: src/Geometry.jl:247-334 (normal = tangent rotated +90 deg in xy)
__device__ __forceinline__ void eval_line(const double* __restrict__ coords, const int32_t* en, int f, double xi,
                                          double* x, double* n, double* dL) {
  double N[3], dN[3];
  int nn;
  if (f == 4) {
    N[0] = ((-0.5) * xi) * (1.0 - xi); N[1] = (0.5 * xi) * (1.0 + xi); N[2] = 1.0 - xi * xi;
    dN[0] = -0.5 + xi; dN[1] = 0.5 + xi; dN[2] = -2.0 * xi;
    nn = 3;
  } else {
    N[0] = 0.5 * (1.0 - xi); N[1] = 0.5 * (1.0 + xi);
    dN[0] = -0.5; dN[1] = 0.5;
    nn = 2;
  }
  double px = 0.0, py = 0.0, pz = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
  for (int k = 0; k < nn; ++k) {
    const double* xa = coords + 3 * (int64_t)en[k];
    px = px + N[k] * xa[0]; py = py + N[k] * xa[1]; pz = pz + N[k] * xa[2];
    tx = tx + dN[k] * xa[0]; ty = ty + dN[k] * xa[1]; tz = tz + dN[k] * xa[2];
  }
  double L = sqrt((tx * tx + ty * ty) + tz * tz);
  double ux = tx / L, uy = ty / L;
  x[0] = px; x[1] = py; x[2] = pz;
  n[0] = -uy; n[1] = ux; n[2] = 0.0;
  *dL = L;
}

// ---------------------------------------------------------------------------
// view-factor kernel
// ---------------------------------------------------------------------------
// Reference formula (src/GPUKernels.jl:204-215 / src/ViewFactorKernel.jl:169-180),
// bit for bit.  dim3: cos*cos/(pi r^2); otherwise cos*cos/(2 r).
template <bool DIM3>
__device__ __forceinline__ double k_reference_inl(double rx, double ry, double rz, double r2, const double* ni,
                                                  const double* nj) {
  double r = sqrt(r2);
  double hx = rx / r, hy = ry / r, hz = rz / r;
  double ci = (ni[0] * hx + ni[1] * hy) + ni[2] * hz;
  double cj = (nj[0] * (-hx) + nj[1] * (-hy)) + nj[2] * (-hz);
  if (ci <= 0.0 || cj <= 0.0) return 0.0;
  return DIM3 ? (ci * cj) / (kPiD * r2) : (ci * cj) / (2.0 * r);
}
// out of line where the caller keeps many registers live across it
template <bool DIM3>
__device__ __noinline__ double k_reference(double rx, double ry, double rz, double r2, const double* ni,
                                           const double* nj) {
  return k_reference_inl<DIM3>(rx, ry, rz, r2, ni, nj);
}

// Fast evaluation with the same K > 0 decision as the reference.
// r = xj - xi and r2 = (rx^2 + ry^2) + rz^2 are formed exactly as the
// reference forms them (so the r2 < 1e-30 cut and the shadow ray match).
// If either |cos| < 1e-5 the sign or the value of the fast form could differ
// from the reference beyond 1e-10 relative, so the reference formula runs.
template <bool DIM3>
__device__ __forceinline__ double k_fast(double rx, double ry, double rz, double r2, const double* ni,
                                         const double* nj) {
  if (r2 < 1e-30) return 0.0;
  double di = fma(ni[0], rx, fma(ni[1], ry, ni[2] * rz));
  double dj = -fma(nj[0], rx, fma(nj[1], ry, nj[2] * rz));
  double thr = 1e-10 * r2;
  if (di * di <= thr || dj * dj <= thr) return k_reference<DIM3>(rx, ry, rz, r2, ni, nj);
  if (di <= 0.0 || dj <= 0.0) return 0.0;
  if (DIM3) return (di * dj) * rcp_nr(kPiD * (r2 * r2));
  return (di * dj) * rcp_nr(2.0 * (r2 * sqrt(r2)));
}

// ---------------------------------------------------------------------------
// shadow rays, FP64, src/GPUBVH.jl:202-285 semantics
// ---------------------------------------------------------------------------
struct RayD {
  double o[3];
  double d[3];
  double inv[3];
  double tmax;
  bool zdir;  // some direction component is exactly zero (NaN-culling possible)
};

// src/GPUKernels.jl:290-300: dir = r * (1/|r|), t_max = |r|
__device__ __forceinline__ bool make_ray(const double* xi, double rx, double ry, double rz, double r2, RayD& R) {
  double rlen = sqrt(r2);
  if (!(rlen > 1e-15)) return false;
  double inv_r = 1.0 / rlen;
  R.o[0] = xi[0]; R.o[1] = xi[1]; R.o[2] = xi[2];
  R.d[0] = rx * inv_r; R.d[1] = ry * inv_r; R.d[2] = rz * inv_r;
  R.inv[0] = 1.0 / R.d[0]; R.inv[1] = 1.0 / R.d[1]; R.inv[2] = 1.0 / R.d[2];
  R.tmax = rlen;
  R.zdir = (R.d[0] == 0.0) | (R.d[1] == 0.0) | (R.d[2] == 0.0);
  return true;
}

// Slab test with Julia's NaN-propagating min/max: identical to fmin/fmax
// except that any NaN slab parameter culls the box.
__device__ __forceinline__ bool slab_d(const NodeD& nd, const RayD& R) {
  double t1x = (nd.lo[0] - R.o[0]) * R.inv[0], t2x = (nd.hi[0] - R.o[0]) * R.inv[0];
  double t1y = (nd.lo[1] - R.o[1]) * R.inv[1], t2y = (nd.hi[1] - R.o[1]) * R.inv[1];
  double t1z = (nd.lo[2] - R.o[2]) * R.inv[2], t2z = (nd.hi[2] - R.o[2]) * R.inv[2];
  double te = fmax(fmax(fmax(fmin(t1x, t2x), fmin(t1y, t2y)), fmin(t1z, t2z)), 0.0);
  double tx = fmin(fmin(fmin(fmax(t1x, t2x), fmax(t1y, t2y)), fmax(t1z, t2z)), R.tmax);
  bool hit = te <= tx;
  if (R.zdir) {
    bool nan = (t1x != t1x) | (t2x != t2x) | (t1y != t1y) | (t2y != t2y) | (t1z != t1z) | (t2z != t2z);
    hit = hit && !nan;
  }
  return hit;
}

// Moller-Trumbore, src/GPUBVH.jl:247-269, on the precomputed v0 / e1 / e2.
__device__ __forceinline__ bool mt_d(const TriD& t, const RayD& R) {
  double hx = R.d[1] * t.e2[2] - R.d[2] * t.e2[1];
  double hy = R.d[2] * t.e2[0] - R.d[0] * t.e2[2];
  double hz = R.d[0] * t.e2[1] - R.d[1] * t.e2[0];
  double a = (t.e1[0] * hx + t.e1[1] * hy) + t.e1[2] * hz;
  if (fabs(a) < 1e-10) return false;
  double f = 1.0 / a;
  double sx = R.o[0] - t.v0[0], sy = R.o[1] - t.v0[1], sz = R.o[2] - t.v0[2];
  double u = f * ((sx * hx + sy * hy) + sz * hz);
  if (u < 0.0 || u > 1.0) return false;
  double qx = sy * t.e1[2] - sz * t.e1[1];
  double qy = sz * t.e1[0] - sx * t.e1[2];
  double qz = sx * t.e1[1] - sy * t.e1[0];
  double v = f * ((R.d[0] * qx + R.d[1] * qy) + R.d[2] * qz);
  if (v < 0.0 || u + v > 1.0) return false;
  double tt = f * ((t.e2[0] * qx + t.e2[1] * qy) + t.e2[2] * qz);
  return tt > kTEps && tt < R.tmax;
}

// 2-D segment blocking test, src/BVH.jl:265-276
__device__ __forceinline__ bool seg_blocks(const SegD& s, const double* xi, const double* xj) {
  const double tol = 1e-8;
  double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
  double ex = s.x1 - s.x0, ey = s.y1 - s.y0;
  double den = dx * ey - dy * ex;
  if (fabs(den) < tol) return false;
  double fx = s.x0 - xi[0], fy = s.y0 - xi[1];
  double sp = (fx * ey - fy * ex) / den;
  double tp = (fx * dy - fy * dx) / den;
  return (tol < sp && sp < 1.0 - tol) && (tol < tp && tp < 1.0 - tol);
}

// ---------------------------------------------------------------------------
// Warp-coherent any-hit traversal of the pre-order BVH.
//
// All 32 lanes walk the same node sequence (node fetches are warp-uniform and
// broadcast); a lane whose slab test fails at node k sleeps until the walk
// reaches miss(k), the first node after k's subtree, so every lane tests
// exactly the nodes its own stackless walk (src/GPUBVH.jl:216-282) would test
// and reaches the same any-hit answer.  The walk descends when any awake lane
// hits, and jumps to the smallest wake-up node when no lane is awake.
// ---------------------------------------------------------------------------
struct TravCount {  // per-thread counts (a thread's share stays far below 2^32)
  uint32_t nodes = 0, prims = 0;
  uint32_t unsure_slab = 0, unsure_prim = 0;  // FP32 traversal: decisions left to FP64
};

template <typename NodeT, typename SlabF, typename LeafF>
__device__ __forceinline__ bool packet_any_hit(bool alive, const NodeT* __restrict__ nodes, int n_nodes, SlabF slab,
                                               LeafF leaf, TravCount& cnt) {
  bool hit = false;
  int wake = 0;
  int node = 0;
  if (!__any_sync(kFull, alive)) return false;
  while (node < n_nodes) {
    const NodeT nd = nodes[node];
    bool act = alive && !hit && node >= wake;
    unsigned am = __ballot_sync(kFull, act);
    if (am == 0) {
      int w = (alive && !hit) ? wake : n_nodes;
      node = __reduce_min_sync(kFull, w);
      continue;
    }
    cnt.nodes += act ? 1 : 0;
    bool sh = act && slab(nd);
    unsigned hm = __ballot_sync(kFull, sh);
    if (nd.b > 0) {
      if (hm) {
        for (int k = nd.a; k < nd.a + nd.b; ++k) {
          bool h = leaf(k, sh && !hit);
          hit = hit || h;
        }
      }
      node = nd.miss;
    } else {
      if (hm) {
        if (act && !sh) wake = nd.miss;
        node = node + 1;
      } else {
        node = nd.miss;
      }
    }
    if (!__any_sync(kFull, alive && !hit)) break;
  }
  return hit;
}

// ---------------------------------------------------------------------------
// bulk copies (cp.async.bulk) with an mbarrier, bounded waits
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared; dst, src 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity; gives up after ~1 s and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 24); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 32) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// linear upper-triangle tile index -> (bi, bj), row-major with bi <= bj
__device__ __forceinline__ void tile_coords(int64_t t, int64_t nT, int64_t& bi, int64_t& bj) {
  double a = 2.0 * nT + 1.0;
  int64_t b = (int64_t)floor((a - sqrt(a * a - 8.0 * (double)t)) * 0.5);
  if (b < 0) b = 0;
  auto off = [nT](int64_t r) { return r * nT - (r * (r - 1)) / 2; };
  while (b + 1 < nT && off(b + 1) <= t) ++b;
  while (b > 0 && off(b) > t) --b;
  bi = b;
  bj = b + (t - off(b));
}

}  // namespace rvf
