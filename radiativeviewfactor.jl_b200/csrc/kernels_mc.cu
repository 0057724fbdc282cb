// kernels_mc.cu -- stratified Monte Carlo pair kernel (src/GPUMCKernels.jl:146-281).
//
// Every pair keeps the reference's own random stream: splitmix64 of
// seed + ((i-1) N + j) * golden (1-based caller indices, i < j), then
// xorshift64 draws u = (s >> 11) / (2^53 - 1), four per sample (u1,u2 for
// element i, u3,u4 for element j), s = floor(sqrt(n)) strata per axis with the
// same stratum on both elements, uniform remainder samples.  Geometry, kernel
// and rays use the reference's FP64 arithmetic bit for bit, and K_sum is
// accumulated in sample order, so raw values equal the reference's exactly.
//
// Areas follow a fixed rule where the reference races (src/GPUMCKernels.jl:
// 258-259): A_i is the estimate of pair (i, i+1) in the i-role, A_N that of
// pair (N-1, N) in the j-role.
//
// Curve meshes (the reference GPU path rejects them): element i is sampled at
// xi = 2*((si+u1)/s) - 1, element j at xi = 2*((sj+u3)/s) - 1 (u2, u4 drawn and
// unused), remainder samples at 2*u1-1 and 2*u3-1, reference measure 2,
// kernel cos*cos/(2r), occlusion by the 2-D segment test.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "kernels.h"

namespace rvf {

namespace {

__device__ __forceinline__ uint64_t init_rng(uint64_t seed, uint64_t tid) {  // src/GPUMCKernels.jl:44-50
  uint64_t z = seed + tid * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double xorshift64(uint64_t& s) {  // src/GPUMCKernels.jl:37-42
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return (double)(s >> 11) / (double)0x001FFFFFFFFFFFFFULL;
}

__device__ __forceinline__ double ref_measure(int f) { return is_quad_fam(f) ? 4.0 : (is_line_fam(f) ? 2.0 : 0.5); }

// sample of one element at (u, v) in [0,1]^2 (src/GPUMCKernels.jl:266-281)
// or, for curves, at reference coordinate u (already mapped to [-1,1]).
// A curve mesh holds line elements only, a surface mesh surface elements
// only: each kernel compiles its own families.
// Surfaces: out of line, so that the six families' geometry does not
// hold the pair kernel's registers.
__device__ __noinline__ void mc_surface(const double* coords, const int32_t* en, int f, double u, double v, double* x,
                                        double* n, double* dA) {
  if (is_quad_fam(f)) {
    eval_surface(coords, en, f, 2.0 * u - 1.0, 2.0 * v - 1.0, x, n, dA);
  } else {
    double xi = u, eta = v;
    if (xi + eta > 1.0) {
      xi = 1.0 - xi;
      eta = 1.0 - eta;
    }
    eval_surface(coords, en, f, xi, eta, x, n, dA);
  }
}

template <bool DIM3>
__device__ __forceinline__ void mc_point(const McArgs& a, const int32_t* en, int f, double u, double v, double* x,
                                         double* n, double* dA) {
  if (!DIM3) {
    eval_line(a.coords, en, f, u, x, n, dA);
  } else {
    mc_surface(a.coords, en, f, u, v, x, n, dA);
  }
}

// sample k of a pair's stream: the two reference coordinates
__device__ __forceinline__ void mc_coords(bool dim3, int k, int s, uint64_t& st, double* ci, double* cj) {
  const double u1 = xorshift64(st), u2 = xorshift64(st), u3 = xorshift64(st), u4 = xorshift64(st);
  if (k < s * s) {
    const int si = k / s, sj = k - si * s;
    if (dim3) {
      ci[0] = (si + u1) / s; ci[1] = (sj + u2) / s;
      cj[0] = (si + u3) / s; cj[1] = (sj + u4) / s;
    } else {
      ci[0] = 2.0 * ((si + u1) / s) - 1.0; ci[1] = 0.0;
      cj[0] = 2.0 * ((sj + u3) / s) - 1.0; cj[1] = 0.0;
    }
  } else if (dim3) {
    ci[0] = u1; ci[1] = u2; cj[0] = u3; cj[1] = u4;
  } else {
    ci[0] = 2.0 * u1 - 1.0; ci[1] = 0.0; cj[0] = 2.0 * u3 - 1.0; cj[1] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Curves with occlusion: per-pair candidate segments.
//
// The reference walks the whole segment tree for every sample ray, testing a
// node when the ray's bounding box overlaps it (src/BVH.jl:285-322).  A
// segment blocks a ray only if the computed test puts their intersection
// inside both, which (rounding included) needs the segment within
// cand_margin of the ray; and every ray of pair (i, j) lies within
// R = max(r_i, r_j) of the segment between the elements' centres (each
// element's points lie within r of its centre).  So one walk per pair with
// that capsule finds every segment that can block any of the pair's rays;
// each sample then tests only these, each behind the overlap test of its own
// leaf (the walk's test at that leaf: the leaf box lies inside every
// ancestor's, so the test passing there means the reference's walk reaches
// it), with the reference's own segment test.  Decisions are identical to
// the full walk's.  Pairs with more than kMcCand candidates walk the tree
// for every sample as before.
// ---------------------------------------------------------------------------
constexpr int kMcCand = 24;

// Centre and radius of a Line3 / Line2 element: the quadratic curve lies in
// the triangle of its end nodes and its Bezier middle control point
// 2 x_mid - (x_a + x_b) / 2; a Line2 between its ends.
__device__ __forceinline__ void line_bounds(const double* coords, const int32_t* en, int f, double* c, double& r) {
  const double* a = coords + 3 * (int64_t)en[0];
  const double* b = coords + 3 * (int64_t)en[1];
  double p[3][2];
  int n = 2;
  p[0][0] = a[0]; p[0][1] = a[1];
  p[1][0] = b[0]; p[1][1] = b[1];
  if (f == 4) {
    const double* m = coords + 3 * (int64_t)en[2];
    p[2][0] = 2.0 * m[0] - 0.5 * (a[0] + b[0]);
    p[2][1] = 2.0 * m[1] - 0.5 * (a[1] + b[1]);
    n = 3;
  }
  c[0] = c[1] = 0.0;
  for (int k = 0; k < n; ++k) {
    c[0] += p[k][0] / n;
    c[1] += p[k][1] / n;
  }
  r = 0.0;
  for (int k = 0; k < n; ++k) r = fmax(r, hypot(p[k][0] - c[0], p[k][1] - c[1]));
  r *= 1.0 + 1e-12;
}

// True when the box, grown by R, certainly misses the segment a -> b (x, y).
__device__ __forceinline__ bool capsule2_misses_box(const double* a, const double* b, double R, const NodeD& nd) {
  double te = 0.0, tx = 1.0;
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const double lo = nd.lo[c] - R, hi = nd.hi[c] + R;
    const double d = b[c] - a[c];
    if (d == 0.0) {
      if (a[c] < lo || a[c] > hi) return true;
      continue;
    }
    const double inv = 1.0 / d;
    const double t1 = (lo - a[c]) * inv, t2 = (hi - a[c]) * inv;
    te = fmax(te, fmin(t1, t2));
    tx = fmin(tx, fmax(t1, t2));
  }
  return te > tx;
}

__device__ __forceinline__ double point_seg_dist2(double px, double py, double ax, double ay, double bx, double by) {
  const double ex = bx - ax, ey = by - ay;
  const double L2 = ex * ex + ey * ey;
  double t = L2 > 0.0 ? ((px - ax) * ex + (py - ay) * ey) / L2 : 0.0;
  t = fmin(1.0, fmax(0.0, t));
  const double dx = ax + t * ex - px, dy = ay + t * ey - py;
  return dx * dx + dy * dy;
}

// Distance between the segments a-b and c-d in the plane (0 when they cross).
__device__ __forceinline__ double seg_seg_dist(const double* a, const double* b, const double* c, const double* d) {
  const double o1 = (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
  const double o2 = (b[0] - a[0]) * (d[1] - a[1]) - (b[1] - a[1]) * (d[0] - a[0]);
  const double o3 = (d[0] - c[0]) * (a[1] - c[1]) - (d[1] - c[1]) * (a[0] - c[0]);
  const double o4 = (d[0] - c[0]) * (b[1] - c[1]) - (d[1] - c[1]) * (b[0] - c[0]);
  if (((o1 <= 0.0 && o2 >= 0.0) || (o1 >= 0.0 && o2 <= 0.0)) && ((o3 <= 0.0 && o4 >= 0.0) || (o3 >= 0.0 && o4 <= 0.0)))
    return 0.0;
  double m = point_seg_dist2(a[0], a[1], c[0], c[1], d[0], d[1]);
  m = fmin(m, point_seg_dist2(b[0], b[1], c[0], c[1], d[0], d[1]));
  m = fmin(m, point_seg_dist2(c[0], c[1], a[0], a[1], b[0], b[1]));
  m = fmin(m, point_seg_dist2(d[0], d[1], a[0], a[1], b[0], b[1]));
  return sqrt(m);
}

// The pair's candidate segments (index and leaf), or -1 when there are more
// than kMcCand (then every sample walks the tree).
__device__ int mc_candidates(const McArgs& a, const double* ca, const double* cb, double R, int32_t gx, int32_t gy,
                             int* cand_seg, int* cand_leaf, TravCount& tc) {
  const double Rm = R + a.cand_margin;
  int n = 0, node = 0;
  while (node < a.n_nodes) {
    const NodeD nd = a.nodes[node];
    ++tc.nodes;
    if (capsule2_misses_box(ca, cb, Rm, nd)) {
      node = nd.miss;
      continue;
    }
    if (nd.b == 0) {
      node = node + 1;
      continue;
    }
    for (int k = nd.a; k < nd.a + nd.b; ++k) {
      const SegD sg = a.segs[k];
      if (sg.group == gx || sg.group == gy) continue;
      const double s0[2] = {sg.x0, sg.y0}, s1[2] = {sg.x1, sg.y1};
      if (seg_seg_dist(ca, cb, s0, s1) > Rm) continue;
      if (n == kMcCand) return -1;
      cand_seg[n] = k;
      cand_leaf[n] = node;
      ++n;
    }
    node = nd.miss;
  }
  return n;
}

}  // namespace

// Area rule: one thread per caller-order element.
// A point of a surface element: with each mid-side node written as its
// edge's midpoint plus a deviation, x_m = (x_a + x_b) / 2 + delta_m, the
// quadratic families reproduce their linear / bilinear interpolant, so
//   x(xi) = sum_c L_c(xi) x_c + sum_m N_m(xi) delta_m
// with L_c >= 0 summing to 1 (the corners' linear or bilinear functions) and
// N_m >= 0 the mid-side functions, whose sum peaks at 2 (Quad8, at the
// centre) and 4/3 (Tri6, at the centroid).  Hence |x - c| <= max_c |x_c - c|
// + (2 or 4/3) max_m |delta_m| for the corners' centroid c.  Node order as
// shape_surface: Quad8 mid-sides 4..7 on edges 0-1, 1-2, 2-3, 3-0; Tri6 3..5
// on edges 0-1, 1-2, 0-2.  The radius is rounded up by a relative 1e-9: a
// Monte Carlo sample point, evaluated in FP64 from the same nodes, lies
// inside it.
__global__ void k_mc_bounds(McBoundsArgs a) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.N) return;
  const int f = a.fam[e];
  const int nc = (f == 0 || f == 2) ? 4 : 3;
  const int32_t* en = a.enodes + 8 * e;
  auto X = [&](int k) { return a.coords + 3 * (int64_t)en[k]; };
  double c[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < nc; ++k)
    for (int d = 0; d < 3; ++d) c[d] += X(k)[d];
  for (int d = 0; d < 3; ++d) c[d] /= nc;
  double r2 = 0.0;
  for (int k = 0; k < nc; ++k) {
    const double* x = X(k);
    const double dx = x[0] - c[0], dy = x[1] - c[1], dz = x[2] - c[2];
    r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
  }
  double dev2 = 0.0, lam = 0.0;
  if (f == 0 || f == 1) {
    static constexpr int q8[4][3] = {{4, 0, 1}, {5, 1, 2}, {6, 2, 3}, {7, 3, 0}};
    static constexpr int t6[3][3] = {{3, 0, 1}, {4, 1, 2}, {5, 0, 2}};
    const int nm = f == 0 ? 4 : 3;
    lam = f == 0 ? 2.0 : 4.0 / 3.0;
    for (int m = 0; m < nm; ++m) {
      const int* mb = f == 0 ? q8[m] : t6[m];
      const double *xm = X(mb[0]), *xa = X(mb[1]), *xb = X(mb[2]);
      double q = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double dd = xm[d] - 0.5 * (xa[d] + xb[d]);
        q += dd * dd;
      }
      dev2 = fmax(dev2, q);
    }
  }
  for (int d = 0; d < 3; ++d) a.cen[3 * e + d] = c[d];
  a.rad[e] = (sqrt(r2) + lam * sqrt(dev2)) * (1.0 + 1e-9);
}

__global__ void k_mc_area(McArgs a) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t N = a.N;
  if (e >= N) return;
  if (N < 2) {
    a.area_orig[e] = 0.0;
    return;
  }
  const bool first = e + 1 < N;
  const int64_t lo = first ? e : e - 1, hi = first ? e + 1 : e;
  uint64_t st = init_rng(a.seed, (uint64_t)(lo * N + hi + 1));
  const int64_t ie = a.inv[e];
  const int f = a.fam[ie];
  const int32_t* en = a.enodes + 8 * ie;
  const int s = (int)floor(sqrt((double)a.n_samples));
  double A = 0.0;
  for (int k = 0; k < a.n_samples; ++k) {
    double ci[2], cj[2];
    mc_coords(a.dim3, k, s, st, ci, cj);
    const double* c = first ? ci : cj;
    double x[3], n[3], dA;
    if (a.dim3) mc_point<true>(a, en, f, c[0], c[1], x, n, &dA);
    else mc_point<false>(a, en, f, c[0], c[1], x, n, &dA);
    A += dA;
  }
  a.area_orig[e] = (A * ref_measure(f)) / (double)a.n_samples;
}

#ifndef RVF_MC2D_MIN_BLOCKS
#define RVF_MC2D_MIN_BLOCKS 3  // curves: resident blocks of 256 per SM the kernel is compiled for
#endif
template <bool DIM3, bool OCC>
__global__ void __launch_bounds__(256, DIM3 ? 2 : RVF_MC2D_MIN_BLOCKS) k_pairs_mc(McArgs a) {
  __shared__ int64_t s_tile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t N = a.N;
  const int s = (int)floor(sqrt((double)a.n_samples));
  uint64_t n_rays = 0, n_pp = 0;
  TravCount tc;
  for (;;) {
    if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(a.tile_counter, 1ull);
    __syncthreads();
    const int64_t tl = s_tile;
    __syncthreads();
    if (tl >= a.tile_count) break;
    const int64_t t = a.tile0 + tl;
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const int64_t j = bj * kTile + lane;
    const int64_t oj = (j < N) ? (int64_t)a.orig[j] : 0;
    // surfaces: the tile's class; a pair outside its row's mask has no
    // sample ray that can be blocked (its rays skip the traversal)
    const uint8_t tcl = (DIM3 && OCC && a.tcls) ? a.tcls[t] : (uint8_t)kClsSlow;
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int64_t i = bi * kTile + warp + 8 * rr;
      if (i >= N) continue;  // warp-uniform
      const bool may_block = !(DIM3 && OCC && a.tcls) ||
                             ((tcl & kClsSlow) && ((a.tmask[t * kTile + warp + 8 * rr] >> lane) & 1u));
      const bool valid = (j < N) && (i < j);
      const int64_t oi = a.orig[i];
      const bool sw = valid && oi > oj;
      // the reference's pair (lo, hi): lo samples with u1,u2 and casts the ray
      const int64_t e_lo = sw ? j : i, e_hi = sw ? i : j;
      const int64_t o_lo = sw ? oj : oi, o_hi = sw ? oi : oj;
      const int f_lo = valid ? a.fam[e_lo] : 0, f_hi = valid ? a.fam[e_hi] : 0;
      const int32_t* en_lo = a.enodes + 8 * (valid ? e_lo : i);
      const int32_t* en_hi = a.enodes + 8 * (valid ? e_hi : i);
      const int32_t g_lo = valid ? a.group[e_lo] : 0, g_hi = valid ? a.group[e_hi] : 0;
      const int32_t gx = a.exclude ? g_lo : 0, gy = a.exclude ? g_hi : 0;
      uint64_t st = init_rng(a.seed, (uint64_t)(o_lo * N + o_hi + 1));
      uint8_t* logp = (a.ray_log && valid) ? a.ray_log + ((uint64_t)o_lo * N + o_hi) * a.n_samples : nullptr;
      // curves with occlusion: the pair's candidate segments (one walk per pair)
      int cand_seg[(!DIM3 && OCC) ? kMcCand : 1], cand_leaf[(!DIM3 && OCC) ? kMcCand : 1];
      int ncand = -1;
      if (!DIM3 && OCC && valid) {
        double c_lo[2], c_hi[2], r_lo, r_hi;
        line_bounds(a.coords, en_lo, f_lo, c_lo, r_lo);
        line_bounds(a.coords, en_hi, f_hi, c_hi, r_hi);
        ncand = mc_candidates(a, c_lo, c_hi, fmax(r_lo, r_hi), gx, gy, cand_seg, cand_leaf, tc);
      }
      double Ks = 0.0;
      for (int k = 0; k < a.n_samples; ++k) {
        double ci[2], cj[2];
        mc_coords(DIM3, k, s, st, ci, cj);
        double xi[3], ni[3], dAi, xj[3], nj[3], dAj;
        mc_point<DIM3>(a, en_lo, f_lo, ci[0], ci[1], xi, ni, &dAi);
        mc_point<DIM3>(a, en_hi, f_hi, cj[0], cj[1], xj, nj, &dAj);
        const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
        const double r2 = (rx * rx + ry * ry) + rz * rz;
        double K = 0.0;
        if (valid && !(r2 < 1e-30)) K = k_reference<DIM3>(rx, ry, rz, r2, ni, nj);
        n_pp += valid ? 1 : 0;
        if (OCC) {
          uint8_t lg = 0;
          if (DIM3) {
            RayD R;
            const bool cast = (K > 0.0) && make_ray(xi, rx, ry, rz, r2, R);
            n_rays += cast ? 1 : 0;
            const bool blocked = packet_any_hit(
                cast && may_block, a.nodes, a.n_nodes, [&](const NodeD& nd) { return slab_d(nd, R); },
                [&](int kk, bool test) {
                  const TriD tr = a.tris[kk];
                  if (!test || tr.group == gx || tr.group == gy) return false;
                  ++tc.prims;
                  return mt_d(tr, R);
                },
                tc);
            if (cast) lg = blocked ? 2 : 1;
            if (blocked) K = 0.0;
          } else {
            const bool cast = K > 0.0;
            n_rays += cast ? 1 : 0;
            const double rxlo = fmin(xi[0], xj[0]), rxhi = fmax(xi[0], xj[0]);
            const double rylo = fmin(xi[1], xj[1]), ryhi = fmax(xi[1], xj[1]);
            bool blocked = false;
            if (cast && ncand >= 0) {
              for (int c = 0; c < ncand && !blocked; ++c) {
                const NodeD nd = a.nodes[cand_leaf[c]];
                ++tc.nodes;
                if (nd.lo[0] > rxhi || nd.hi[0] < rxlo || nd.lo[1] > ryhi || nd.hi[1] < rylo) continue;
                ++tc.prims;
                blocked = seg_blocks(a.segs[cand_seg[c]], xi, xj);
              }
            }
            const bool walk = cast && ncand < 0;
            if (__any_sync(kFull, walk)) {
              const bool bw = packet_any_hit(
                walk, a.nodes, a.n_nodes,
                [&](const NodeD& nd) {
                  return !(nd.lo[0] > rxhi || nd.hi[0] < rxlo || nd.lo[1] > ryhi || nd.hi[1] < rylo);
                },
                [&](int kk, bool test) {
                  const SegD sg = a.segs[kk];
                  if (!test || sg.group == gx || sg.group == gy) return false;
                  ++tc.prims;
                  return seg_blocks(sg, xi, xj);
                },
                tc);
              if (walk) blocked = bw;
            }
            if (cast) lg = blocked ? 2 : 1;
            if (blocked) K = 0.0;
          }
          if (logp) logp[k] = lg;
        }
        Ks += (K * dAi) * dAj;
      }
      if (valid) {
        const double raw = ((Ks * ref_measure(f_lo)) * ref_measure(f_hi)) / (double)a.n_samples;
        a.F[oi + oj * N] = raw / a.area_orig[oi];
        a.F[oj + oi * N] = raw / a.area_orig[oj];
      } else if (j == i) {
        a.F[oi + oi * N] = 0.0 / a.area_orig[oi];
      }
    }
  }
  n_rays = warp_sum_u64(n_rays);
  n_pp = warp_sum_u64(n_pp);
  const uint64_t s_nodes = warp_sum_u64(tc.nodes), s_prims = warp_sum_u64(tc.prims);
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, n_pp);
    atomicAdd(a.counters + 1, n_rays);
    atomicAdd(a.counters + 2, s_nodes);
    atomicAdd(a.counters + 3, s_prims);
  }
}

template <bool D3, bool O>
static cudaError_t launch_mc_t(const McArgs& a, int sm_count, cudaStream_t st) {
  // persistent blocks: as many as are resident at once
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs_mc<D3, O>, 256, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  int64_t grid = (int64_t)sm_count * per_sm;
  if (grid > a.tile_count) grid = a.tile_count;
  k_pairs_mc<D3, O><<<(unsigned)grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

int mc_resident_blocks(const McArgs& a, int sm_count) {
  const bool occ = a.n_nodes > 0;
  int per_sm = 1;
  const void* fn = a.dim3 ? (occ ? (const void*)k_pairs_mc<true, true> : (const void*)k_pairs_mc<true, false>)
                          : (occ ? (const void*)k_pairs_mc<false, true> : (const void*)k_pairs_mc<false, false>);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
  return sm_count * per_sm;
}

cudaError_t launch_mc_bounds(const McBoundsArgs& a, cudaStream_t st) {
  if (a.N <= 0) return cudaSuccess;
  k_mc_bounds<<<(unsigned)((a.N + 127) / 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mc(const McArgs& a, int sm_count, cudaStream_t st) {
  if (a.N == 0) return cudaSuccess;
  if (a.area_pass) {
    k_mc_area<<<(unsigned)((a.N + 127) / 128), 128, 0, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (a.tile_count <= 0) return cudaSuccess;
  const bool occ = a.n_nodes > 0;
  if (a.dim3) return occ ? launch_mc_t<true, true>(a, sm_count, st) : launch_mc_t<true, false>(a, sm_count, st);
  return occ ? launch_mc_t<false, true>(a, sm_count, st) : launch_mc_t<false, false>(a, sm_count, st);
}

}  // namespace rvf
