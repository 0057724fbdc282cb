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

}  // namespace

// Area rule: one thread per caller-order element.
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
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int64_t i = bi * kTile + warp + 8 * rr;
      if (i >= N) continue;  // warp-uniform
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
                cast, a.nodes, a.n_nodes, [&](const NodeD& nd) { return slab_d(nd, R); },
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
            const bool blocked = packet_any_hit(
                cast, a.nodes, a.n_nodes,
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
