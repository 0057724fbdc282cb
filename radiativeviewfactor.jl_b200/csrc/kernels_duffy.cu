// kernels_duffy.cu -- Sauter-Schwab / Duffy integrals for Quad8 pairs that
// share a vertex or an edge (src/DuffyKernel.jl:95-487), on the device.
//
// One block per singular pair.  The block's threads cover the 8*nq^4
// (vertex) or 5*nq^4 (edge) points of the transformed 4-D domain; each point
// evaluates both elements (_eval_quad, src/DuffyKernel.jl:134-139), the view
// factor kernel and, with obstruction, the shadow ray of the GPU path; the
// terms are reduced in a fixed tree order (deterministic).  The result
// overwrites F[i,j] and F[j,i] written by the pair kernel, so it must run on
// the same stream after it.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "kernels.h"

namespace rvf {

namespace {

__device__ __constant__ double kCornerUV[4][2] = {{0.0, 0.0}, {1.0, 0.0}, {1.0, 1.0}, {0.0, 1.0}};

// src/DuffyKernel.jl:288-314
__device__ __forceinline__ void vertex_map(int region, double r, double a, double b, double c, double u0i, double v0i,
                                           double u0j, double v0j, double* U) {
  double du, dv, ds, dt;
  switch (region) {
    case 1: du = r; dv = r * a; ds = r * b; dt = (r * b) * c; break;
    case 2: du = r; dv = r * a; ds = (r * b) * c; dt = r * b; break;
    case 3: du = r * a; dv = r; ds = r * b; dt = (r * b) * c; break;
    case 4: du = r * a; dv = r; ds = (r * b) * c; dt = r * b; break;
    case 5: du = r * b; dv = (r * b) * c; ds = r; dt = r * a; break;
    case 6: du = (r * b) * c; dv = r * b; ds = r; dt = r * a; break;
    case 7: du = r * b; dv = (r * b) * c; ds = r * a; dt = r; break;
    default: du = (r * b) * c; dv = r * b; ds = r * a; dt = r; break;
  }
  U[0] = u0i + (u0i == 0.0 ? du : -du);
  U[1] = v0i + (v0i == 0.0 ? dv : -dv);
  U[2] = u0j + (u0j == 0.0 ? ds : -ds);
  U[3] = v0j + (v0j == 0.0 ? dt : -dt);
}

// src/DuffyKernel.jl:375-408 (region 4 in its final, overriding form)
__device__ __forceinline__ void edge_map(int region, double r, double a, double b, double c, double* U) {
  switch (region) {
    case 1: {
      double A = r * (1 - a * (1 - c));
      U[0] = A;
      U[1] = ((r * a) * b) * c;
      U[2] = (A - ((r * a) * (1 - b)) * c) + ((r * a) * b) * c;
      U[3] = ((r * a) * (1 - b)) * c;
      break;
    }
    case 2: {
      double A = r * (1 - (a * b) * c);
      U[0] = A;
      U[1] = ((r * a) * c) * (1 - b);
      U[2] = (A + ((r * a) * b) * c) - (r * a) * c;
      U[3] = ((r * a) * b) * c;
      break;
    }
    case 3: {
      double A = r * (1 - a * b);
      U[0] = A;
      U[1] = ((r * a) * b) * c;
      U[2] = A - ((r * a) * b) * (1 - c);
      U[3] = ((r * a) * b) * (1 - c);
      break;
    }
    case 4:
      U[0] = r * (b * c + a * (1 - b * c));
      U[1] = ((r * (1 - a)) * b) * c;
      U[2] = (r * b) * c;
      U[3] = ((r * (1 - a)) * b) * c;
      break;
    default:
      U[0] = (r * a) * c;
      U[1] = ((r * (1 - a)) * b) * c;
      U[2] = (((r * a) * c) * (1 - b)) + (((r * a) * b) * c);
      U[3] = ((r * (1 - a)) * b) * c;
      break;
  }
}

// src/DuffyKernel.jl:423-429
__device__ __forceinline__ void rotate_to_edge(double u, double v, int e, double* ou, double* ov) {
  switch (e) {
    case 2: *ou = 1.0 - v; *ov = u; return;
    case 3: *ou = 1.0 - u; *ov = 1.0 - v; return;
    case 4: *ou = v; *ov = 1.0 - u; return;
    default: *ou = u; *ov = v; return;
  }
}

}  // namespace

__global__ void __launch_bounds__(256, 2) k_duffy(DuffyArgs a) {
  const int64_t pi = blockIdx.x;
  const DuffyPair P = a.pairs[pi];
  const int nq = a.nq;
  const int nq4 = nq * nq * nq * nq;
  const int nreg = P.stype == 1 ? 8 : 5;
  const int total = nreg * nq4;
  const int32_t* eni = a.enodes + 8 * (int64_t)P.ii;  // node table is in internal order
  const int32_t* enj = a.enodes + 8 * (int64_t)P.jj;
  const double u0i = kCornerUV[P.ci0 - 1][0], v0i = kCornerUV[P.ci0 - 1][1];
  const double u0j = kCornerUV[P.cj0 - 1][0], v0j = kCornerUV[P.cj0 - 1][1];
  double part = 0.0;
  uint64_t rays = 0;
  TravCount tc;
  // iterate in whole warps so the packet traversal sees converged lanes
  for (int base = 0; base < total; base += blockDim.x) {
    const int k = base + threadIdx.x;
    double term = 0.0;
    bool cast = false;
    RayD R;
    if (k < total) {
      int t = k;
      const int i3 = t % nq; t /= nq;
      const int i2 = t % nq; t /= nq;
      const int i1 = t % nq; t /= nq;
      const int ir = t % nq; t /= nq;
      const int region = t + 1;
      const double r = a.p01[ir], wr = a.w01[ir];
      const double aa = a.p01[i1], wa = a.w01[i1];
      const double bb = a.p01[i2], wb = a.w01[i2];
      const double cc = a.p01[i3], wc = a.w01[i3];
      double U[4];
      if (P.stype == 1) {
        vertex_map(region, r, aa, bb, cc, u0i, v0i, u0j, v0j, U);
      } else {
        double E[4];
        edge_map(region, r, aa, bb, cc, E);
        rotate_to_edge(E[0], E[1], P.edge_i, &U[0], &U[1]);
        rotate_to_edge(E[2], E[3], P.edge_j, &U[2], &U[3]);
      }
      const bool inside = !(U[0] < 0 || U[0] > 1 || U[1] < 0 || U[1] > 1 || U[2] < 0 || U[2] > 1 || U[3] < 0 ||
                            U[3] > 1);
      if (inside) {
        double xi[3], ni[3], dAi, xj[3], nj[3], dAj;
        eval_surface(a.coords, eni, 0, 2 * U[0] - 1.0, 2 * U[1] - 1.0, xi, ni, &dAi);
        eval_surface(a.coords, enj, 0, 2 * U[2] - 1.0, 2 * U[3] - 1.0, xj, nj, &dAj);
        dAi = dAi * 4.0;
        dAj = dAj * 4.0;
        const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
        const double r2 = (rx * rx + ry * ry) + rz * rz;
        const double K = k_fast<true>(rx, ry, rz, r2, ni, nj);
        if (K != 0.0) {
          const double jac = (r * r) * r;
          term = ((((((wr * wa) * wb) * wc) * jac) * K) * dAi) * dAj;
          if (a.n_nodes > 0) cast = make_ray(xi, rx, ry, rz, r2, R);
        }
      }
    }
    if (a.n_nodes > 0) {  // block-uniform
      rays += cast ? 1 : 0;
      const bool blocked = packet_any_hit(
          cast, a.nodes, a.n_nodes, [&](const NodeD& nd) { return slab_d(nd, R); },
          [&](int kk, bool test) {
            const TriD tr = a.tris[kk];
            if (!test || tr.group == P.gi || tr.group == P.gj) return false;
            ++tc.prims;
            return mt_d(tr, R);
          },
          tc);
      if (blocked) term = 0.0;
    }
    part += term;
  }
  // deterministic block reduction
  __shared__ double red[256];
  red[threadIdx.x] = part;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double raw = red[0];
    const int64_t N = a.N;
    a.F[(int64_t)P.i + (int64_t)P.j * N] = raw / a.area_orig[P.i];
    a.F[(int64_t)P.j + (int64_t)P.i * N] = raw / a.area_orig[P.j];
  }
  if (a.counters) {
    rays = warp_sum_u64(rays);
    const uint64_t s_prims = warp_sum_u64(tc.prims), s_nodes = warp_sum_u64(tc.nodes);
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(a.counters + 1, rays);
      atomicAdd(a.counters + 2, s_nodes);
      atomicAdd(a.counters + 3, s_prims);
    }
  }
}

cudaError_t launch_duffy(const DuffyArgs& a, cudaStream_t st) {
  if (a.n_pairs == 0) return cudaSuccess;
  k_duffy<<<(unsigned)a.n_pairs, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace rvf
