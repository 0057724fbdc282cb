// kernels_self.cu -- self view factors: the diagonal pairs (i, i).
//
// The reference integrates the pair (i, i) only on its CPU path, when
// self_vf is set (src/Assembly.jl:173,193: j_start = self_vf ? i : i + 1),
// with the integrator of every other pair (src/ViewFactorKernel.jl:199-303):
// K = 0 where two points coincide (r^2 < 1e-30) or where either cosine is
// <= 0, so only a curved, concave element sees itself.  Occlusion uses the
// obstruction groups other than the element's own (src/Assembly.jl:121-125).
//
// One warp integrates one element.  Its lanes take the point pairs (p, q) in
// turn, 32 at a time; where K > 0 the lane forms the shadow ray from point p
// to point q with the reference's arithmetic (make_ray / the 2-D segment),
// and the rays of the 32 pairs are traced together (trace_batch, the
// traversal of the pair pipeline's queues, with the element's group skipped).
// Each lane sums its terms in its own order and the warp adds the 32 partial
// sums in a fixed butterfly, so the result does not depend on timing.  The
// self pairs run in FP64 in both precision modes: N pairs next to the
// N (N - 1) / 2 of the pipeline.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_trace.cuh"
#include "kernels.h"

namespace rvf {

constexpr int kSelfWarps = 4;  // warps per block (one ray bank each in shared memory)

template <bool DIM3>
__global__ void __launch_bounds__(32 * kSelfWarps) k_self(PairArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  RayBank* banks = reinterpret_cast<RayBank*>(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RayBank& bank = banks[warp];
  const int64_t N = a.N;
  const int pm = a.pmax;
  const bool occ = a.n_nodes > 0;
  const int64_t stride = (int64_t)gridDim.x * kSelfWarps;
  uint64_t n_pp = 0, n_rays = 0;
  TravCount tc;
  for (int64_t i = (int64_t)blockIdx.x * kSelfWarps + warp; i < N; i += stride) {  // warp-uniform
    const int np = a.np[i];
    const double* b = a.tab + (i / kTile) * kComp * pm * kTile + (i % kTile);
    const int32_t g = a.group[i];
    const int total = np * np;
    double acc = 0.0;
    for (int base = 0; base < total; base += 32) {  // warp-uniform trip count
      const int t = base + lane;
      const bool have = t < total;
      const int p = have ? t / np : 0, q = have ? t % np : 0;
      double xi[3], ni[3], xj[3], nj[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        xi[c] = b[(c * pm + p) * kTile];
        ni[c] = b[((3 + c) * pm + p) * kTile];
        xj[c] = b[(c * pm + q) * kTile];
        nj[c] = b[((3 + c) * pm + q) * kTile];
      }
      const double wp = b[(6 * pm + p) * kTile], wq = b[(6 * pm + q) * kTile];
      const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
      const double r2 = (rx * rx + ry * ry) + rz * rz;
      double K = have ? k_fast<DIM3>(rx, ry, rz, r2, ni, nj) : 0.0;
      n_pp += have ? 1 : 0;
      if (occ) {
        bool cast;
        int r = kMiss;
        if (DIM3) {
          PolD3 pol;
          pol.tris = a.tris;
          cast = (K > 0.0) && make_ray(xi, rx, ry, rz, r2, pol.R);
          if (__any_sync(kFull, cast)) {
            if (cast) pol.store(bank, lane, g, g);
            r = trace_batch(cast, GlobalNodes<NodeD>{a.nodes}, a.n_nodes, bank, pol, tc);
          }
        } else {
          PolD2 pol;
          pol.segs = a.segs;
          pol.a[0] = xi[0];
          pol.a[1] = xi[1];
          pol.b[0] = xj[0];
          pol.b[1] = xj[1];
          cast = K > 0.0;
          if (__any_sync(kFull, cast)) {
            if (cast) pol.store(bank, lane, g, g);
            r = trace_batch(cast, GlobalNodes<NodeD>{a.nodes}, a.n_nodes, bank, pol, tc);
          }
        }
        n_rays += cast ? 1 : 0;
        if (cast && r == kHit) K = 0.0;
      }
      acc = fma(wq, wp * K, acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane == 0) {
      const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
      a.F[oi + oi * N] = acc / a.area[i];
    }
  }
  const uint64_t s_pp = warp_sum_u64(n_pp), s_rays = warp_sum_u64(n_rays), s_nodes = warp_sum_u64(tc.nodes),
                 s_prims = warp_sum_u64(tc.prims);
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, s_pp);
    atomicAdd(a.counters + 1, s_rays);
    atomicAdd(a.counters + 2, s_nodes);
    atomicAdd(a.counters + 3, s_prims);
  }
}

cudaError_t launch_self(const PairArgs& a, cudaStream_t st) {
  if (a.N <= 0) return cudaSuccess;
  const int64_t blocks = (a.N + kSelfWarps - 1) / kSelfWarps;
  const size_t smem = sizeof(RayBank) * kSelfWarps;
  if (a.dim3) k_self<true><<<(unsigned)blocks, 32 * kSelfWarps, smem, st>>>(a);
  else k_self<false><<<(unsigned)blocks, 32 * kSelfWarps, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace rvf
