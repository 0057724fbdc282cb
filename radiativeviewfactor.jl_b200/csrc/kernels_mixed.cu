// kernels_mixed.cu -- mixed-precision pair integration (surface meshes).
//
// Far-field pairs (centroid distance >= near_field_factor x the larger element
// diameter) integrate in FP32 with FP32 per-pair accumulation; positions are
// FP32 offsets from an FP64 per-element anchor, so r = (anchor_j - anchor_i)
// + (off_q - off_p) keeps ~1e-7 relative accuracy.  FP64 is kept where
// stability needs it:
//   * near-field pairs: the whole pair runs the FP64 path of k_pairs_fp64;
//   * grazing point pairs (|cos| < 1e-5 in FP32): the reference's K in FP64;
//   * every shadow ray whose FP32 traversal met an uncertain decision (or
//     whose direction has a component below 1e-4): traced again in FP64 with
//     the reference's arithmetic, so every visibility decision is the
//     reference's (device_mixed.cuh);
//   * F = raw/A and the group / row reductions stay FP64.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_mixed.cuh"
#include "kernels.h"

namespace rvf {

// FP32 table: per point the offset from the element centroid, the normal and
// w*dA, tile-blocked like the FP64 table ([tile][7][pmax][32] floats).
__global__ void k_prep_f32(PrepF32Args a) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.N) return;
  const int64_t tile = e / kTile;
  const int lane = (int)(e % kTile);
  const double* src = a.tab + tile * kComp * a.pmax * kTile + lane;
  float* dst = a.tabf + tile * kComp * a.pmax * kTile + lane;
  const int np = a.np[e];
  const double c0 = a.cen[3 * e], c1 = a.cen[3 * e + 1], c2 = a.cen[3 * e + 2];
  for (int p = 0; p < np; ++p) {
    dst[(0 * a.pmax + p) * kTile] = (float)(src[(0 * a.pmax + p) * kTile] - c0);
    dst[(1 * a.pmax + p) * kTile] = (float)(src[(1 * a.pmax + p) * kTile] - c1);
    dst[(2 * a.pmax + p) * kTile] = (float)(src[(2 * a.pmax + p) * kTile] - c2);
    for (int c = 3; c < kComp; ++c) dst[(c * a.pmax + p) * kTile] = (float)src[(c * a.pmax + p) * kTile];
  }
}

template <bool OCC>
__global__ void __launch_bounds__(256, 2) k_pairs_mixed(MixedArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  float* iblk = reinterpret_cast<float*>(smem);
  NodeF* snodes = reinterpret_cast<NodeF*>(smem + (size_t)kComp * a.pmax * kTile * sizeof(float));
  uint64_t* bar = reinterpret_cast<uint64_t*>(snodes + (a.nodesf_in_smem ? a.n_nodes : 0));
  __shared__ int64_t s_tile;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const NodeF* nodesf = a.nodesf;
  if (OCC && a.nodesf_in_smem) {
    const int4* src = reinterpret_cast<const int4*>(a.nodesf);
    int4* dst = reinterpret_cast<int4*>(snodes);
    for (int k = threadIdx.x; k < a.n_nodes * 2; k += blockDim.x) dst[k] = src[k];
    nodesf = snodes;
  }
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();

  const int pm = a.pmax;
  const uint32_t blk_bytes = (uint32_t)(kComp * pm * kTile * sizeof(float));
  uint32_t phase = 0;
  uint64_t n_pp = 0, n_rays = 0, n_rays64 = 0, n_near = 0, n_graze = 0, n_unsure = 0, n_baddir = 0;
  TravCount tc, tc64;
  for (;;) {
    if (threadIdx.x == 0) {
      s_tile = (int64_t)atomicAdd(a.tile_counter, 1ull);
      if (s_tile < a.n_tiles) {
        int64_t bi, bj;
        tile_coords(s_tile, a.nT, bi, bj);
        mbar_expect_tx(bar, blk_bytes);
        bulk_g2s(iblk, a.tabf + bi * kComp * pm * kTile, blk_bytes, bar);
      }
    }
    __syncthreads();
    const int64_t t = s_tile;
    if (t >= a.n_tiles) break;
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const bool ok = mbar_wait_bounded(bar, phase);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(a.err, kErrWaitTimeout);
      break;
    }
    phase ^= 1u;

    const int64_t j = bj * kTile + lane;
    const int64_t N = a.N;
    const int64_t oj = (j < N) ? (a.orig ? (int64_t)a.orig[j] : j) : 0;
    const float* jbf = a.tabf + bj * kComp * pm * kTile + lane;
    const double* jb64 = a.tab + bj * kComp * pm * kTile + lane;
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int li = warp + 8 * rr;
      const int64_t i = bi * kTile + li;
      double acc64 = 0.0;
      float acc32 = 0.0f;
      if (i < a.N) {  // warp-uniform
        const bool valid = (j < a.N) && (i < j);
        const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
        const bool sw = valid && oi > oj;  // rays leave the element with the lower caller index
        const int npi = a.np[i];
        int npj = valid ? a.np[j] : 0;
        if (valid && a.flat[i] && a.flat[j] && a.nrm[3 * i] == a.nrm[3 * j] &&
            a.nrm[3 * i + 1] == a.nrm[3 * j + 1] && a.nrm[3 * i + 2] == a.nrm[3 * j + 2])
          npj = 0;
        const int qmax = __reduce_max_sync(kFull, npj);
        const int32_t gi = a.group[i];
        const int32_t gj = valid ? a.group[j] : gi;
        const double ci0 = a.cen[3 * i], ci1 = a.cen[3 * i + 1], ci2 = a.cen[3 * i + 2];
        double dc0 = 0.0, dc1 = 0.0, dc2 = 0.0;
        bool near = false;
        if (valid) {
          dc0 = a.cen[3 * j] - ci0; dc1 = a.cen[3 * j + 1] - ci1; dc2 = a.cen[3 * j + 2] - ci2;
          const double dm = fmax(a.diam[i], a.diam[j]) * a.near_factor;
          near = (dc0 * dc0 + dc1 * dc1 + dc2 * dc2) < dm * dm;
        }
        n_near += (near && npj > 0) ? 1 : 0;
        const float d0 = (float)dc0, d1 = (float)dc1, d2 = (float)dc2;
        // FP32 ray origin anchor: the centroid of the casting element
        const float ai0 = (float)(ci0 + (sw ? dc0 : 0.0)), ai1 = (float)(ci1 + (sw ? dc1 : 0.0)),
                    ai2 = (float)(ci2 + (sw ? dc2 : 0.0));
        const float* ibf = iblk + li;
        const double* ib64 = a.tab + bi * kComp * pm * kTile + li;
        uint8_t* logp = (a.ray_log && valid)
                            ? a.ray_log + ((uint64_t)(sw ? oj : oi) * a.N + (sw ? oi : oj)) * a.log_pm * a.log_pm
                            : nullptr;
        for (int q = 0; q < qmax; ++q) {
          const bool lq = q < npj;
          const bool far = lq && !near;
          float oq0 = 0.f, oq1 = 0.f, oq2 = 0.f, nq0 = 0.f, nq1 = 0.f, nq2 = 0.f, wq = 0.f;
          if (far) {
            oq0 = jbf[(0 * pm + q) * kTile]; oq1 = jbf[(1 * pm + q) * kTile]; oq2 = jbf[(2 * pm + q) * kTile];
            nq0 = jbf[(3 * pm + q) * kTile]; nq1 = jbf[(4 * pm + q) * kTile]; nq2 = jbf[(5 * pm + q) * kTile];
            wq = jbf[(6 * pm + q) * kTile];
          }
          bool have64 = false;
          double xj[3] = {0.0, 0.0, 0.0}, nj[3] = {0.0, 0.0, 0.0}, wj64 = 0.0;
          float inner = 0.0f;
          for (int p = 0; p < npi; ++p) {
            // ---- stage A: FP32 far field ----
            const float op0 = ibf[(0 * pm + p) * kTile], op1 = ibf[(1 * pm + p) * kTile],
                        op2 = ibf[(2 * pm + p) * kTile];
            const float np0 = ibf[(3 * pm + p) * kTile], np1 = ibf[(4 * pm + p) * kTile],
                        np2 = ibf[(5 * pm + p) * kTile];
            const float wp = ibf[(6 * pm + p) * kTile];
            const float rx = d0 + (oq0 - op0), ry = d1 + (oq1 - op1), rz = d2 + (oq2 - op2);
            const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
            const float di = fmaf(np0, rx, fmaf(np1, ry, np2 * rz));
            const float dj = -fmaf(nq0, rx, fmaf(nq1, ry, nq2 * rz));
            const bool graze = far && (di * di <= 1e-10f * r2 || dj * dj <= 1e-10f * r2 || r2 < 1e-18f);
            float K32 = 0.0f;
            if (far && !graze && di > 0.0f && dj > 0.0f) K32 = (di * dj) * rcp_approx(3.14159265f * (r2 * r2));
            bool cast32 = far && !graze && K32 > 0.0f;
            bool hit32 = false, unsure = false, badray = false;
            n_pp += lq ? 1 : 0;
            if (OCC) {
              RayF R;
              bool rok = false;
              if (cast32) {
                const float xo[3] = {ai0 + (sw ? oq0 : op0), ai1 + (sw ? oq1 : op1), ai2 + (sw ? oq2 : op2)};
                rok = sw ? make_ray_f(xo, -rx, -ry, -rz, r2, a.delta, R) : make_ray_f(xo, rx, ry, rz, r2, a.delta, R);
                badray = !rok;
              }
              n_rays += cast32 ? 1 : 0;
              hit32 = packet_any_hit_f(
                  cast32 && rok, nodesf, a.n_nodes, R,
                  [&](int k, bool test) -> int {
                    if (!test) return kMiss;
                    const TriF tr = a.trisf[k];
                    if (tr.group == gi || tr.group == gj) return kMiss;
                    ++tc.prims;
                    return mt_f(tr, R);
                  },
                  unsure, tc);
              n_unsure += (unsure || badray) ? 1 : 0;
              n_baddir += badray ? 1 : 0;
            }
            // ---- stage B: FP64 (near field, grazing, uncertain rays) ----
            const bool need64 = lq && (near || graze || unsure || badray);
            double K64 = 0.0;
            bool hit64 = false;
            uint8_t lg = cast32 ? (hit32 ? 2 : 1) : 0;
            if (__any_sync(kFull, need64)) {
              double xi[3], ni[3];
              xi[0] = ib64[(0 * pm + p) * kTile]; xi[1] = ib64[(1 * pm + p) * kTile]; xi[2] = ib64[(2 * pm + p) * kTile];
              ni[0] = ib64[(3 * pm + p) * kTile]; ni[1] = ib64[(4 * pm + p) * kTile]; ni[2] = ib64[(5 * pm + p) * kTile];
              const double wi64 = ib64[(6 * pm + p) * kTile];
              if (need64 && !have64) {
                xj[0] = jb64[(0 * pm + q) * kTile]; xj[1] = jb64[(1 * pm + q) * kTile]; xj[2] = jb64[(2 * pm + q) * kTile];
                nj[0] = jb64[(3 * pm + q) * kTile]; nj[1] = jb64[(4 * pm + q) * kTile]; nj[2] = jb64[(5 * pm + q) * kTile];
                wj64 = jb64[(6 * pm + q) * kTile];
                have64 = true;
              }
              const double rx64 = xj[0] - xi[0], ry64 = xj[1] - xi[1], rz64 = xj[2] - xi[2];
              const double r264 = (rx64 * rx64 + ry64 * ry64) + rz64 * rz64;
              const bool exactK = need64 && (near || graze);
              if (exactK) K64 = k_fast<true>(rx64, ry64, rz64, r264, ni, nj);
              if (OCC) {
                RayD R64;
                bool cast64 = need64 && ((exactK && K64 > 0.0) || (!exactK)) &&
                              (sw ? make_ray(xj, -rx64, -ry64, -rz64, r264, R64) : make_ray(xi, rx64, ry64, rz64, r264, R64));
                n_rays64 += cast64 ? 1 : 0;
                n_rays += (cast64 && exactK) ? 1 : 0;
                hit64 = packet_any_hit(
                    cast64, a.nodes, a.n_nodes, [&](const NodeD& nd) { return slab_d(nd, R64); },
                    [&](int k, bool test) {
                      const TriD tr = a.tris[k];
                      if (!test || tr.group == gi || tr.group == gj) return false;
                      ++tc64.prims;
                      return mt_d(tr, R64);
                    },
                    tc64);
                if (cast64) lg = hit64 ? 2 : 1;
                else if (exactK) lg = 0;
              }
              if (exactK) {
                n_graze += graze ? 1 : 0;
                if (hit64) K64 = 0.0;
                acc64 = fma(wi64 * wj64, K64, acc64);
              }
            }
            if (far && !graze) {
              float K = K32;
              if (hit32 || ((unsure || badray) && hit64)) K = 0.0f;
              inner = fmaf(wp, K, inner);
            }
            if (OCC && logp && lq) logp[sw ? q * a.log_pm + p : p * a.log_pm + q] = lg;
          }
          acc32 = fmaf(wq, inner, acc32);
        }
        const double raw = acc64 + (double)acc32;
        if (valid) {
          a.F[oi + oj * N] = raw / a.area[i];
          a.F[oj + oi * N] = raw / a.area[j];
        } else if (j == i) {
          a.F[oi + oi * N] = 0.0 / a.area[i];
        }
      }
    }
    __syncthreads();
  }
  n_pp = warp_sum_u64(n_pp);
  n_rays = warp_sum_u64(n_rays);
  n_rays64 = warp_sum_u64(n_rays64);
  n_near = warp_sum_u64(n_near);
  n_graze = warp_sum_u64(n_graze);
  n_unsure = warp_sum_u64(n_unsure);
  n_baddir = warp_sum_u64(n_baddir);
  tc.unsure_slab = warp_sum_u64(tc.unsure_slab);
  tc.unsure_prim = warp_sum_u64(tc.unsure_prim);
  tc.nodes = warp_sum_u64(tc.nodes + tc64.nodes);
  tc.prims = warp_sum_u64(tc.prims + tc64.prims);
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, n_pp);
    atomicAdd(a.counters + 1, n_rays);
    atomicAdd(a.counters + 2, tc.nodes);
    atomicAdd(a.counters + 3, tc.prims);
    atomicAdd(a.counters + 4, n_rays64);
    atomicAdd(a.counters + 5, n_near);
    atomicAdd(a.counters + 6, n_graze);
    atomicAdd(a.counters + 7, n_unsure);
    atomicAdd(a.counters + 8, tc.unsure_slab);
    atomicAdd(a.counters + 9, tc.unsure_prim);
    atomicAdd(a.counters + 10, n_baddir);
  }
}

cudaError_t launch_prep_f32(const PrepF32Args& a, cudaStream_t st) {
  if (a.N == 0) return cudaSuccess;
  k_prep_f32<<<(unsigned)((a.N + 127) / 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

size_t mixed_smem_bytes(int pmax, int n_nodes_smem) {
  return (size_t)kComp * pmax * kTile * sizeof(float) + (size_t)n_nodes_smem * sizeof(NodeF) + 16;
}

template <bool O>
static cudaError_t launch_mixed_t(const MixedArgs& a, int grid, size_t smem, cudaStream_t st) {
  auto fn = k_pairs_mixed<O>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_pairs_mixed(const MixedArgs& a, int sm_count, cudaStream_t st) {
  const size_t smem = mixed_smem_bytes(a.pmax, a.nodesf_in_smem ? a.n_nodes : 0);
  int per_sm = (int)((200 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 4) per_sm = 4;
  int64_t grid = (int64_t)sm_count * per_sm;
  if (grid > a.n_tiles) grid = a.n_tiles;
  if (grid < 1) grid = 1;
  return a.n_nodes > 0 ? launch_mixed_t<true>(a, (int)grid, smem, st) : launch_mixed_t<false>(a, (int)grid, smem, st);
}

}  // namespace rvf
