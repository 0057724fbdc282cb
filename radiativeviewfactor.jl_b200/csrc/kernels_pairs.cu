// kernels_pairs.cu -- quadrature tables, the tiled pair-integration kernel
// (with warp-coherent shadow rays) and the result reductions.
//
// Replaces _vf_pair_kernel! (src/GPUKernels.jl:226-323), launch_vf_kernel!
// (src/GPUKernels.jl:454-500), gpu_intersect_bvh (src/GPUBVH.jl:202-285),
// the host-side F = raw ./ A (src/GPUAssembly.jl:91) and _aggregate
// (src/Results.jl:56-82).
#include <cuda_runtime.h>

#include <cstdint>

#include "device_trace.cuh"
#include "kernels.h"

namespace rvf {

// ---------------------------------------------------------------------------
// Quadrature tables.  One thread per element evaluates every quadrature point
// exactly as _sample does (src/GPUKernels.jl:187-202) and stores
//   tab[(tile*kComp + c)*pmax*32 + p*32 + lane],  c = x,y,z,nx,ny,nz,w*dA
// so that one tile of 32 elements is one contiguous block (one bulk copy).
// area[e] = sum_p w_p dA_p in the reference's order (src/GPUKernels.jl:262-267).
// ---------------------------------------------------------------------------
__global__ void k_prep(PrepArgs a) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.N) return;
  const int f = a.fam[e];
  const int32_t* en = a.enodes + 8 * e;
  const int64_t tile = e / kTile;
  const int lane = (int)(e % kTile);
  double* base = a.tab + tile * kComp * a.pmax * kTile + lane;
  int np;
  const double *rx, *re, *rw;
  if (is_line_fam(f)) { np = a.nline; rx = a.lx; re = a.lx; rw = a.lw; }
  else if (is_quad_fam(f)) { np = a.nquadpts; rx = a.qx; re = a.qe; rw = a.qw; }
  else { np = a.ntripts; rx = a.tx; re = a.te; rw = a.tw; }
  double A = 0.0;
  double n0[3] = {0.0, 0.0, 0.0};
  bool flat = true;
  double cx = 0.0, cy = 0.0, cz = 0.0;
  for (int p = 0; p < np; ++p) {
    double x[3], n[3], dA;
    if (is_line_fam(f)) eval_line(a.coords, en, f, rx[p], x, n, &dA);
    else eval_surface(a.coords, en, f, rx[p], re[p], x, n, &dA);
    A = A + rw[p] * dA;
    double wd = rw[p] * dA;
    base[(0 * a.pmax + p) * kTile] = x[0];
    base[(1 * a.pmax + p) * kTile] = x[1];
    base[(2 * a.pmax + p) * kTile] = x[2];
    base[(3 * a.pmax + p) * kTile] = n[0];
    base[(4 * a.pmax + p) * kTile] = n[1];
    base[(5 * a.pmax + p) * kTile] = n[2];
    base[(6 * a.pmax + p) * kTile] = wd;
    if (p == 0) { n0[0] = n[0]; n0[1] = n[1]; n0[2] = n[2]; }
    else flat = flat && (n[0] == n0[0]) && (n[1] == n0[1]) && (n[2] == n0[2]);
    cx += x[0]; cy += x[1]; cz += x[2];
    if (!(dA > 0.0) || !(dA < 1e300)) atomicOr(a.err, kErrBadInput);
  }
  a.area[e] = A;
  if (a.area_orig) a.area_orig[a.orig ? a.orig[e] : e] = A;
  a.np[e] = (int8_t)np;
  a.flat[e] = flat ? 1 : 0;
  a.nrm[3 * e + 0] = n0[0];
  a.nrm[3 * e + 1] = n0[1];
  a.nrm[3 * e + 2] = n0[2];
  // centroid of the quadrature points and element diameter (corner-to-corner)
  double inv = 1.0 / np;
  a.cen[3 * e + 0] = cx * inv;
  a.cen[3 * e + 1] = cy * inv;
  a.cen[3 * e + 2] = cz * inv;
  int nc = (f == 0 || f == 2) ? 4 : (f == 1 || f == 3) ? 3 : 2;
  double dm = 0.0;
  for (int u = 0; u < nc; ++u)
    for (int v = u + 1; v < nc; ++v) {
      const double* pu = a.coords + 3 * (int64_t)en[u];
      const double* pv = a.coords + 3 * (int64_t)en[v];
      double dx = pu[0] - pv[0], dy = pu[1] - pv[1], dz = pu[2] - pv[2];
      dm = fmax(dm, sqrt(dx * dx + dy * dy + dz * dz));
    }
  a.diam[e] = dm;
  if (a.rad) {
    double r2max = 0.0;
    for (int p = 0; p < np; ++p) {
      const double dx = base[(0 * a.pmax + p) * kTile] - a.cen[3 * e + 0];
      const double dy = base[(1 * a.pmax + p) * kTile] - a.cen[3 * e + 1];
      const double dz = base[(2 * a.pmax + p) * kTile] - a.cen[3 * e + 2];
      r2max = fmax(r2max, dx * dx + dy * dy + dz * dz);
    }
    a.rad[e] = sqrt(r2max) * (1.0 + 1e-12);
  }
}

// ---------------------------------------------------------------------------
// Pair kernel.
//
// Persistent blocks pull 32x32 tiles of the upper triangle (bi <= bj) from a
// global counter.  The source tile's quadrature block (32 elements x pmax
// points x 7 doubles) is staged into shared memory with one cp.async.bulk;
// warp w integrates rows i = 32 bi + w + 8k against the 32 destination
// elements j = 32 bj + lane, whose points are read as coalesced SoA loads.
//
// Shadow rays (src/GPUKernels.jl:289-304) are formed with the reference's
// arithmetic.  A ray that misses the root box is visible and its term is
// summed at once; the others go to the warp's buffer with their term
// w_j (w_i K), and every 32 buffered rays are traced together, one per lane
// (device_trace.cuh).  The owners add the terms of their visible rays in
// buffer order after each batch, and the last partial batch of a row is
// traced before the row's F entries are written.
// ---------------------------------------------------------------------------
// Traces the first n buffered rays of the warp (rows of one source element
// against the destination tile jt) and adds the visible terms to accd.  Kept
// out of line: it runs once per 32 rays and would otherwise raise the
// register pressure of the quadrature loop.
template <bool DIM3>
__device__ __noinline__ void flush_fp64(const PairArgs& a, WarpScratch& ws, const NodeD* nodes, const double* ib,
                                        const double* jt, int n, int& nbuf, int32_t gi, int32_t gj, int64_t oi,
                                        int64_t oj, double& accd, TravCount& tc) {
  const int lane = threadIdx.x & 31;
  const int pm = a.pmax;
  const bool have = lane < n;
  const uint32_t e = have ? ws.meta[0][lane] : 0u;
  const int L = ent_lane(e), p = ent_p(e), q = ent_q(e);
  const bool esw = ent_sw(e);
  const int32_t gL = __shfl_sync(kFull, gj, L);
  const int64_t oL = __shfl_sync(kFull, oj, L);
  double xi[3], xj[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    xi[c] = have ? ib[(c * pm + p) * kTile] : 0.0;
    xj[c] = have ? jt[(c * pm + q) * kTile + L] : 0.0;
  }
  int r;
  if (DIM3) {
    PolD3 pol;
    pol.tris = a.tris;
    const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
    const double r2 = (rx * rx + ry * ry) + rz * rz;
    if (have) {
      if (esw) make_ray(xj, -rx, -ry, -rz, r2, pol.R);
      else make_ray(xi, rx, ry, rz, r2, pol.R);
      pol.store(ws.bank, lane, gi, gL);
    }
    r = trace_batch(have, GlobalNodes<NodeD>{nodes}, a.n_nodes, ws.bank, pol, tc);
  } else {
    PolD2 pol;
    pol.segs = a.segs;
    pol.a[0] = esw ? xj[0] : xi[0];
    pol.a[1] = esw ? xj[1] : xi[1];
    pol.b[0] = esw ? xi[0] : xj[0];
    pol.b[1] = esw ? xi[1] : xj[1];
    if (have) pol.store(ws.bank, lane, gi, gL);
    r = trace_batch(have, GlobalNodes<NodeD>{nodes}, a.n_nodes, ws.bank, pol, tc);
  }
  if (have && a.ray_log) {
    uint8_t* lp = a.ray_log + ((uint64_t)(esw ? oL : oi) * a.N + (esw ? oi : oL)) * a.log_pm * a.log_pm;
    lp[esw ? q * a.log_pm + p : p * a.log_pm + q] = (r == kHit) ? 2 : 1;
  }
  const uint32_t vis = __ballot_sync(kFull, have && r != kHit);
  buf_collect(ws, 0, n, vis, accd);
  buf_shift(ws, 0, nbuf, n);
}

template <bool DIM3, bool OCC>
__global__ void __launch_bounds__(256, 2) k_pairs_fp64(PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int pm = a.pmax;
  double* iblk = reinterpret_cast<double*>(smem);
  NodeD* snodes = reinterpret_cast<NodeD*>(iblk + kComp * pm * kTile);
  WarpScratch* wsa = reinterpret_cast<WarpScratch*>(snodes + (a.nodes_in_smem ? a.n_nodes : 0));
  uint64_t* bar = reinterpret_cast<uint64_t*>(wsa + (OCC ? 8 : 0));
  __shared__ int64_t s_tile;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpScratch& ws = wsa[OCC ? warp : 0];
  const NodeD* nodes = a.nodes;
  if (OCC && a.nodes_in_smem) {
    const int4* src = reinterpret_cast<const int4*>(a.nodes);
    int4* dst = reinterpret_cast<int4*>(snodes);
    for (int k = threadIdx.x; k < a.n_nodes * 4; k += blockDim.x) dst[k] = src[k];
    nodes = snodes;
  }
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();

  const uint32_t blk_bytes = (uint32_t)(kComp * pm * kTile * sizeof(double));
  uint32_t phase = 0;
  uint32_t n_rays = 0, n_pp = 0;
  TravCount tc;
  for (;;) {
    if (threadIdx.x == 0) {
      s_tile = (int64_t)atomicAdd(a.tile_counter, 1ull);
      if (s_tile < a.n_tiles) {
        int64_t bi, bj;
        tile_coords(s_tile, a.nT, bi, bj);
        mbar_expect_tx(bar, blk_bytes);
        bulk_g2s(iblk, a.tab + bi * kComp * pm * kTile, blk_bytes, bar);
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

    const int64_t N = a.N;
    const int64_t j = bj * kTile + lane;
    const int64_t oj = (j < N) ? (a.orig ? (int64_t)a.orig[j] : j) : 0;
    const double* jt = a.tab + bj * kComp * pm * kTile;  // destination tile block
    const double* jb = jt + lane;
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int li = warp + 8 * rr;
      const int64_t i = bi * kTile + li;
      if (i >= N) continue;  // warp-uniform
      const bool valid = (j < N) && (i < j);
      const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
      // the reference casts from the element with the lower (caller's) index
      const bool sw = valid && oi > oj;
      const int npi = a.np[i];
      int npj = valid ? a.np[j] : 0;
      // Two elements whose points all share one normal, bit for bit, have
      // cos_j = -cos_i exactly at every point pair: K = 0, no rays.
      if (valid && a.flat[i] && a.flat[j] && a.nrm[3 * i] == a.nrm[3 * j] &&
          a.nrm[3 * i + 1] == a.nrm[3 * j + 1] && a.nrm[3 * i + 2] == a.nrm[3 * j + 2])
        npj = 0;
      const int qmax = __reduce_max_sync(kFull, npj);
      const int32_t gi = a.group[i];
      const int32_t gj = valid ? a.group[j] : gi;
      const double* ib = iblk + li;
      uint8_t* logp = (a.ray_log && valid)
                          ? a.ray_log + ((uint64_t)(sw ? oj : oi) * N + (sw ? oi : oj)) * a.log_pm * a.log_pm
                          : nullptr;
      double acc = 0.0, accd = 0.0;
      int nbuf = 0;  // warp-uniform buffer fill

      for (int q = 0; q < qmax; ++q) {
        const bool lq = q < npj;
        double xj[3], nj[3], wj;
        if (lq) {
          xj[0] = jb[(0 * pm + q) * kTile];
          xj[1] = jb[(1 * pm + q) * kTile];
          xj[2] = jb[(2 * pm + q) * kTile];
          nj[0] = jb[(3 * pm + q) * kTile];
          nj[1] = jb[(4 * pm + q) * kTile];
          nj[2] = jb[(5 * pm + q) * kTile];
          wj = jb[(6 * pm + q) * kTile];
        } else {
          xj[0] = xj[1] = xj[2] = 0.0;
          nj[0] = nj[1] = nj[2] = 0.0;
          wj = 0.0;
        }
        double inner = 0.0;
        for (int p = 0; p < npi; ++p) {
          double xi[3], ni[3];
          xi[0] = ib[(0 * pm + p) * kTile];
          xi[1] = ib[(1 * pm + p) * kTile];
          xi[2] = ib[(2 * pm + p) * kTile];
          ni[0] = ib[(3 * pm + p) * kTile];
          ni[1] = ib[(4 * pm + p) * kTile];
          ni[2] = ib[(5 * pm + p) * kTile];
          const double wi = ib[(6 * pm + p) * kTile];
          const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
          const double r2 = (rx * rx + ry * ry) + rz * rz;
          double K = lq ? k_fast<DIM3>(rx, ry, rz, r2, ni, nj) : 0.0;
          n_pp += lq ? 1 : 0;
          if (OCC) {
            bool cast, defer = false;
            const NodeD& root = nodes[0];
            if (DIM3) {
              RayD R;
              cast = (K > 0.0) && (sw ? make_ray(xj, -rx, -ry, -rz, r2, R) : make_ray(xi, rx, ry, rz, r2, R));
              if (cast) defer = slab_d(root, R);
            } else {
              cast = K > 0.0;
              if (cast) {
                PolD2 pol;
                pol.a[0] = xi[0]; pol.a[1] = xi[1];
                pol.b[0] = xj[0]; pol.b[1] = xj[1];
                defer = pol.node(root) == kHit;
              }
            }
            n_rays += cast ? 1 : 0;
            if (logp && cast && !defer) logp[sw ? q * a.log_pm + p : p * a.log_pm + q] = 1;
            buf_push(ws, 0, nbuf, defer, enc_entry(lane, sw, p, q), wj * (wi * K));
            if (defer) K = 0.0;
            if (nbuf >= 32) flush_fp64<DIM3>(a, ws, nodes, ib, jt, 32, nbuf, gi, gj, oi, oj, accd, tc);
          }
          inner = fma(wi, K, inner);
        }
        acc = fma(wj, inner, acc);
      }
      if (OCC && nbuf > 0) flush_fp64<DIM3>(a, ws, nodes, ib, jt, nbuf, nbuf, gi, gj, oi, oj, accd, tc);
      const double raw = acc + accd;
      // F[i,j] = raw/A_i and F[j,i] = raw/A_j in the caller's element order
      if (valid) {
        a.F[oi + oj * N] = raw / a.area[i];
        a.F[oj + oi * N] = raw / a.area[j];
      } else if (j == i) {
        a.F[oi + oi * N] = 0.0 / a.area[i];
      }
    }
    __syncthreads();
  }
  // counters (one atomic per warp)
  const uint64_t s_rays = warp_sum_u64(n_rays), s_pp = warp_sum_u64(n_pp), s_nodes = warp_sum_u64(tc.nodes),
                 s_prims = warp_sum_u64(tc.prims);
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, s_pp);
    atomicAdd(a.counters + 1, s_rays);
    atomicAdd(a.counters + 2, s_nodes);
    atomicAdd(a.counters + 3, s_prims);
  }
}

// ---------------------------------------------------------------------------
// Reductions (deterministic).  Pass 1: thread per row i and column chunk,
// Neumaier-compensated sums over the chunk's columns of each group.
// Pass 2: per row, sum the chunks in order -> row-group sums S[h][i] and row
// sums.  Pass 3: F_group[g,h] = sum_{i in g} A_i S[h][i] / A_g.
// ---------------------------------------------------------------------------
struct Neu {
  double s = 0.0, c = 0.0;
  __device__ void add(double v) {
    double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
  }
  __device__ double val() const { return s + c; }
};

__global__ void k_rowgroup_partial(RedArgs a) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int chunk = blockIdx.y;
  if (i >= a.N) return;
  for (int h = 0; h < a.G; ++h) {
    const int64_t b = a.member_off[h], e = a.member_off[h + 1];
    const int64_t len = e - b;
    const int64_t cb = b + (len * chunk) / a.n_chunks, ce = b + (len * (chunk + 1)) / a.n_chunks;
    Neu s;
    for (int64_t k = cb; k < ce; ++k) s.add(a.F[i + (int64_t)a.members[k] * a.N]);
    a.part[((int64_t)chunk * a.G + h) * a.N + i] = s.val();
  }
}

__global__ void k_rowgroup_final(RedArgs a) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  Neu row;
  for (int h = 0; h < a.G; ++h) {
    Neu s;
    for (int c = 0; c < a.n_chunks; ++c) s.add(a.part[((int64_t)c * a.G + h) * a.N + i]);
    double v = s.val();
    a.rowgroup[(int64_t)h * a.N + i] = v;
    row.add(v);
  }
  a.rowsum[i] = row.val();
}

// one block per (g, h)
__global__ void k_group_final(RedArgs a) {
  const int g = blockIdx.x, h = blockIdx.y;
  __shared__ double sh_s[256], sh_c[256], sh_a[256], sh_ac[256];
  const int64_t b = a.member_off[g], e = a.member_off[g + 1];
  Neu s, ag;
  for (int64_t k = b + threadIdx.x; k < e; k += blockDim.x) {
    const int64_t i = a.members[k];
    s.add(a.area[i] * a.rowgroup[(int64_t)h * a.N + i]);
    ag.add(a.area[i]);
  }
  sh_s[threadIdx.x] = s.s; sh_c[threadIdx.x] = s.c;
  sh_a[threadIdx.x] = ag.s; sh_ac[threadIdx.x] = ag.c;
  __syncthreads();
  if (threadIdx.x == 0) {
    Neu S, A;
    for (int t = 0; t < blockDim.x; ++t) {
      S.add(sh_s[t]); S.add(sh_c[t]);
      A.add(sh_a[t]); A.add(sh_ac[t]);
    }
    const double Ag = A.val();
    a.Fgroup[g + (int64_t)h * a.G] = S.val() / Ag;
    if (h == 0) a.Agroup[g] = Ag;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
cudaError_t launch_prep(const PrepArgs& a, cudaStream_t st) {
  if (a.N == 0) return cudaSuccess;
  int bs = 128;
  k_prep<<<(unsigned)((a.N + bs - 1) / bs), bs, 0, st>>>(a);
  return cudaGetLastError();
}

size_t pair_smem_bytes(int pmax, int n_nodes_smem, bool occ) {
  return (size_t)kComp * pmax * kTile * sizeof(double) + (size_t)n_nodes_smem * sizeof(NodeD) +
         (occ ? 8 * sizeof(WarpScratch) : 0) + 16;
}

template <bool D3, bool O>
static cudaError_t launch_pairs_t(const PairArgs& a, int grid, size_t smem, cudaStream_t st) {
  auto fn = k_pairs_fp64<D3, O>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<grid, 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_pairs_fp64(const PairArgs& a, int sm_count, cudaStream_t st) {
  const size_t smem = pair_smem_bytes(a.pmax, a.nodes_in_smem ? a.n_nodes : 0, a.n_nodes > 0);
  int per_sm = (int)((200 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 4) per_sm = 4;
  int64_t grid = (int64_t)sm_count * per_sm;
  if (grid > a.n_tiles) grid = a.n_tiles;
  if (grid < 1) grid = 1;
  const bool occ = a.n_nodes > 0;
  if (a.dim3) return occ ? launch_pairs_t<true, true>(a, (int)grid, smem, st) : launch_pairs_t<true, false>(a, (int)grid, smem, st);
  return occ ? launch_pairs_t<false, true>(a, (int)grid, smem, st) : launch_pairs_t<false, false>(a, (int)grid, smem, st);
}

cudaError_t launch_reduce(const RedArgs& a, cudaStream_t st) {
  if (a.N == 0 || a.G == 0) return cudaSuccess;
  dim3 g1((unsigned)((a.N + 127) / 128), (unsigned)a.n_chunks);
  k_rowgroup_partial<<<g1, 128, 0, st>>>(a);
  k_rowgroup_final<<<(unsigned)((a.N + 127) / 128), 128, 0, st>>>(a);
  dim3 g3((unsigned)a.G, (unsigned)a.G);
  k_group_final<<<g3, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace rvf
