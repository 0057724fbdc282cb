// kernels_pairs.cu -- quadrature tables, the tiled pair-integration kernel
// (with warp-coherent shadow rays) and the result reductions.
//
// Replaces _vf_pair_kernel! (src/GPUKernels.jl:226-323), launch_vf_kernel!
// (src/GPUKernels.jl:454-500), gpu_intersect_bvh (src/GPUBVH.jl:202-285),
// the host-side F = raw ./ A (src/GPUAssembly.jl:91) and _aggregate
// (src/Results.jl:56-82).
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
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
}

// ---------------------------------------------------------------------------
// Pair kernel.
//
// Persistent blocks pull 32x32 tiles of the upper triangle (bi <= bj) from a
// global counter.  The source tile's quadrature block (32 elements x pmax
// points x 7 doubles) is staged into shared memory with one cp.async.bulk;
// warp w integrates rows i = 32 bi + w + 8k against the 32 destination
// elements j = 32 bj + lane, whose points are read as coalesced SoA loads.
// Each lane keeps one destination point in registers and loops over the
// warp-uniform source points, so every shadow ray of a warp step leaves the
// same origin towards 32 neighbouring targets and the traversal is coherent.
// The raw tile goes through shared memory so that both F[i,j] = raw/A_i and
// F[j,i] = raw/A_j are written as full 256-byte column segments.
// ---------------------------------------------------------------------------
template <bool DIM3, bool OCC>
__global__ void __launch_bounds__(256) k_pairs_fp64(PairArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  double* iblk = reinterpret_cast<double*>(smem);
  NodeD* snodes = reinterpret_cast<NodeD*>(iblk + kComp * a.pmax * kTile);
  uint64_t* bar = reinterpret_cast<uint64_t*>(snodes + (a.nodes_in_smem ? a.n_nodes : 0));
  __shared__ int64_t s_tile;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const NodeD* nodes = a.nodes;
  if (OCC && a.nodes_in_smem) {
    const int4* src = reinterpret_cast<const int4*>(a.nodes);
    int4* dst = reinterpret_cast<int4*>(snodes);
    for (int k = threadIdx.x; k < a.n_nodes * 4; k += blockDim.x) dst[k] = src[k];
    nodes = snodes;
  }
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();

  const uint32_t blk_bytes = (uint32_t)(kComp * a.pmax * kTile * sizeof(double));
  uint32_t phase = 0;
  uint64_t n_rays = 0, n_pp = 0;
  TravCount tc;
  for (;;) {
    if (threadIdx.x == 0) {
      s_tile = (int64_t)atomicAdd(a.tile_counter, 1ull);
      if (s_tile < a.n_tiles) {
        int64_t bi, bj;
        tile_coords(s_tile, a.nT, bi, bj);
        mbar_expect_tx(bar, blk_bytes);
        bulk_g2s(iblk, a.tab + bi * kComp * a.pmax * kTile, blk_bytes, bar);
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
    const double* jb = a.tab + bj * kComp * a.pmax * kTile + lane;
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int li = warp + 8 * rr;
      const int64_t i = bi * kTile + li;
      double acc = 0.0;
      if (i < a.N) {  // warp-uniform
        const bool valid = (j < a.N) && (i < j);
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
                            ? a.ray_log + ((uint64_t)(sw ? oj : oi) * a.N + (sw ? oi : oj)) * a.log_pm * a.log_pm
                            : nullptr;
        for (int q = 0; q < qmax; ++q) {
          const bool lq = q < npj;
          double xj[3], nj[3], wj;
          if (lq) {
            xj[0] = jb[(0 * a.pmax + q) * kTile];
            xj[1] = jb[(1 * a.pmax + q) * kTile];
            xj[2] = jb[(2 * a.pmax + q) * kTile];
            nj[0] = jb[(3 * a.pmax + q) * kTile];
            nj[1] = jb[(4 * a.pmax + q) * kTile];
            nj[2] = jb[(5 * a.pmax + q) * kTile];
            wj = jb[(6 * a.pmax + q) * kTile];
          } else {
            xj[0] = xj[1] = xj[2] = 0.0;
            nj[0] = nj[1] = nj[2] = 0.0;
            wj = 0.0;
          }
          double inner = 0.0;
          for (int p = 0; p < npi; ++p) {
            double xi[3], ni[3];
            xi[0] = ib[(0 * a.pmax + p) * kTile];
            xi[1] = ib[(1 * a.pmax + p) * kTile];
            xi[2] = ib[(2 * a.pmax + p) * kTile];
            ni[0] = ib[(3 * a.pmax + p) * kTile];
            ni[1] = ib[(4 * a.pmax + p) * kTile];
            ni[2] = ib[(5 * a.pmax + p) * kTile];
            const double wi = ib[(6 * a.pmax + p) * kTile];
            const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
            const double r2 = (rx * rx + ry * ry) + rz * rz;
            double K = lq ? k_fast<DIM3>(rx, ry, rz, r2, ni, nj) : 0.0;
            n_pp += lq ? 1 : 0;
            if (OCC) {
              uint8_t lg = 0;
              if (DIM3) {
                RayD R;
                bool cast = (K > 0.0) && (sw ? make_ray(xj, -rx, -ry, -rz, r2, R) : make_ray(xi, rx, ry, rz, r2, R));
                n_rays += cast ? 1 : 0;
                bool blocked = packet_any_hit(
                    cast, nodes, a.n_nodes, [&](const NodeD& nd) { return slab_d(nd, R); },
                    [&](int k, bool test) {
                      const TriD tr = a.tris[k];
                      if (!test || tr.group == gi || tr.group == gj) return false;
                      ++tc.prims;
                      return mt_d(tr, R);
                    },
                    tc);
                if (cast) lg = blocked ? 2 : 1;
                if (blocked) K = 0.0;
              } else {
                bool cast = K > 0.0;
                n_rays += cast ? 1 : 0;
                const double rxlo = fmin(xi[0], xj[0]), rxhi = fmax(xi[0], xj[0]);
                const double rylo = fmin(xi[1], xj[1]), ryhi = fmax(xi[1], xj[1]);
                bool blocked = packet_any_hit(
                    cast, nodes, a.n_nodes,
                    [&](const NodeD& nd) {
                      return !(nd.lo[0] > rxhi || nd.hi[0] < rxlo || nd.lo[1] > ryhi || nd.hi[1] < rylo);
                    },
                    [&](int k, bool test) {
                      const SegD sg = a.segs[k];
                      if (!test || sg.group == gi || sg.group == gj) return false;
                      ++tc.prims;
                      return sw ? seg_blocks(sg, xj, xi) : seg_blocks(sg, xi, xj);
                    },
                    tc);
                if (cast) lg = blocked ? 2 : 1;
                if (blocked) K = 0.0;
              }
              if (logp && lq) logp[sw ? q * a.log_pm + p : p * a.log_pm + q] = lg;
            }
            inner = fma(wi, K, inner);
          }
          acc = fma(wj, inner, acc);
        }
        // F[i,j] = raw/A_i and F[j,i] = raw/A_j in the caller's element order
        if (valid) {
          a.F[oi + oj * N] = acc / a.area[i];
          a.F[oj + oi * N] = acc / a.area[j];
        } else if (j == i) {
          a.F[oi + oi * N] = 0.0 / a.area[i];
        }
      }
    }
    __syncthreads();
  }
  // counters (one atomic per warp)
  n_rays = warp_sum_u64(n_rays);
  n_pp = warp_sum_u64(n_pp);
  tc.nodes = warp_sum_u64(tc.nodes);
  tc.prims = warp_sum_u64(tc.prims);
  if (lane == 0 && a.counters) {
    atomicAdd(a.counters + 0, n_pp);
    atomicAdd(a.counters + 1, n_rays);
    atomicAdd(a.counters + 2, tc.nodes);
    atomicAdd(a.counters + 3, tc.prims);
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

size_t pair_smem_bytes(int pmax, int n_nodes_smem) {
  return (size_t)kComp * pmax * kTile * sizeof(double) + (size_t)n_nodes_smem * sizeof(NodeD) + 16;
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
  const size_t smem = pair_smem_bytes(a.pmax, a.nodes_in_smem ? a.n_nodes : 0);
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
