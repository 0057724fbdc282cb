// kernels_wave.cu -- the wavefront pair pipeline with occlusion.
//
// Replaces _vf_pair_kernel! (src/GPUKernels.jl:226-323) with its shadow rays
// (src/GPUKernels.jl:289-304, gpu_intersect_bvh src/GPUBVH.jl:202-285) when
// the mesh has obstructions.  One chunk of the upper-triangle tiles runs as
//   1. generation: the quadrature of every pair (tile-staged as in the fused
//      kernel).  A ray that misses the root box is visible and its term is
//      summed at once; every other ray is appended to a global ray queue as
//      (pending-pair slot, p, q, swapped), and its pair gets a slot holding
//      (i, j, sum of the immediate terms).  Pairs without queued rays write F.
//   2. pair lists (3-D triangles): one warp per pending pair finds the
//      triangles any ray of the pair can hit (k_plist, below).
//   3. traversal: one queued ray per lane, 32 rays per warp traced together,
//      each against its pair's list or by a walk of the tree
//      (device_trace.cuh), at the occupancy a traversal-only kernel allows.
//      Each visible ray sets its (p, q) bit in its slot's visibility words
//      with an integer atomicOr -- order-independent, hence deterministic.
//   4. resolve: per pending pair, the terms of the visible queued rays are
//      formed again with the generation's arithmetic and added, in (p, q)
//      order, to the immediate sum; F[i,j] and F[j,i] are written.
// Mixed precision adds an FP32 queue: FP32 rays whose certified traversal is
// uncertain are appended to the FP64 queue, which is traced after it.
//
// Queue capacity is reserved per tile for the worst case (every point pair
// queued) when a block claims the tile and released down to the actual use
// when the tile ends, so a chunk never overflows; the host runs chunks until
// every tile is claimed.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_lists.cuh"
#include "device_trace.cuh"
#include "kernels.h"

namespace rvf {

namespace {

// ray record: q (6 bits), p (6 bits), swapped (1 bit), slot
__device__ __forceinline__ uint64_t rec_make(int64_t slot, bool sw, int p, int q) {
  return ((uint64_t)slot << 13) | ((uint64_t)sw << 12) | ((uint64_t)p << 6) | (uint64_t)q;
}
__device__ __forceinline__ int64_t rec_slot(uint64_t r) { return (int64_t)(r >> 13); }
__device__ __forceinline__ bool rec_sw(uint64_t r) { return ((r >> 12) & 1u) != 0; }
__device__ __forceinline__ int rec_p(uint64_t r) { return (int)((r >> 6) & 63u); }
__device__ __forceinline__ int rec_q(uint64_t r) { return (int)(r & 63u); }

// (element e, component c, point p) in a tile-blocked table
__device__ __forceinline__ int64_t tab_at(int64_t e, int c, int p, int pm) {
  return ((e >> 5) * kComp + c) * (int64_t)pm * kTile + (int64_t)p * kTile + (e & 31);
}

__device__ __forceinline__ unsigned long long neg(unsigned long long v) { return ~v + 1ull; }

// Per-warp staging of queue records in shared memory.
__device__ __forceinline__ void stage_push(uint64_t* st, int& n, bool push, uint64_t rec) {
  const uint32_t m = __ballot_sync(kFull, push);
  if (m == 0) return;
  if (push) st[n + __popc(m & lanemask_lt())] = rec;
  n += __popc(m);
  __syncwarp();
}

// Appends the first k (<= 32) staged records to the queue; keeps the rest.
__device__ __forceinline__ void stage_flush(uint64_t* st, int& n, int k, uint64_t* queue,
                                            unsigned long long* count, unsigned long long* tile_used) {
  const int lane = threadIdx.x & 31;
  unsigned long long base = 0;
  if (lane == 0) {
    base = atomicAdd(count, (unsigned long long)k);
    atomicAdd(tile_used, (unsigned long long)k);
  }
  base = __shfl_sync(kFull, base, 0);
  if (lane < k) queue[base + lane] = st[lane];
  const int rest = n - k;
  const uint64_t v = (lane < rest) ? st[k + lane] : 0;
  __syncwarp();
  if (lane < rest) st[lane] = v;
  n = rest;
  __syncwarp();
}

// Per-lane runs of queue records.  Each lane collects the deferred rays of
// its own pair in a ring of kRun records in shared memory (entry k of thread t
// at ring[k * 256 + t]) and appends it to the queue as one contiguous run when
// it is full and when the pair ends.  A traversal warp takes 32 consecutive
// records, so its rays come from one or two pairs -- thin bundles whose walks
// agree -- instead of one ray from each of 32 pairs.
constexpr int kRun = 16;     // FP64 generation: 32 would cost a third of its occupancy
constexpr int kRunMix = 32;  // mixed generation (two blocks per SM anyway): one pair per traversal warp

__device__ __forceinline__ void run_push(uint64_t* ring, int& nr, bool push, uint64_t rec) {
  if (push) {
    ring[nr * 256] = rec;
    ++nr;
  }
}

// Appends the full runs (all runs when `all`) of the warp's lanes, lane by
// lane, with one counter update.  Warp-uniform call.
template <int RUN>
__device__ __forceinline__ void run_flush(uint64_t* ring, int& nr, bool all, uint64_t* queue,
                                          unsigned long long* count, unsigned long long* tile_used) {
  const int lane = threadIdx.x & 31;
  const int mine = (all || nr == RUN) ? nr : 0;
  int incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  unsigned long long base = 0;
  if (lane == 0) {
    base = atomicAdd(count, (unsigned long long)total);
    atomicAdd(tile_used, (unsigned long long)total);
  }
  base = __shfl_sync(kFull, base, 0);
  uint64_t* dst = queue + base + (incl - mine);
  for (int k = 0; k < mine; ++k) dst[k] = ring[k * 256];
  if (mine > 0) nr = 0;
}

// Gives lanes with `need` a fresh pending-pair slot and clears its visibility words.
__device__ __forceinline__ void slot_alloc(const WaveQ& q, bool need, int64_t& slot, unsigned long long* tile_slots) {
  const uint32_t m = __ballot_sync(kFull, need);
  if (m == 0) return;
  const int lane = threadIdx.x & 31;
  unsigned long long base = 0;
  if (lane == 0) {
    base = atomicAdd(q.ctr + kCtrSlots, (unsigned long long)__popc(m));
    atomicAdd(tile_slots, (unsigned long long)__popc(m));
  }
  base = __shfl_sync(kFull, base, 0);
  if (need) {
    slot = (int64_t)base + __popc(m & lanemask_lt());
    for (int w = 0; w < q.vis_words; ++w) q.vis[slot * q.vis_words + w] = 0ull;
  }
}

// Queue reservations: records in the low 38 bits, pending-pair slots above,
// in one counter, so that a claim checks and takes both capacities at once.
__device__ __forceinline__ unsigned long long resv_pack(unsigned long long recs, unsigned long long slots) {
  return recs | (slots << 38);
}

// Gives back part of a reservation (never more than was taken).
__device__ __forceinline__ void resv_release(const WaveQ& q, unsigned long long recs, unsigned long long slots) {
  atomicAdd(q.ctr + kCtrResv, neg(resv_pack(recs, slots)));
}

// Block-level tile claim with worst-case queue reservation.  Returns the
// tile, or -1 when the chunk's queues have no room for another tile or every
// tile is claimed.  The reservation is a compare-and-swap that only succeeds
// when both capacities hold, so concurrent claims never over-reserve; the
// retry loop is bounded (a block that keeps losing the race ends its chunk
// and raises kErrClaimGaveUp, which the host turns into RVF_ETIMEDOUT only
// when a whole chunk claimed nothing).
__device__ __forceinline__ int64_t claim_tile(const WaveQ& q, int64_t n_tiles, bool occ,
                                              unsigned long long need, unsigned long long need_s, int retries,
                                              int* err) {
  if (occ) {
    unsigned long long* c = q.ctr + kCtrResv;
    unsigned long long cur = *(volatile unsigned long long*)c;
    bool ok = false, full = false;
    for (int it = 0; it < retries; ++it) {
      const unsigned long long recs = cur & ((1ull << 38) - 1), slots = cur >> 38;
      if (recs + need > (unsigned long long)q.cap || slots + need_s > (unsigned long long)q.scap) {
        full = true;
        break;
      }
      const unsigned long long prev = atomicCAS(c, cur, cur + resv_pack(need, need_s));
      if (prev == cur) {
        ok = true;
        break;
      }
      cur = prev;
    }
    if (!ok) {
      if (!full) atomicOr(err, kErrClaimGaveUp);
      return -1;
    }
  }
  const int64_t t = (int64_t)atomicAdd(q.ctr + kCtrTile, 1ull);
  if (t >= n_tiles) {
    if (occ) resv_release(q, need, need_s);
    return -1;
  }
  return t;
}

// True when every segment between a point of element i and a point of
// element j certainly misses the box: each such segment stays within
// R = max(rad_i, rad_j) of the centroid segment (convexity), so it suffices
// that the centroid segment misses the box grown by R plus a margin that
// dwarfs every rounding error of the reference's slab test.  2-D uses x, y.
template <bool DIM3>
__device__ __forceinline__ bool pair_misses_box(const double* ci, const double* cj, double R, const NodeD& nd) {
  double te = 0.0, tx = 1.0;
#pragma unroll
  for (int c = 0; c < (DIM3 ? 3 : 2); ++c) {
    const double lo = nd.lo[c] - R, hi = nd.hi[c] + R;
    const double d = cj[c] - ci[c];
    if (d == 0.0) {
      if (ci[c] < lo || ci[c] > hi) return true;
      continue;
    }
    const double inv = 1.0 / d;
    const double t1 = (lo - ci[c]) * inv, t2 = (hi - ci[c]) * inv;
    te = fmax(te, fmin(t1, t2));
    tx = fmin(tx, fmax(t1, t2));
  }
  return te > tx;
}

// bytes of one tile block of the quadrature table in shared memory (a
// multiple of 128: kComp * pmax * 32 elements of 4 or 8 bytes)
__host__ __device__ __forceinline__ size_t gen_tab_bytes(bool mixed, int pmax) {
  return (size_t)kComp * pmax * kTile * (mixed ? sizeof(float) : sizeof(double));
}

// request r of the launch with tile_base[r] <= t < tile_base[r+1]
__device__ __forceinline__ int find_req(const int64_t* tile_base, int n_req, int64_t t) {
  int lo = 0, hi = n_req - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_base[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace

// ---------------------------------------------------------------------------
// 1a. Generation of a tile without shadow-ray work (the tile classification
// found no pair whose rays may be blocked, or the mesh has no obstruction):
// the quadrature alone, register-blocked.  Lane l owns destination
// j = 32 bj + l and holds QB of its points in registers; the warp walks the
// source element's points p, read once per QB point pairs from the staged
// block in shared memory (broadcast), so each point pair costs the kernel's
// arithmetic and about 7/QB shared loads.  Sums run in the pipeline's order
// (over p inside, then w_q * inner over q), so an FP64 fast tile is bit for
// bit what the ray pipeline gives for pairs whose rays are all visible.
// Out of line: their registers are allocated apart from the ray pipeline's.
// ---------------------------------------------------------------------------
template <bool DIM3, bool OCC, int QB>
__device__ __forceinline__ void gen_fast_fp64_body(const PairArgs& a, const double* iblk, int64_t bi, int64_t bj,
                                                   int li0, int lane, uint32_t& n_pp, uint32_t& n_rays) {
  const int64_t N = a.N;
  const int pm = a.pmax;
  const int64_t j = bj * kTile + lane;
  const bool jok = j < N;
  const int64_t oj = jok ? (a.orig ? (int64_t)a.orig[j] : j) : 0;
  const int npj0 = jok ? a.np[j] : 0;
  const double* jb = a.tab + bj * kComp * pm * kTile + lane;
  // li0 < 8: the warp's rows li0, li0 + 8, ...; li0 >= 8: the single row li0 - 8
  const int r_last = li0 < 8 ? kTile / 8 : 1;
  for (int rr = 0; rr < r_last; ++rr) {
    const int li = li0 < 8 ? li0 + 8 * rr : li0 - 8;
    const int64_t i = bi * kTile + li;
    if (i >= N) break;  // warp-uniform; later rows are further out
    const bool valid = jok && i < j;
    const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
    const int npi = a.np[i];
    int npj = valid ? npj0 : 0;
    if (valid && a.flat[i] && a.flat[j] && a.nrm[3 * i] == a.nrm[3 * j] && a.nrm[3 * i + 1] == a.nrm[3 * j + 1] &&
        a.nrm[3 * i + 2] == a.nrm[3 * j + 2])
      npj = 0;
    const int qmax = __reduce_max_sync(kFull, npj);
    const double* ib = iblk + li;
    double acc = 0.0;
    for (int q0 = 0; q0 < qmax; q0 += QB) {
      double xq[QB][3], nq[QB][3], wq[QB];
#pragma unroll
      for (int u = 0; u < QB; ++u) {
        const int q = q0 + u;
        const bool lq = q < npj;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          xq[u][c] = lq ? jb[(c * pm + q) * kTile] : 0.0;
          nq[u][c] = lq ? jb[((3 + c) * pm + q) * kTile] : 0.0;
        }
        wq[u] = lq ? jb[(6 * pm + q) * kTile] : 0.0;
      }
      double inner[QB];
#pragma unroll
      for (int u = 0; u < QB; ++u) inner[u] = 0.0;
      // k_fast with its grazing branch taken out of the loop: a lane that
      // meets a grazing point pair (either |cos| within 1e-5 of zero) forms
      // the chunk again below with k_fast's own arithmetic
      bool graze = false;
      uint32_t cast = 0;
      const int ulim = npj - q0;
      for (int p = 0; p < npi; ++p) {
        double xi[3], ni[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          xi[c] = ib[(c * pm + p) * kTile];
          ni[c] = ib[((3 + c) * pm + p) * kTile];
        }
        const double wi = ib[(6 * pm + p) * kTile];
        // straight-line over the block: a point q0 + u >= npj has zero
        // normal and weight, so its dj is -0 and its K zero (it only must not
        // ask for the grazing redo)
#pragma unroll
        for (int u = 0; u < QB; ++u) {
          const double rx = xq[u][0] - xi[0], ry = xq[u][1] - xi[1], rz = xq[u][2] - xi[2];
          const double r2 = (rx * rx + ry * ry) + rz * rz;
          const double di = fma(ni[0], rx, fma(ni[1], ry, ni[2] * rz));
          const double dj = -fma(nq[u][0], rx, fma(nq[u][1], ry, nq[u][2] * rz));
          const double thr = 1e-10 * r2;
          const bool big = !(r2 < 1e-30);
          graze = graze || (u < ulim && big && (di * di <= thr || dj * dj <= thr));
          double K = 0.0;
          if (big && di > 0.0 && dj > 0.0)
            K = DIM3 ? (di * dj) * rcp_nr(kPiD * (r2 * r2)) : (di * dj) * rcp_nr(2.0 * (r2 * sqrt(r2)));
          cast += K > 0.0 ? 1 : 0;
          inner[u] = fma(wi, K, inner[u]);
        }
      }
      if (__any_sync(kFull, graze) && graze) {  // rare: the chunk again, exactly as the ray pipeline forms it
        cast = 0;
#pragma unroll
        for (int u = 0; u < QB; ++u) inner[u] = 0.0;
        for (int p = 0; p < npi; ++p) {
          double xi[3], ni[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            xi[c] = ib[(c * pm + p) * kTile];
            ni[c] = ib[((3 + c) * pm + p) * kTile];
          }
          const double wi = ib[(6 * pm + p) * kTile];
#pragma unroll
          for (int u = 0; u < QB; ++u) {
            if (q0 + u < npj) {
              const double rx = xq[u][0] - xi[0], ry = xq[u][1] - xi[1], rz = xq[u][2] - xi[2];
              const double r2 = (rx * rx + ry * ry) + rz * rz;
              // k_fast, with the reference formula in line
              double K = 0.0;
              if (!(r2 < 1e-30)) {
                const double di = fma(ni[0], rx, fma(ni[1], ry, ni[2] * rz));
                const double dj = -fma(nq[u][0], rx, fma(nq[u][1], ry, nq[u][2] * rz));
                const double thr = 1e-10 * r2;
                if (di * di <= thr || dj * dj <= thr) K = k_reference_inl<DIM3>(rx, ry, rz, r2, ni, nq[u]);
                else if (di > 0.0 && dj > 0.0)
                  K = DIM3 ? (di * dj) * rcp_nr(kPiD * (r2 * r2)) : (di * dj) * rcp_nr(2.0 * (r2 * sqrt(r2)));
              }
              cast += K > 0.0 ? 1 : 0;
              inner[u] = fma(wi, K, inner[u]);
            }
          }
        }
      }
      if (OCC) n_rays += cast;
#pragma unroll
      for (int u = 0; u < QB; ++u)
        if (q0 + u < npj) acc = fma(wq[u], inner[u], acc);
    }
    n_pp += (uint32_t)(npi * npj);
    if (valid) {
      a.F[oi + oj * N] = acc / a.area[i];
      a.F[oj + oi * N] = acc / a.area[j];
    } else if (j == i) {
      a.F[oi + oi * N] = 0.0 / a.area[i];
    }
  }
}

// Mixed precision: the FP32 far-field arithmetic of k_gen_mixed (offsets
// from the element centroids, FP32 per-pair sums), for tiles with neither
// near-field nor nearly coincident pairs.  Grazing point pairs stay in FP32
// here: no ray depends on the sign of their K, and their FP32 error is that
// of any other far-field term.
template <bool OCC, int QB>
__device__ __forceinline__ void gen_fast_mixed_body(const MixedArgs& a, const float* iblk, int64_t bi, int64_t bj,
                                                    int li0, int lane, uint32_t& n_pp, uint32_t& n_rays) {
  const int64_t N = a.N;
  const int pm = a.pmax;
  const int64_t j = bj * kTile + lane;
  const bool jok = j < N;
  const int64_t oj = jok ? (a.orig ? (int64_t)a.orig[j] : j) : 0;
  const int npj0 = jok ? a.np[j] : 0;
  const float* jbf = a.tabf + bj * kComp * pm * kTile + lane;
  const double cj0 = jok ? a.cen[3 * j] : 0.0, cj1 = jok ? a.cen[3 * j + 1] : 0.0, cj2 = jok ? a.cen[3 * j + 2] : 0.0;
  // li0 < 8: the warp's rows li0, li0 + 8, ...; li0 >= 8: the single row li0 - 8
  const int r_last = li0 < 8 ? kTile / 8 : 1;
  for (int rr = 0; rr < r_last; ++rr) {
    const int li = li0 < 8 ? li0 + 8 * rr : li0 - 8;
    const int64_t i = bi * kTile + li;
    if (i >= N) break;  // warp-uniform
    const bool valid = jok && i < j;
    const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
    const int npi = a.np[i];
    int npj = valid ? npj0 : 0;
    if (valid && a.flat[i] && a.flat[j] && a.nrm[3 * i] == a.nrm[3 * j] && a.nrm[3 * i + 1] == a.nrm[3 * j + 1] &&
        a.nrm[3 * i + 2] == a.nrm[3 * j + 2])
      npj = 0;
    const int qmax = __reduce_max_sync(kFull, npj);
    const float d0 = (float)(cj0 - a.cen[3 * i]), d1 = (float)(cj1 - a.cen[3 * i + 1]),
                d2 = (float)(cj2 - a.cen[3 * i + 2]);
    const float* ibf = iblk + li;
    float acc32 = 0.0f;
    uint32_t cast = 0;
    for (int q0 = 0; q0 < qmax; q0 += QB) {
      float oq[QB][3], nq[QB][3], wq[QB];
#pragma unroll
      for (int u = 0; u < QB; ++u) {
        const int q = q0 + u;
        const bool lq = q < npj;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          oq[u][c] = lq ? jbf[(c * pm + q) * kTile] : 0.0f;
          nq[u][c] = lq ? jbf[((3 + c) * pm + q) * kTile] : 0.0f;
        }
        wq[u] = lq ? jbf[(6 * pm + q) * kTile] : 0.0f;
      }
      float inner[QB];
#pragma unroll
      for (int u = 0; u < QB; ++u) inner[u] = 0.0f;
      for (int p = 0; p < npi; ++p) {
        const float op0 = ibf[(0 * pm + p) * kTile], op1 = ibf[(1 * pm + p) * kTile], op2 = ibf[(2 * pm + p) * kTile];
        const float np0 = ibf[(3 * pm + p) * kTile], np1 = ibf[(4 * pm + p) * kTile], np2 = ibf[(5 * pm + p) * kTile];
        const float wp = ibf[(6 * pm + p) * kTile];
        // straight-line over the block: a point q0 + u >= npj has zero
        // normal, so its dj is -0 and its K zero
#pragma unroll
        for (int u = 0; u < QB; ++u) {
          const float rx = d0 + (oq[u][0] - op0), ry = d1 + (oq[u][1] - op1), rz = d2 + (oq[u][2] - op2);
          const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
          const float di = fmaf(np0, rx, fmaf(np1, ry, np2 * rz));
          const float dj = -fmaf(nq[u][0], rx, fmaf(nq[u][1], ry, nq[u][2] * rz));
          const float K32 = (di > 0.0f && dj > 0.0f) ? (di * dj) * rcp_approx(3.14159265f * (r2 * r2)) : 0.0f;
          cast += K32 > 0.0f ? 1 : 0;
          inner[u] = fmaf(wp, K32, inner[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < QB; ++u)
        if (q0 + u < npj) acc32 = fmaf(wq[u], inner[u], acc32);
    }
    if (OCC) n_rays += cast;
    n_pp += (uint32_t)(npi * npj);
    const double raw = 0.0 + (double)acc32;
    if (valid) {
      a.F[oi + oj * N] = raw / a.area[i];
      a.F[oj + oi * N] = raw / a.area[j];
    } else if (j == i) {
      a.F[oi + oi * N] = 0.0 / a.area[i];
    }
  }
}

// Out of line inside the chunked generation kernels, whose own registers are
// allocated for the ray pipeline.
template <bool DIM3, bool OCC, int QB>
__device__ __noinline__ void gen_fast_fp64(const PairArgs& a, const double* iblk, int64_t bi, int64_t bj, int li0,
                                           int lane, uint32_t& n_pp, uint32_t& n_rays) {
  gen_fast_fp64_body<DIM3, OCC, QB>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
}
template <bool OCC, int QB>
__device__ __noinline__ void gen_fast_mixed(const MixedArgs& a, const float* iblk, int64_t bi, int64_t bj, int li0,
                                            int lane, uint32_t& n_pp, uint32_t& n_rays) {
  gen_fast_mixed_body<OCC, QB>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
}

// The fast loop with the point block for the rule's size (li0 as there).
template <bool DIM3, bool OCC>
__device__ __forceinline__ void fast_fp64(const PairArgs& a, const double* iblk, int64_t bi, int64_t bj, int li0,
                                          int lane, uint32_t& n_pp, uint32_t& n_rays) {
  if (a.pmax <= 3) gen_fast_fp64<DIM3, OCC, 3>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
  else gen_fast_fp64<DIM3, OCC, 4>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
}
template <bool OCC>
__device__ __forceinline__ void fast_mixed(const MixedArgs& a, const float* iblk, int64_t bi, int64_t bj, int li0,
                                           int lane, uint32_t& n_pp, uint32_t& n_rays) {
  const int pm = a.pmax;
  if (pm == 7 || pm == 13 || pm == 49) gen_fast_mixed<OCC, 7>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
  else if (pm == 5 || pm == 25) gen_fast_mixed<OCC, 5>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
  else if (pm == 3 || pm == 9) gen_fast_mixed<OCC, 3>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
  else gen_fast_mixed<OCC, 8>(a, iblk, bi, bj, li0, lane, n_pp, n_rays);
}

// Tile class of request-local tile t (kernels_cull.cu) and the mask words of
// its rows in shared memory; without classes every pair keeps its rays.
__device__ __forceinline__ uint8_t load_tile_class(const uint8_t* tcls, const uint32_t* tmask, int64_t t,
                                                   uint32_t* s_mask) {
  const uint8_t cls = tcls ? tcls[t] : (uint8_t)kClsSlow;
  if (threadIdx.x < kTile)
    s_mask[threadIdx.x] = !tcls ? 0xffffffffu : (cls & kClsSlow) ? tmask[t * kTile + threadIdx.x] : 0u;
  return cls;
}

// ---------------------------------------------------------------------------
// 1. Generation, FP64 (surfaces and curves).
// ---------------------------------------------------------------------------
template <bool DIM3, bool OCC>
__global__ void __launch_bounds__(256, 2) k_gen_fp64(const GenBatch* __restrict__ Lp) {
  extern __shared__ __align__(128) unsigned char smem[];
  const GenBatch& L = *Lp;
  const int pmL = L.pmax_max;
  double* iblk = reinterpret_cast<double*>(smem);
  uint64_t* ring = reinterpret_cast<uint64_t*>(iblk + kComp * pmL * kTile) + threadIdx.x;
  uint64_t* bar = reinterpret_cast<uint64_t*>(iblk + kComp * pmL * kTile) + (OCC ? kRun * 256 : 0);
  __shared__ int64_t s_tile;
  __shared__ int s_req;
  __shared__ unsigned long long s_used, s_slots;
  __shared__ NodeD s_root;  // the request's root box: the only node the generation tests
  __shared__ uint32_t s_mask[kTile];  // pairs of the tile whose rays may be blocked (row -> lanes)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();

  const WaveQ& Q = L.q;
  const unsigned long long need = (unsigned long long)kTile * kTile * pmL * pmL, need_s = kTile * kTile;
  uint32_t phase = 0;
  uint32_t n_rays = 0, n_pp = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const int64_t g = claim_tile(Q, L.total_tiles, OCC, need, need_s, L.claim_retries, L.err);
      s_used = 0;
      s_slots = 0;
      s_tile = -1;
      if (g >= 0) {
        const int r = find_req(L.tile_base, L.n_req, g);
        const PairArgs& a = L.reqs[r];
        s_req = r;
        s_tile = g - L.tile_base[r] + a.tile0;
        if (a.work) s_tile = a.work[s_tile];
        if (OCC) s_root = a.nodes[0];
        int64_t bi, bj;
        tile_coords(s_tile, a.nT, bi, bj);
        const uint32_t blk_bytes = (uint32_t)(kComp * a.pmax * kTile * sizeof(double));
        mbar_expect_tx(bar, blk_bytes);
        bulk_g2s(iblk, a.tab + bi * kComp * a.pmax * kTile, blk_bytes, bar);
      }
    }
    __syncthreads();
    const int64_t t = s_tile;
    if (t < 0) break;
    const int req = s_req;
    const PairArgs& a = L.reqs[req];
    const int pm = a.pmax;
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const uint8_t cls = load_tile_class(a.tcls, a.tmask, t, s_mask);
    const bool ok = mbar_wait_bounded(bar, phase);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(L.err, kErrWaitTimeout);
        if (OCC) resv_release(Q, need, need_s);  // give the whole reservation back
      }
      break;
    }
    phase ^= 1u;

    if (a.tcls && !(cls & kClsSlow) && !a.ray_log) {  // block-uniform: no ray of the tile can be blocked
      if (!a.fast_done) fast_fp64<DIM3, OCC>(a, iblk, bi, bj, warp, lane, n_pp, n_rays);
      __syncthreads();
      if (OCC && threadIdx.x == 0) resv_release(Q, need, need_s);
      continue;
    }
    const int64_t N = a.N;
    const int64_t j = bj * kTile + lane;
    const int64_t oj = (j < N) ? (a.orig ? (int64_t)a.orig[j] : j) : 0;
    const double* jb = a.tab + bj * kComp * pm * kTile + lane;
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int li = warp + 8 * rr;
      const int64_t i = bi * kTile + li;
      if (i >= N) continue;  // warp-uniform
      if (a.tcls && !a.ray_log && s_mask[li] == 0u) {  // no ray of this row can be blocked
        fast_fp64<DIM3, OCC>(a, iblk, bi, bj, li + 8, lane, n_pp, n_rays);
        continue;
      }
      const bool valid = (j < N) && (i < j);
      const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
      const bool sw = valid && oi > oj;  // the reference casts from the lower caller index
      const int npi = a.np[i];
      int npj = valid ? a.np[j] : 0;
      // Two elements whose points all share one normal, bit for bit, have
      // cos_j = -cos_i exactly at every point pair: K = 0, no rays.
      if (valid && a.flat[i] && a.flat[j] && a.nrm[3 * i] == a.nrm[3 * j] &&
          a.nrm[3 * i + 1] == a.nrm[3 * j + 1] && a.nrm[3 * i + 2] == a.nrm[3 * j + 2])
        npj = 0;
      const int qmax = __reduce_max_sync(kFull, npj);
      const double* ib = iblk + li;
      uint8_t* logp = (a.ray_log && valid)
                          ? a.ray_log + ((uint64_t)(sw ? oj : oi) * N + (sw ? oi : oj)) * a.log_pm * a.log_pm
                          : nullptr;
      // pairs whose rays all certainly miss the root box need no ray at all
      const bool cullp = OCC && npj > 0 &&
                         (!((s_mask[li] >> lane) & 1u) ||
                          (a.rad && pair_misses_box<DIM3>(a.cen + 3 * i, a.cen + 3 * j,
                                                          fmax(a.rad[i], a.rad[j]) + a.cull_margin, s_root)));
      double acc = 0.0;
      int64_t slot = -1;
      int nr = 0;
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
            const NodeD& root = s_root;
            if (cullp) {
              cast = (K > 0.0) && (!DIM3 || sqrt(r2) > 1e-15);  // make_ray's cast rule
            } else if (DIM3) {
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
            if (__any_sync(kFull, defer)) {
              slot_alloc(Q, defer && slot < 0, slot, &s_slots);
              run_push(ring, nr, defer, rec_make(slot, sw, p, q));
              if (__any_sync(kFull, nr == kRun))
                run_flush<kRun>(ring, nr, false, Q.rec64, Q.ctr + kCtrRec64, &s_used);
              if (defer) K = 0.0;
            }
          }
          inner = fma(wi, K, inner);
        }
        acc = fma(wj, inner, acc);
      }
      if (OCC && __any_sync(kFull, nr > 0)) run_flush<kRun>(ring, nr, true, Q.rec64, Q.ctr + kCtrRec64, &s_used);
      if (slot >= 0) {
        PendSlot ps;
        ps.i = (int32_t)i;
        ps.j = (int32_t)j;
        ps.req = req;
        ps.pad = 0;
        ps.acc = acc;
        Q.slots[slot] = ps;
      } else if (valid) {
        // F[i,j] = raw/A_i and F[j,i] = raw/A_j in the caller's element order
        a.F[oi + oj * N] = acc / a.area[i];
        a.F[oj + oi * N] = acc / a.area[j];
      } else if (j == i) {
        a.F[oi + oi * N] = 0.0 / a.area[i];
      }
    }
    __syncthreads();
    if (OCC && threadIdx.x == 0) resv_release(Q, need - s_used, need_s - s_slots);  // keep what the tile used
  }
  const uint64_t s_rays = warp_sum_u64(n_rays), s_pp = warp_sum_u64(n_pp);
  if (lane == 0 && L.counters) {
    atomicAdd(L.counters + 0, s_pp);
    atomicAdd(L.counters + 1, s_rays);
  }
}

// ---------------------------------------------------------------------------
// 1'. Generation, mixed precision (surfaces).
// ---------------------------------------------------------------------------

// FP64 point pair of the mixed generation (near field, grazing, or an FP32
// direction unusable for the certified traversal): the reference's K when
// exactK, the FP32 term otherwise, and the reference's ray.
template <bool OCC>
__device__ __noinline__ void gen_mixed64(const MixedArgs& a, const NodeD* nodes, const double* it64,
                                         const double* jb64, int p, int q, bool need64, bool exactK_in, bool graze,
                                         bool sw, bool cullp, double contrib32, uint8_t* logp, bool& defer64,
                                         double& accd,
                                         uint32_t& n_rays, uint32_t& n_rays64, uint32_t& n_graze) {
  const int pm = a.pmax;
  double xi[3], ni[3];
  xi[0] = it64[(0 * pm + p) * kTile]; xi[1] = it64[(1 * pm + p) * kTile]; xi[2] = it64[(2 * pm + p) * kTile];
  ni[0] = it64[(3 * pm + p) * kTile]; ni[1] = it64[(4 * pm + p) * kTile]; ni[2] = it64[(5 * pm + p) * kTile];
  const double wi64 = it64[(6 * pm + p) * kTile];
  double xj[3] = {0.0, 0.0, 0.0}, nj[3] = {0.0, 0.0, 0.0}, wj64 = 0.0;
  if (need64) {
    xj[0] = jb64[(0 * pm + q) * kTile]; xj[1] = jb64[(1 * pm + q) * kTile]; xj[2] = jb64[(2 * pm + q) * kTile];
    nj[0] = jb64[(3 * pm + q) * kTile]; nj[1] = jb64[(4 * pm + q) * kTile]; nj[2] = jb64[(5 * pm + q) * kTile];
    wj64 = jb64[(6 * pm + q) * kTile];
  }
  const double rx64 = xj[0] - xi[0], ry64 = xj[1] - xi[1], rz64 = xj[2] - xi[2];
  const double r264 = (rx64 * rx64 + ry64 * ry64) + rz64 * rz64;
  const bool exactK = need64 && exactK_in;
  const double K64 = exactK ? k_fast<true>(rx64, ry64, rz64, r264, ni, nj) : 0.0;
  n_graze += (exactK && graze) ? 1 : 0;
  const double contrib64 = exactK ? wj64 * (wi64 * K64) : contrib32;
  bool cast64 = false;
  defer64 = false;
  if (OCC && need64 && (!exactK || K64 > 0.0)) {
    if (cullp) {
      cast64 = sqrt(r264) > 1e-15;  // make_ray's cast rule; the ray certainly misses the root
    } else {
      RayD R64;
      cast64 = sw ? make_ray(xj, -rx64, -ry64, -rz64, r264, R64) : make_ray(xi, rx64, ry64, rz64, r264, R64);
      if (cast64) defer64 = slab_d(nodes[0], R64);
    }
    if (cast64 && !defer64 && logp) logp[sw ? q * a.log_pm + p : p * a.log_pm + q] = 1;
  }
  n_rays64 += cast64 ? 1 : 0;
  n_rays += (cast64 && exactK) ? 1 : 0;
  if (need64 && !defer64) accd += contrib64;
}

template <bool OCC>
__global__ void __launch_bounds__(256, 2) k_gen_mixed(const GenBatch* __restrict__ Lp) {
  extern __shared__ __align__(128) unsigned char smem[];
  const GenBatch& L = *Lp;
  const int pmL = L.pmax_max;
  float* iblk = reinterpret_cast<float*>(smem);
  // FP32 rays: per-lane runs; FP64 rays (near field, grazing, unusable
  // directions, a few per cent): per-warp staging
  uint64_t* stage_all = reinterpret_cast<uint64_t*>(smem + gen_tab_bytes(true, pmL));
  uint64_t* ring = stage_all + (OCC ? 8 * 64 : 0) + threadIdx.x;
  uint64_t* bar = stage_all + (OCC ? 8 * 64 + kRunMix * 256 : 0);
  __shared__ int64_t s_tile;
  __shared__ int s_req;
  __shared__ unsigned long long s_used, s_slots;
  __shared__ NodeF s_rootf;  // the request's root box, FP32 and FP64
  __shared__ NodeD s_root;
  __shared__ uint32_t s_mask[kTile];  // pairs of the tile whose rays may be blocked (row -> lanes)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* st64 = stage_all + warp * 64;
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();

  const WaveQ& Q = L.q;
  const unsigned long long need = (unsigned long long)kTile * kTile * pmL * pmL, need_s = kTile * kTile;
  uint32_t phase = 0;
  uint32_t n_pp = 0, n_rays = 0, n_rays64 = 0, n_near = 0, n_graze = 0, n_baddir = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const int64_t g = claim_tile(Q, L.total_tiles, OCC, need, need_s, L.claim_retries, L.err);
      s_used = 0;
      s_slots = 0;
      s_tile = -1;
      if (g >= 0) {
        const int r = find_req(L.tile_base, L.n_req, g);
        const MixedArgs& a = L.mreqs[r];
        s_req = r;
        s_tile = g - L.tile_base[r] + a.tile0;
        if (a.work) s_tile = a.work[s_tile];
        if (OCC) {
          s_rootf = a.nodesf[0];
          s_root = a.nodes[0];
        }
        int64_t bi, bj;
        tile_coords(s_tile, a.nT, bi, bj);
        const uint32_t blk_bytes = (uint32_t)(kComp * a.pmax * kTile * sizeof(float));
        mbar_expect_tx(bar, blk_bytes);
        bulk_g2s(iblk, a.tabf + bi * kComp * a.pmax * kTile, blk_bytes, bar);
      }
    }
    __syncthreads();
    const int64_t t = s_tile;
    if (t < 0) break;
    const int req = s_req;
    const MixedArgs& a = L.mreqs[req];
    const int pm = a.pmax;
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const uint8_t cls = load_tile_class(a.tcls, a.tmask, t, s_mask);
    const bool ok = mbar_wait_bounded(bar, phase);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicOr(L.err, kErrWaitTimeout);
        if (OCC) resv_release(Q, need, need_s);
      }
      break;
    }
    phase ^= 1u;

    if (a.tcls && !(cls & (kClsSlow | kClsNear | kClsTiny)) && !a.ray_log) {  // block-uniform
      if (!a.fast_done) fast_mixed<OCC>(a, iblk, bi, bj, warp, lane, n_pp, n_rays);
      __syncthreads();
      if (OCC && threadIdx.x == 0) resv_release(Q, need, need_s);
      continue;
    }

    const int64_t N = a.N;
    const int64_t j = bj * kTile + lane;
    const int64_t oj = (j < N) ? (a.orig ? (int64_t)a.orig[j] : j) : 0;
    const float* jbf = a.tabf + bj * kComp * pm * kTile + lane;
    const double* jb64 = a.tab + bj * kComp * pm * kTile + lane;
    for (int rr = 0; rr < kTile / 8; ++rr) {
      const int li = warp + 8 * rr;
      const int64_t i = bi * kTile + li;
      if (i >= N) continue;  // warp-uniform
      const bool valid = (j < N) && (i < j);
      const int64_t oi = a.orig ? (int64_t)a.orig[i] : i;
      const bool sw = valid && oi > oj;  // rays leave the element with the lower caller index
      const int npi = a.np[i];
      int npj = valid ? a.np[j] : 0;
      if (valid && a.flat[i] && a.flat[j] && a.nrm[3 * i] == a.nrm[3 * j] &&
          a.nrm[3 * i + 1] == a.nrm[3 * j + 1] && a.nrm[3 * i + 2] == a.nrm[3 * j + 2])
        npj = 0;
      const int qmax = __reduce_max_sync(kFull, npj);
      const double ci0 = a.cen[3 * i], ci1 = a.cen[3 * i + 1], ci2 = a.cen[3 * i + 2];
      double dc0 = 0.0, dc1 = 0.0, dc2 = 0.0;
      bool near = false;
      if (valid) {
        dc0 = a.cen[3 * j] - ci0; dc1 = a.cen[3 * j + 1] - ci1; dc2 = a.cen[3 * j + 2] - ci2;
        const double dm = fmax(a.diam[i], a.diam[j]) * a.near_factor;
        near = (dc0 * dc0 + dc1 * dc1 + dc2 * dc2) < dm * dm;
      }
      if (a.tcls && !a.ray_log && s_mask[li] == 0u) {
        bool close = near;
        if (valid && !close) {
          const double sr = a.rad[i] + a.rad[j] + a.tiny_gap;
          close = (dc0 * dc0 + dc1 * dc1 + dc2 * dc2) <= sr * sr;
        }
        if (!__any_sync(kFull, close)) {  // no ray can be blocked, every pair far field
          fast_mixed<OCC>(a, iblk, bi, bj, li + 8, lane, n_pp, n_rays);
          continue;
        }
      }
      n_near += (near && npj > 0) ? 1 : 0;
      const float d0 = (float)dc0, d1 = (float)dc1, d2 = (float)dc2;
      // FP32 ray origin anchor: the centroid of the casting element
      const float an0 = (float)(ci0 + (sw ? dc0 : 0.0)), an1 = (float)(ci1 + (sw ? dc1 : 0.0)),
                  an2 = (float)(ci2 + (sw ? dc2 : 0.0));
      const float* ibf = iblk + li;
      const double* it64 = a.tab + bi * kComp * pm * kTile + li;
      const bool cullp = OCC && npj > 0 &&
                         (!((s_mask[li] >> lane) & 1u) ||
                          (a.rad && pair_misses_box<true>(a.cen + 3 * i, a.cen + 3 * j,
                                                          fmax(a.rad[i], a.rad[j]) + a.cull_margin, s_root)));
      uint8_t* logp = (a.ray_log && valid)
                          ? a.ray_log + ((uint64_t)(sw ? oj : oi) * N + (sw ? oi : oj)) * a.log_pm * a.log_pm
                          : nullptr;
      double accd = 0.0;   // FP64 terms
      float acc32 = 0.0f;  // FP32 far-field terms
      int64_t slot = -1;
      int n64 = 0, nr = 0;
      for (int q = 0; q < qmax; ++q) {
        const bool lq = q < npj;
        const bool far = lq && !near;
        float oq0 = 0.f, oq1 = 0.f, oq2 = 0.f, nq0 = 0.f, nq1 = 0.f, nq2 = 0.f, wq = 0.f;
        if (far) {
          oq0 = jbf[(0 * pm + q) * kTile]; oq1 = jbf[(1 * pm + q) * kTile]; oq2 = jbf[(2 * pm + q) * kTile];
          nq0 = jbf[(3 * pm + q) * kTile]; nq1 = jbf[(4 * pm + q) * kTile]; nq2 = jbf[(5 * pm + q) * kTile];
          wq = jbf[(6 * pm + q) * kTile];
        }
        float inner = 0.0f;
        for (int p = 0; p < npi; ++p) {
          const float op0 = ibf[(0 * pm + p) * kTile], op1 = ibf[(1 * pm + p) * kTile], op2 = ibf[(2 * pm + p) * kTile];
          const float np0 = ibf[(3 * pm + p) * kTile], np1 = ibf[(4 * pm + p) * kTile], np2 = ibf[(5 * pm + p) * kTile];
          const float wp = ibf[(6 * pm + p) * kTile];
          const float rx = d0 + (oq0 - op0), ry = d1 + (oq1 - op1), rz = d2 + (oq2 - op2);
          const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
          const float di = fmaf(np0, rx, fmaf(np1, ry, np2 * rz));
          const float dj = -fmaf(nq0, rx, fmaf(nq1, ry, nq2 * rz));
          // Grazing point pairs (a cosine within 1e-5 of zero) take FP64 only
          // with occlusion, where the sign of K decides whether a ray is cast.
          // Without it the FP32 term's absolute error, ~2^-20 (|di|+|dj|)|r|/(pi r^4),
          // is the same as for any other far-field term.
          const bool graze = far && (r2 < 1e-18f || (OCC && (di * di <= 1e-10f * r2 || dj * dj <= 1e-10f * r2)));
          float K32 = 0.0f;
          if (far && !graze && di > 0.0f && dj > 0.0f) K32 = (di * dj) * rcp_approx(3.14159265f * (r2 * r2));
          const bool cast32 = far && !graze && K32 > 0.0f;
          bool badray = false, defer32 = false;
          n_pp += lq ? 1 : 0;
          if (OCC && cast32 && cullp) {
            if (logp) logp[sw ? q * a.log_pm + p : p * a.log_pm + q] = 1;
          } else if (OCC && cast32) {
            RayF R;
            const float xo[3] = {an0 + (sw ? oq0 : op0), an1 + (sw ? oq1 : op1), an2 + (sw ? oq2 : op2)};
            const bool rok =
                sw ? make_ray_f(xo, -rx, -ry, -rz, r2, a.delta, R) : make_ray_f(xo, rx, ry, rz, r2, a.delta, R);
            badray = !rok;
            if (rok) {
              defer32 = slab_f(s_rootf, R) != kMiss;
              if (!defer32 && logp) logp[sw ? q * a.log_pm + p : p * a.log_pm + q] = 1;
            }
          }
          n_rays += cast32 ? 1 : 0;
          n_baddir += badray ? 1 : 0;
          // FP64: near field, grazing point pairs, unusable FP32 directions
          const bool need64 = lq && (near || graze || badray);
          bool defer64 = false;
          if (__any_sync(kFull, need64))
            gen_mixed64<OCC>(a, &s_root, it64, jb64, p, q, need64, near || graze, graze, sw, cullp,
                             (double)(wq * (wp * K32)), logp, defer64, accd, n_rays, n_rays64, n_graze);
          if (OCC && __any_sync(kFull, defer32 || defer64)) {
            slot_alloc(Q, (defer32 || defer64) && slot < 0, slot, &s_slots);
            stage_push(st64, n64, defer64, rec_make(slot, sw, p, q));
            if (n64 >= 32) stage_flush(st64, n64, 32, Q.rec64, Q.ctr + kCtrRec64, &s_used);
            run_push(ring, nr, defer32, rec_make(slot, sw, p, q));
            if (__any_sync(kFull, nr == kRunMix))
              run_flush<kRunMix>(ring, nr, false, Q.rec32, Q.ctr + kCtrRec32, &s_used);
          }
          if (far && !graze && !badray && !defer32) inner = fmaf(wp, K32, inner);
        }
        acc32 = fmaf(wq, inner, acc32);
      }
      if (OCC) {
        if (n64 > 0) stage_flush(st64, n64, n64, Q.rec64, Q.ctr + kCtrRec64, &s_used);
        if (__any_sync(kFull, nr > 0)) run_flush<kRunMix>(ring, nr, true, Q.rec32, Q.ctr + kCtrRec32, &s_used);
      }
      const double raw = accd + (double)acc32;
      if (slot >= 0) {
        PendSlot ps;
        ps.i = (int32_t)i;
        ps.j = (int32_t)j;
        ps.req = req;
        ps.pad = 0;
        ps.acc = raw;
        Q.slots[slot] = ps;
      } else if (valid) {
        a.F[oi + oj * N] = raw / a.area[i];
        a.F[oj + oi * N] = raw / a.area[j];
      } else if (j == i) {
        a.F[oi + oi * N] = 0.0 / a.area[i];
      }
    }
    __syncthreads();
    if (OCC && threadIdx.x == 0) resv_release(Q, need - s_used, need_s - s_slots);
  }
  const uint64_t s_pp = warp_sum_u64(n_pp), s_rays = warp_sum_u64(n_rays), s_r64 = warp_sum_u64(n_rays64),
                 s_near = warp_sum_u64(n_near), s_graze = warp_sum_u64(n_graze), s_bad = warp_sum_u64(n_baddir);
  if (lane == 0 && L.counters) {
    atomicAdd(L.counters + 0, s_pp);
    atomicAdd(L.counters + 1, s_rays);
    atomicAdd(L.counters + 4, s_r64);
    atomicAdd(L.counters + 5, s_near);
    atomicAdd(L.counters + 6, s_graze);
    atomicAdd(L.counters + 10, s_bad);
  }
}

// ---------------------------------------------------------------------------
// 2. Traversal kernels.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void log_ray(const TraceArgs& a, int64_t i, int64_t j, bool sw, int p, int q, uint8_t v) {
  const int64_t oi = a.orig ? (int64_t)a.orig[i] : i, oj = a.orig ? (int64_t)a.orig[j] : j;
  uint8_t* lp = a.ray_log + ((uint64_t)(sw ? oj : oi) * a.N + (sw ? oi : oj)) * a.log_pm * a.log_pm;
  lp[sw ? q * a.log_pm + p : p * a.log_pm + q] = v;
}

// ---------------------------------------------------------------------------
// 1b. Pair lists (3-D triangles with occlusion).
//
// Once per pending pair, the triangles that any shadow ray of the pair can
// hit under the reference's FP64 tests (src/GPUBVH.jl:202-285):
//  * leaves: a walk of the tree with the pair's capsule -- the centroid
//    segment grown by R = max(rad_i, rad_j) plus the cull margin, which holds
//    every ray segment of the pair -- skipping each subtree whose box no ray
//    of the pair can hit (pair_misses_box, as for the root in the generation);
//  * triangles of the leaves left: dropped when their group is the pair's
//    own, or when a separating axis (the triangle's normal, or the centroid
//    segment's direction crossed with an edge) puts the triangle farther than
//    R + M_T from the centroid segment.  M_T bounds how far rounding can move
//    a hit of the reference's Moller-Trumbore test: with eps = 2^-53, a hit
//    needs |a| >= 1e-10, and then its u and v differ from the exact
//    line-plane values by at most (eps / 1e-10)(8.3 S Lx + 6.6 Lx^2) and its
//    t by (eps / 1e-10) 14.7 S Lx^2, S bounding |o - v0| and t_max and Lx the
//    edge lengths; a hit therefore puts a point of the ray segment within
//    E_t + 3 (E_u + E_v) Lx of the triangle.  The list kernel uses twice that.
// A ray of the pair tests the listed triangles only, each behind the slab
// test of its own leaf box: with a finite 1/d the reference's slab test is
// monotone under box inclusion (rounding is monotone and the box bounds only
// widen the parameter intervals), every ancestor box contains the leaf box
// (boxes are min/max unions over the triangles), so the leaf's test passing
// means the reference's walk reaches the leaf.  A pair with more than
// kListMax triangles keeps n = -1 and its rays walk the tree.
// ---------------------------------------------------------------------------
// The list of one pending pair, built by its warp: a breadth-first walk of
// the tree with the capsule test from the precomputed start nodes (one node
// per lane; every start node's box lies inside its ancestors', so skipping
// the ancestors' tests only tests more), then the triangles of the candidate
// leaves, four leaves of up to eight triangles per round of 32 lanes.
// Returns the list length (entries in `list`, in a deterministic order), or
// -1 when a frontier, the candidate leaves or the list exceed their
// capacity.  Warp-uniform.
__device__ int build_pair_list(const TraceArgs& a, const PendSlot& ps, int* front, int* leaves, int* list) {
  const int lane = threadIdx.x & 31;
  const int64_t i = ps.i, j = ps.j;
  CapsuleF cap;
  float bf[3];
  const double R = fmax(a.rad[i], a.rad[j]) + a.cull_margin;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double A = a.cen[3 * i + c], B = a.cen[3 * j + c];
    const double dd = B - A;
    cap.A[c] = (float)A;
    bf[c] = (float)B;
    cap.zero[c] = dd == 0.0;
    cap.inv[c] = cap.zero[c] ? 0.0f : (float)(1.0 / dd);
  }
  cap.R = (float)R + a.sat_em;
  int* cur = front;
  int* nxt = front + kListFront;
  if (lane < a.n_frontier) cur[lane] = a.frontier[lane];
  __syncwarp();
  int ncur = a.n_frontier, nleaf = 0;
  while (ncur > 0) {  // each round descends one level: bounded by the tree depth
    int nnext = 0;
    for (int b = 0; b < ncur; b += 32) {
      const int t = b + lane;
      bool pass = false, leaf = false;
      int k = 0, right = 0;
      if (t < ncur && cur[t] < a.n_nodes) {
        k = cur[t];
        const NodeF nd = a.nodesf[k];
        pass = !capsule_misses_box(cap, nd);
        leaf = (nd.ab & 15) > 0;
        if (pass && !leaf) right = a.nodesf[k + 1].miss;  // the right child follows the left subtree
      }
      const uint32_t ml = __ballot_sync(kFull, pass && leaf), mi = __ballot_sync(kFull, pass && !leaf);
      const int pl = nleaf + __popc(ml & lanemask_lt());
      if (pass && leaf && pl < kListLeaves) leaves[pl] = k;
      nleaf += __popc(ml);
      const int pi = nnext + 2 * __popc(mi & lanemask_lt());
      if (pass && !leaf && pi + 1 < kListFront) {
        nxt[pi] = k + 1;
        nxt[pi + 1] = right;
      }
      nnext += 2 * __popc(mi);
    }
    __syncwarp();
    if (nleaf > kListLeaves || nnext > kListFront) return -1;
    int* tmp = cur;
    cur = nxt;
    nxt = tmp;
    ncur = nnext;
  }
  // triangles of the candidate leaves
  const float df[3] = {bf[0] - cap.A[0], bf[1] - cap.A[1], bf[2] - cap.A[2]};
  const float Rf = (float)R;
  const int32_t gi = a.group[i], gj = a.group[j];
  int n = 0;
  for (int b = 0; b < nleaf; b += 4) {
    const int li = b + (lane >> 3), u8 = lane & 7;
    bool keep = false;
    int u = 0;
    if (li < nleaf) {
      const int32_t ab = a.nodesf[leaves[li]].ab;
      if (u8 < (ab & 15)) {
        u = (ab >> 4) + u8;
        const float4 p0 = a.sat[3 * u], p1 = a.sat[3 * u + 1], p2 = a.sat[3 * u + 2];
        const int32_t g = __float_as_int(p1.w);
        keep = g != gi && g != gj && !pair_misses_tri(cap.A, bf, df, Rf, a.sat_em, p0, p1, p2);
      }
    }
    const uint32_t m = __ballot_sync(kFull, keep);
    const int pos = n + __popc(m & lanemask_lt());
    if (keep && pos < kListCap) list[pos] = u;
    n += __popc(m);
    if (n > kListCap) return -1;
  }
  __syncwarp();
  return n;
}

// One warp per pending pair of the chunk.
__global__ void __launch_bounds__(256) k_plist(const TraceBatch* __restrict__ Lp) {
  __shared__ int s_front[8][2 * kListFront];
  __shared__ int s_leaf[8][kListLeaves];
  __shared__ int s_list[8][kListCap];
  const TraceBatch& L = *Lp;
  const WaveQ& Q = L.q;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned long long ns = *(volatile unsigned long long*)(Q.ctr + kCtrSlots);
  const unsigned long long stride = (unsigned long long)gridDim.x * 8;
  uint32_t n_list = 0, n_walk = 0;
  for (unsigned long long s = (unsigned long long)blockIdx.x * 8 + warp; s < ns; s += stride) {
    const PendSlot ps = Q.slots[s];
    const TraceArgs& a = L.reqs[ps.req];
    int n = -1;
    if (a.dim3 && a.leaf_of && a.rad && a.sat && a.nodesf && a.frontier)
      n = build_pair_list(a, ps, s_front[warp], s_leaf[warp], s_list[warp]);
    long long off = 0;
    if (n > 0) {
      if (lane == 0) off = (long long)atomicAdd(Q.ctr + kCtrPool, (unsigned long long)n);
      off = __shfl_sync(kFull, off, 0);
      if (off + n > Q.pool_cap) n = -1;  // pool full: this pair walks
      else
        for (int e = lane; e < n; e += 32) Q.pool[off + e] = s_list[warp][e];
    }
    if (lane == 0) {
      PairList pl;
      pl.n = n;
      pl.off = (int32_t)off;
      Q.plist[s] = pl;
      n_list += n >= 0 ? 1 : 0;
      n_walk += n < 0 ? 1 : 0;
    }
    __syncwarp();
  }
  if (lane == 0 && L.counters) {
    atomicAdd(L.counters + 11, (unsigned long long)n_list);
    atomicAdd(L.counters + 12, (unsigned long long)n_walk);
  }
}

// A ray against its pair's list (entries e[0..n) of the pool): kHit
// (blocked), kMiss or, for FP32 rays, kUnsure (some certified decision was
// not certain and no certain hit was found).
template <typename Src, typename Pol, typename Tri>
__device__ __forceinline__ int trace_list(const int32_t* e, int n, const Src& nodes, const Tri* tris,
                                          const int32_t* leaf_of, const Pol& pol, TravCount& cnt) {
  int last = -1, s = kMiss;
  bool unsure = false;
  // software-pipelined: the triangle of entry k and the index and leaf of
  // entry k+1 are loaded before entry k's box test, so the loads of one
  // entry overlap the tests of the previous one
  int u = n > 0 ? e[0] : 0;
  int lf = n > 0 ? leaf_of[u] : 0;
  for (int k = 0; k < n; ++k) {
    const Tri t = tris[u];
    int un = 0, lfn = 0;
    if (k + 1 < n) {
      un = e[k + 1];
      lfn = leaf_of[un];
    }
    if (lf != last) {
      last = lf;
      s = pol.node(nodes(lf));
      ++cnt.nodes;
      if (s == kUnsure) ++cnt.unsure_slab;
    }
    if (s != kMiss) {
      ++cnt.prims;
      const int m = pol.prim_direct(t);
      if (m == kUnsure) ++cnt.unsure_prim;
      if (m == kHit && s == kHit) return kHit;
      if (m != kMiss) unsure = true;
    }
    u = un;
    lf = lfn;
  }
  return unsure ? kUnsure : kMiss;
}

// Sets the (p, q) visibility bits of the warp's visible rays.  The rays of one
// pair sit in consecutive lanes, so the bits of each run of lanes with the
// same (slot, word) are OR-combined by a segmented scan and the last lane of
// the run issues one atomicOr.  Lanes whose key also appears in a run further
// back only add bits of that same word, which OR absorbs.  Warp-uniform call.
__device__ __forceinline__ void set_visible_warp(const WaveQ& Q, bool vis, int64_t slot, int pm, int p, int q) {
  const int lane = threadIdx.x & 31;
  const int b = p * pm + q;
  const long long key = vis ? (long long)(slot * Q.vis_words + (b >> 6)) : -1ll - lane;
  unsigned long long bits = vis ? (1ull << (b & 63)) : 0ull;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long k2 = __shfl_up_sync(kFull, key, o);
    const unsigned long long b2 = __shfl_up_sync(kFull, bits, o);
    if (lane >= o && k2 == key) bits |= b2;
  }
  const long long next = __shfl_down_sync(kFull, key, 1);
  if (vis && (lane == 31 || next != key)) atomicOr(reinterpret_cast<unsigned long long*>(Q.vis + key), bits);
}

// A queued ray: its record, its pair and its request.
struct QRay {
  int64_t slot, i, j;
  int p, q, req;
  bool sw;
};

__device__ __forceinline__ QRay read_ray(const WaveQ& Q, uint64_t r) {
  QRay x;
  x.slot = rec_slot(r);
  x.sw = rec_sw(r);
  x.p = rec_p(r);
  x.q = rec_q(r);
  const PendSlot ps = Q.slots[x.slot];
  x.i = ps.i;
  x.j = ps.j;
  x.req = ps.req;
  return x;
}

template <bool DIM3>
__global__ void __launch_bounds__(256, 3) k_trace64(const TraceBatch* __restrict__ Lp) {
  extern __shared__ __align__(128) unsigned char smem[];
  const TraceBatch& L = *Lp;
  NodeD* snodes = reinterpret_cast<NodeD*>(smem);
  const bool in_smem = L.nodes64_in_smem;
  RayBank* wsa = reinterpret_cast<RayBank*>(snodes + (in_smem ? L.n_nodes_smem : 0));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RayBank& ws = wsa[warp];
  if (in_smem) SwizNodes<NodeD>::fill(reinterpret_cast<int4*>(snodes), L.smem_nodes64, L.n_nodes_smem);
  __syncthreads();
  const WaveQ& Q = L.q;
  const unsigned long long n = *(volatile unsigned long long*)(Q.ctr + kCtrRec64);
  TravCount tc;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(Q.ctr + kCtrHead64, 32ull);
    base = __shfl_sync(kFull, base, 0);
    if (base >= n) break;
    const bool have = base + lane < n;
    const QRay x = have ? read_ray(Q, Q.rec64[base + lane]) : QRay{0, 0, 0, 0, 0, 0, false};
    const TraceArgs& a = L.reqs[x.req];
    const int pm = a.pmax;
    double xi[3], xj[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xi[c] = have ? a.tab[tab_at(x.i, c, x.p, pm)] : 0.0;
      xj[c] = have ? a.tab[tab_at(x.j, c, x.q, pm)] : 0.0;
    }
    const int32_t gi = have ? a.group[x.i] : 0, gj = have ? a.group[x.j] : 0;
    const int n_nodes = have ? a.n_nodes : 0;
    int res;
    if (DIM3) {
      PolD3 pol;
      pol.tris = a.tris;
      const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
      const double r2 = (rx * rx + ry * ry) + rz * rz;
      if (have) {
        if (x.sw) make_ray(xj, -rx, -ry, -rz, r2, pol.R);
        else make_ray(xi, rx, ry, rz, r2, pol.R);
        pol.store(ws, lane, gi, gj);
      }
      // the pair's list when it has one and the ray's 1/d is finite
      int ln = -1;
      const int32_t* le = nullptr;
      if (have && Q.plist) {
        const PairList pl = Q.plist[x.slot];
        ln = pl.n;
        le = Q.pool + pl.off;
        if (pol.R.zdir || !(isfinite(pol.R.inv[0]) && isfinite(pol.R.inv[1]) && isfinite(pol.R.inv[2]))) ln = -1;
      }
      const bool walk = have && ln < 0;
      res = kMiss;
      if (have && ln >= 0)
        res = in_smem ? trace_list(le, ln, SwizNodes<NodeD>{reinterpret_cast<const int4*>(snodes)}, a.tris, a.leaf_of,
                                   pol, tc)
                      : trace_list(le, ln, GlobalNodes<NodeD>{a.nodes}, a.tris, a.leaf_of, pol, tc);
      if (__any_sync(kFull, walk)) {
        const int rw =
            in_smem ? trace_batch(walk, SwizNodes<NodeD>{reinterpret_cast<const int4*>(snodes)}, n_nodes, ws, pol, tc)
                    : trace_batch(walk, GlobalNodes<NodeD>{a.nodes}, n_nodes, ws, pol, tc);
        if (walk) res = rw;
      }
    } else {
      PolD2 pol;
      pol.segs = a.segs;
      pol.a[0] = x.sw ? xj[0] : xi[0];
      pol.a[1] = x.sw ? xj[1] : xi[1];
      pol.b[0] = x.sw ? xi[0] : xj[0];
      pol.b[1] = x.sw ? xi[1] : xj[1];
      if (have) pol.store(ws, lane, gi, gj);
      res = in_smem ? trace_batch(have, SwizNodes<NodeD>{reinterpret_cast<const int4*>(snodes)}, n_nodes, ws, pol, tc)
                            : trace_batch(have, GlobalNodes<NodeD>{a.nodes}, n_nodes, ws, pol, tc);
    }
    set_visible_warp(Q, have && res != kHit, x.slot, pm, x.p, x.q);
    if (have && a.ray_log) log_ray(a, x.i, x.j, x.sw, x.p, x.q, res == kHit ? 2 : 1);
  }
  const uint64_t s_nodes = warp_sum_u64(tc.nodes), s_prims = warp_sum_u64(tc.prims);
  if (lane == 0 && L.counters) {
    atomicAdd(L.counters + 2, s_nodes);
    atomicAdd(L.counters + 3, s_prims);
  }
}

__global__ void __launch_bounds__(256, 4) k_trace32(const TraceBatch* __restrict__ Lp) {
  extern __shared__ __align__(128) unsigned char smem[];
  const TraceBatch& L = *Lp;
  NodeF* snodes = reinterpret_cast<NodeF*>(smem);
  const bool in_smem = L.nodes32_in_smem;
  RayBankF* wsa = reinterpret_cast<RayBankF*>(snodes + (in_smem ? L.n_nodes_smem : 0));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RayBankF& ws = wsa[warp];
  if (in_smem) SwizNodes<NodeF>::fill(reinterpret_cast<int4*>(snodes), L.smem_nodes32, L.n_nodes_smem);
  __syncthreads();
  const WaveQ& Q = L.q;
  const unsigned long long n = *(volatile unsigned long long*)(Q.ctr + kCtrRec32);
  TravCount tc;
  uint32_t n_unsure = 0;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(Q.ctr + kCtrHead32, 32ull);
    base = __shfl_sync(kFull, base, 0);
    if (base >= n) break;
    const bool have = base + lane < n;
    const uint64_t rec = have ? Q.rec32[base + lane] : 0ull;
    const QRay x = have ? read_ray(Q, rec) : QRay{0, 0, 0, 0, 0, 0, false};
    const TraceArgs& a = L.reqs[x.req];
    const int pm = a.pmax;
    PolF3 pol;
    pol.tris = a.trisf;
    if (have) {
      // the generation's FP32 ray, operation for operation
      const int64_t i = x.i, j = x.j;
      const bool sw = x.sw;
      const double ci0 = a.cen[3 * i], ci1 = a.cen[3 * i + 1], ci2 = a.cen[3 * i + 2];
      const double dc0 = a.cen[3 * j] - ci0, dc1 = a.cen[3 * j + 1] - ci1, dc2 = a.cen[3 * j + 2] - ci2;
      const float d0 = (float)dc0, d1 = (float)dc1, d2 = (float)dc2;
      const float an0 = (float)(ci0 + (sw ? dc0 : 0.0)), an1 = (float)(ci1 + (sw ? dc1 : 0.0)),
                  an2 = (float)(ci2 + (sw ? dc2 : 0.0));
      const float op0 = a.tabf[tab_at(i, 0, x.p, pm)], op1 = a.tabf[tab_at(i, 1, x.p, pm)],
                  op2 = a.tabf[tab_at(i, 2, x.p, pm)];
      const float oq0 = a.tabf[tab_at(j, 0, x.q, pm)], oq1 = a.tabf[tab_at(j, 1, x.q, pm)],
                  oq2 = a.tabf[tab_at(j, 2, x.q, pm)];
      const float rx = d0 + (oq0 - op0), ry = d1 + (oq1 - op1), rz = d2 + (oq2 - op2);
      const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
      const float xo[3] = {an0 + (sw ? oq0 : op0), an1 + (sw ? oq1 : op1), an2 + (sw ? oq2 : op2)};
      if (sw) make_ray_f(xo, -rx, -ry, -rz, r2, a.delta, pol.R);
      else make_ray_f(xo, rx, ry, rz, r2, a.delta, pol.R);
      pol.store(ws, lane, a.group[i], a.group[j]);
    }
    const int n_nodes = have ? a.n_nodes : 0;
    // the pair's list when it has one (FP32 rays always have a finite 1/d)
    int ln = -1;
    const int32_t* le = nullptr;
    if (have && Q.plist) {
      const PairList pl = Q.plist[x.slot];
      ln = pl.n;
      le = Q.pool + pl.off;
    }
    const bool walk = have && ln < 0;
    int res = kMiss;
    if (have && ln >= 0)
      res = in_smem ? trace_list(le, ln, SwizNodes<NodeF>{reinterpret_cast<const int4*>(snodes)}, a.trisf, a.leaf_of,
                                 pol, tc)
                    : trace_list(le, ln, GlobalNodes<NodeF>{a.nodesf}, a.trisf, a.leaf_of, pol, tc);
    if (__any_sync(kFull, walk)) {
      const int rw =
          in_smem ? trace_batch(walk, SwizNodes<NodeF>{reinterpret_cast<const int4*>(snodes)}, n_nodes, ws, pol, tc)
                  : trace_batch(walk, GlobalNodes<NodeF>{a.nodesf}, n_nodes, ws, pol, tc);
      if (walk) res = rw;
    }
    set_visible_warp(Q, have && res == kMiss, x.slot, pm, x.p, x.q);
    if (have && a.ray_log && res != kUnsure) log_ray(a, x.i, x.j, x.sw, x.p, x.q, res == kHit ? 2 : 1);
    // uncertain rays go to the FP64 queue
    const bool uns = have && res == kUnsure;
    const uint32_t m = __ballot_sync(kFull, uns);
    if (m) {
      unsigned long long b64 = 0;
      if (lane == 0) b64 = atomicAdd(Q.ctr + kCtrRec64, (unsigned long long)__popc(m));
      b64 = __shfl_sync(kFull, b64, 0);
      if (uns) Q.rec64[b64 + __popc(m & lanemask_lt())] = rec;
    }
    n_unsure += uns ? 1 : 0;
  }
  const uint64_t s_nodes = warp_sum_u64(tc.nodes), s_prims = warp_sum_u64(tc.prims),
                 s_us = warp_sum_u64(tc.unsure_slab), s_up = warp_sum_u64(tc.unsure_prim),
                 s_un = warp_sum_u64(n_unsure);
  if (lane == 0 && L.counters) {
    atomicAdd(L.counters + 2, s_nodes);
    atomicAdd(L.counters + 3, s_prims);
    atomicAdd(L.counters + 4, s_un);
    atomicAdd(L.counters + 7, s_un);
    atomicAdd(L.counters + 8, s_us);
    atomicAdd(L.counters + 9, s_up);
  }
}

// ---------------------------------------------------------------------------
// 3. Resolve: one thread per pending pair.
// ---------------------------------------------------------------------------
template <bool DIM3>
__global__ void __launch_bounds__(256) k_resolve64(const ResolveBatch* __restrict__ Lp) {
  const WaveQ& Q = Lp->q;
  const unsigned long long ns = *(volatile unsigned long long*)(Q.ctr + kCtrSlots);
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < ns;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const PendSlot ps = Q.slots[s];
    const ResolveArgs& a = Lp->reqs[ps.req];
    const int pm = a.pmax;
    const int64_t i = ps.i, j = ps.j;
    double raw = ps.acc;
    for (int w = 0; w < Q.vis_words; ++w) {
      unsigned long long bits = Q.vis[s * Q.vis_words + w];
      while (bits) {
        const int b = w * 64 + (__ffsll((long long)bits) - 1);
        bits &= bits - 1ull;
        const int p = b / pm, q = b - p * pm;
        double xi[3], ni[3], xj[3], nj[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          xi[c] = a.tab[tab_at(i, c, p, pm)];
          ni[c] = a.tab[tab_at(i, 3 + c, p, pm)];
          xj[c] = a.tab[tab_at(j, c, q, pm)];
          nj[c] = a.tab[tab_at(j, 3 + c, q, pm)];
        }
        const double wi = a.tab[tab_at(i, 6, p, pm)], wj = a.tab[tab_at(j, 6, q, pm)];
        const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
        const double r2 = (rx * rx + ry * ry) + rz * rz;
        const double K = k_fast<DIM3>(rx, ry, rz, r2, ni, nj);
        raw += wj * (wi * K);
      }
    }
    const int64_t oi = a.orig ? (int64_t)a.orig[i] : i, oj = a.orig ? (int64_t)a.orig[j] : j;
    a.F[oi + oj * a.N] = raw / a.area[i];
    a.F[oj + oi * a.N] = raw / a.area[j];
  }
}

__global__ void __launch_bounds__(256) k_resolve_mixed(const ResolveBatch* __restrict__ Lp) {
  const WaveQ& Q = Lp->q;
  const unsigned long long ns = *(volatile unsigned long long*)(Q.ctr + kCtrSlots);
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < ns;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const PendSlot ps = Q.slots[s];
    const ResolveArgs& a = Lp->reqs[ps.req];
    const int pm = a.pmax;
    const int64_t i = ps.i, j = ps.j;
    double raw = ps.acc;
    // the generation's near-field and FP32 quantities, operation for operation
    const double ci0 = a.cen[3 * i], ci1 = a.cen[3 * i + 1], ci2 = a.cen[3 * i + 2];
    const double dc0 = a.cen[3 * j] - ci0, dc1 = a.cen[3 * j + 1] - ci1, dc2 = a.cen[3 * j + 2] - ci2;
    const double dm = fmax(a.diam[i], a.diam[j]) * a.near_factor;
    const bool near = (dc0 * dc0 + dc1 * dc1 + dc2 * dc2) < dm * dm;
    const float d0 = (float)dc0, d1 = (float)dc1, d2 = (float)dc2;
    for (int w = 0; w < Q.vis_words; ++w) {
      unsigned long long bits = Q.vis[s * Q.vis_words + w];
      while (bits) {
        const int b = w * 64 + (__ffsll((long long)bits) - 1);
        bits &= bits - 1ull;
        const int p = b / pm, q = b - p * pm;
        bool exact = near;
        double c = 0.0;
        if (!near) {
          const float op0 = a.tabf[tab_at(i, 0, p, pm)], op1 = a.tabf[tab_at(i, 1, p, pm)], op2 = a.tabf[tab_at(i, 2, p, pm)];
          const float np0 = a.tabf[tab_at(i, 3, p, pm)], np1 = a.tabf[tab_at(i, 4, p, pm)], np2 = a.tabf[tab_at(i, 5, p, pm)];
          const float wp = a.tabf[tab_at(i, 6, p, pm)];
          const float oq0 = a.tabf[tab_at(j, 0, q, pm)], oq1 = a.tabf[tab_at(j, 1, q, pm)], oq2 = a.tabf[tab_at(j, 2, q, pm)];
          const float nq0 = a.tabf[tab_at(j, 3, q, pm)], nq1 = a.tabf[tab_at(j, 4, q, pm)], nq2 = a.tabf[tab_at(j, 5, q, pm)];
          const float wq = a.tabf[tab_at(j, 6, q, pm)];
          const float rx = d0 + (oq0 - op0), ry = d1 + (oq1 - op1), rz = d2 + (oq2 - op2);
          const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
          const float di = fmaf(np0, rx, fmaf(np1, ry, np2 * rz));
          const float dj = -fmaf(nq0, rx, fmaf(nq1, ry, nq2 * rz));
          const bool graze = (di * di <= 1e-10f * r2 || dj * dj <= 1e-10f * r2 || r2 < 1e-18f);
          if (graze) {
            exact = true;
          } else {
            float K32 = 0.0f;
            if (di > 0.0f && dj > 0.0f) K32 = (di * dj) * rcp_approx(3.14159265f * (r2 * r2));
            c = (double)(wq * (wp * K32));
          }
        }
        if (exact) {
          double xi[3], ni[3], xj[3], nj[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            xi[k] = a.tab[tab_at(i, k, p, pm)];
            ni[k] = a.tab[tab_at(i, 3 + k, p, pm)];
            xj[k] = a.tab[tab_at(j, k, q, pm)];
            nj[k] = a.tab[tab_at(j, 3 + k, q, pm)];
          }
          const double wi = a.tab[tab_at(i, 6, p, pm)], wj = a.tab[tab_at(j, 6, q, pm)];
          const double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
          const double r2 = (rx * rx + ry * ry) + rz * rz;
          c = wj * (wi * k_fast<true>(rx, ry, rz, r2, ni, nj));
        }
        raw += c;
      }
    }
    const int64_t oi = a.orig ? (int64_t)a.orig[i] : i, oj = a.orig ? (int64_t)a.orig[j] : j;
    a.F[oi + oj * a.N] = raw / a.area[i];
    a.F[oj + oi * a.N] = raw / a.area[j];
  }
}

// ---------------------------------------------------------------------------
// 1c. Tiles without shadow-ray work, in a kernel of their own before the
// chunks: each warp claims whole tiles, reads the source element's points
// from the table in global memory (L1 / L2 resident; the warp's lanes read
// the same address) and runs the quadrature-only loop over the tile's 32
// rows -- no shared-memory staging, no block barriers, and the registers of
// that loop alone (the chunked generation then skips these tiles).
// ---------------------------------------------------------------------------
// resident blocks of 256 per SM the quadrature-only kernels are compiled for
#ifndef RVF_FAST_MIN_BLOCKS
#define RVF_FAST_MIN_BLOCKS 2
#endif

// A task is one row group of a tile: groups = 1 (the whole tile: row
// classes li0 = 0..7, each the rows li0, li0 + 8, ...), 2, 4 or 8 (half, a
// quarter or one of the row classes), or 32 (one row: li0 = 8 + row), so
// small meshes spread over more warps.  The shape changes no sum: every pair
// is formed by the same loop.
__device__ __forceinline__ bool fast_task(unsigned long long* task_ctr, int64_t n_tiles, int groups,
                                          const uint8_t* tcls, uint8_t skip, int lane, int64_t& t, int& r0,
                                          int& r1) {
  for (;;) {
    unsigned long long k = 0;
    if (lane == 0) k = atomicAdd(task_ctr, 1ull);
    k = __shfl_sync(kFull, k, 0);
    const unsigned long long tile = k / (unsigned)groups;
    if (tile >= (unsigned long long)n_tiles) return false;
    if (tcls[tile] & skip) continue;
    const int g = (int)(k - tile * (unsigned)groups);
    t = (int64_t)tile;
    if (groups <= 8) {
      r0 = g * (8 / groups);
      r1 = r0 + 8 / groups;
    } else {
      r0 = 8 + g;
      r1 = r0 + 1;
    }
    return true;
  }
}

template <bool DIM3, bool OCC, int QB>
__global__ void __launch_bounds__(256, RVF_FAST_MIN_BLOCKS) k_fast_fp64(const PairArgs a, unsigned long long* task_ctr,
                                                                       unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  uint32_t n_pp = 0, n_rays = 0;
  int64_t t;
  int r0, r1;
  while (fast_task(task_ctr, a.n_tiles, a.fast_groups, a.tcls, kClsSlow, lane, t, r0, r1)) {
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const double* ib = a.tab + bi * kComp * a.pmax * kTile;
    for (int r = r0; r < r1; ++r) gen_fast_fp64_body<DIM3, OCC, QB>(a, ib, bi, bj, r, lane, n_pp, n_rays);
  }
  const uint64_t s_pp = warp_sum_u64(n_pp), s_rays = warp_sum_u64(n_rays);
  if (lane == 0 && counters) {
    atomicAdd(counters + 0, s_pp);
    atomicAdd(counters + 1, s_rays);
  }
}

template <bool OCC, int QB>
__global__ void __launch_bounds__(256, RVF_FAST_MIN_BLOCKS) k_fast_mixed(const MixedArgs a, unsigned long long* task_ctr,
                                                                        unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  uint32_t n_pp = 0, n_rays = 0;
  int64_t t;
  int r0, r1;
  while (fast_task(task_ctr, a.n_tiles, a.fast_groups, a.tcls, kClsSlow | kClsNear | kClsTiny, lane, t, r0, r1)) {
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const float* ib = a.tabf + bi * kComp * a.pmax * kTile;
    for (int r = r0; r < r1; ++r) gen_fast_mixed_body<OCC, QB>(a, ib, bi, bj, r, lane, n_pp, n_rays);
  }
  const uint64_t s_pp = warp_sum_u64(n_pp), s_rays = warp_sum_u64(n_rays);
  if (lane == 0 && counters) {
    atomicAdd(counters + 0, s_pp);
    atomicAdd(counters + 1, s_rays);
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
int fast_qb_default(bool mixed, int pmax) {
  if (!mixed) return pmax <= 3 ? 3 : 4;
  if (pmax == 7 || pmax == 13 || pmax == 49) return 7;
  if (pmax == 5 || pmax == 25) return 5;
  if (pmax == 3 || pmax == 9) return 3;
  return 8;
}
bool fast_qb_supported(bool mixed, int qb) {
  return mixed ? (qb == 2 || qb == 3 || qb == 4 || qb == 5 || qb == 7 || qb == 8) : (qb >= 2 && qb <= 4);
}

// Loads every compiled quadrature-only kernel (module loading is lazy: a
// kernel's first launch would otherwise also pay for it).
cudaError_t preload_fast() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaSuccess;
  auto touch = [&](const void* fn) {
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
  };
#define RVF_TOUCH_MIXED(Q)                        \
  touch((const void*)k_fast_mixed<true, Q>);      \
  touch((const void*)k_fast_mixed<false, Q>);
#define RVF_TOUCH_FP64(Q)                             \
  touch((const void*)k_fast_fp64<true, true, Q>);     \
  touch((const void*)k_fast_fp64<true, false, Q>);    \
  touch((const void*)k_fast_fp64<false, true, Q>);    \
  touch((const void*)k_fast_fp64<false, false, Q>);
  RVF_TOUCH_MIXED(2) RVF_TOUCH_MIXED(3) RVF_TOUCH_MIXED(4) RVF_TOUCH_MIXED(5) RVF_TOUCH_MIXED(7) RVF_TOUCH_MIXED(8)
  RVF_TOUCH_FP64(2) RVF_TOUCH_FP64(3) RVF_TOUCH_FP64(4)
#undef RVF_TOUCH_MIXED
#undef RVF_TOUCH_FP64
  return e;
}

cudaError_t launch_fast(bool mixed, bool dim3, bool occ, int qb, const PairArgs& a, const MixedArgs& m,
                        unsigned long long* task_ctr, unsigned long long* counters, int sm_count, cudaStream_t st) {
  auto launch = [&](auto fn, const auto& args) -> cudaError_t {
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    fn<<<(unsigned)(sm_count * per_sm), 256, 0, st>>>(args, task_ctr, counters);
    return cudaGetLastError();
  };
  if (mixed) {
    switch (qb) {
      case 2: return occ ? launch(k_fast_mixed<true, 2>, m) : launch(k_fast_mixed<false, 2>, m);
      case 3: return occ ? launch(k_fast_mixed<true, 3>, m) : launch(k_fast_mixed<false, 3>, m);
      case 4: return occ ? launch(k_fast_mixed<true, 4>, m) : launch(k_fast_mixed<false, 4>, m);
      case 5: return occ ? launch(k_fast_mixed<true, 5>, m) : launch(k_fast_mixed<false, 5>, m);
      case 7: return occ ? launch(k_fast_mixed<true, 7>, m) : launch(k_fast_mixed<false, 7>, m);
      case 8: return occ ? launch(k_fast_mixed<true, 8>, m) : launch(k_fast_mixed<false, 8>, m);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (qb) {
#define RVF_FAST64(Q)                                                                          \
  case Q:                                                                                      \
    if (dim3) return occ ? launch(k_fast_fp64<true, true, Q>, a) : launch(k_fast_fp64<true, false, Q>, a); \
    return occ ? launch(k_fast_fp64<false, true, Q>, a) : launch(k_fast_fp64<false, false, Q>, a);
    RVF_FAST64(2)
    RVF_FAST64(3)
    RVF_FAST64(4)
#undef RVF_FAST64
    default: return cudaErrorInvalidValue;
  }
}
size_t gen_smem_bytes(bool mixed, int pmax, bool occ) {
  // tile block, then (occlusion) the per-warp FP64 staging (mixed) and the
  // per-lane runs, then the mbarrier
  const size_t stage = occ ? ((mixed ? (size_t)8 * 64 + kRunMix * 256 : (size_t)kRun * 256)) * sizeof(uint64_t) : 0;
  return gen_tab_bytes(mixed, pmax) + stage + 16;
}

size_t trace_smem_bytes(bool fp32, int n_nodes_smem) {
  return (size_t)n_nodes_smem * (fp32 ? sizeof(NodeF) : sizeof(NodeD)) + 8 * (fp32 ? sizeof(RayBankF) : sizeof(RayBank));
}

template <typename F>
static cudaError_t set_smem(F fn, size_t smem) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename F>
static int grid_for(F fn, size_t smem, int sm_count, int cap) {
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  if (per_sm > cap) per_sm = cap;
  return sm_count * per_sm;
}

cudaError_t launch_gen(const WaveShape& sh, const GenBatch* g, int sm_count, cudaStream_t st) {
  const size_t smem = gen_smem_bytes(sh.mixed, sh.pmax_max, sh.occ);
  auto launch = [&](auto fn) -> cudaError_t {
    cudaError_t e = set_smem(fn, smem);
    if (e != cudaSuccess) return e;
    const int grid = grid_for(fn, smem, sm_count, sh.gen_bps > 0 ? sh.gen_bps : 4);
    fn<<<(unsigned)grid, 256, smem, st>>>(g);
    return cudaGetLastError();
  };
  if (sh.mixed) return sh.occ ? launch(k_gen_mixed<true>) : launch(k_gen_mixed<false>);
  if (sh.dim3) return sh.occ ? launch(k_gen_fp64<true, true>) : launch(k_gen_fp64<true, false>);
  return sh.occ ? launch(k_gen_fp64<false, true>) : launch(k_gen_fp64<false, false>);
}

cudaError_t launch_trace(const WaveShape& sh, const TraceBatch* t, bool fp32, int sm_count, cudaStream_t st) {
  const bool in_smem = fp32 ? sh.trace32_nodes_smem : sh.trace64_nodes_smem;
  const size_t smem = trace_smem_bytes(fp32, in_smem ? sh.n_nodes_smem : 0);
  auto launch = [&](auto fn) -> cudaError_t {
    cudaError_t e = set_smem(fn, smem);
    if (e != cudaSuccess) return e;
    const int grid = grid_for(fn, smem, sm_count, sh.trace_bps > 0 ? sh.trace_bps : 8);
    fn<<<(unsigned)grid, 256, smem, st>>>(t);
    return cudaGetLastError();
  };
  if (fp32) return launch(k_trace32);
  return sh.dim3 ? launch(k_trace64<true>) : launch(k_trace64<false>);
}

cudaError_t launch_plist(const TraceBatch* t, int sm_count, cudaStream_t st) {
  k_plist<<<(unsigned)(sm_count * 8), 256, 0, st>>>(t);
  return cudaGetLastError();
}

cudaError_t launch_resolve(const WaveShape& sh, const ResolveBatch* r, int sm_count, cudaStream_t st) {
  const int grid = sm_count * 8;
  if (sh.mixed) k_resolve_mixed<<<grid, 256, 0, st>>>(r);
  else if (sh.dim3) k_resolve64<true><<<grid, 256, 0, st>>>(r);
  else k_resolve64<false><<<grid, 256, 0, st>>>(r);
  return cudaGetLastError();
}

}  // namespace rvf
