// kernels_cull.cu -- tile classification before the pair pipeline.
//
// The reference casts a shadow ray for every point pair with K > 0
// (src/GPUKernels.jl:289-304) and walks the whole flat BVH for it
// (src/GPUBVH.jl:202-285).  Most of those rays cannot be blocked: with the
// reference's transposed triangle read (src/GPUBVH.jl:243-245) the triangles
// a ray actually tests are thin slivers, and a ray only reaches a triangle
// after passing the slab test of its (true-geometry) leaf box.  One warp per
// 32 x 32 tile of the upper triangle decides, with certified bounds, which
// pairs of the tile have a ray that can be blocked at all:
//
//  1. The tile's hull.  Every shadow ray of pair (i, j) lies within
//     R_ij = max(rad_i, rad_j) of the centroid segment [c_i, c_j] (convexity;
//     rad = largest distance of a quadrature point from the centroid), and
//     that segment lies in H = conv(B_I u B_J), B_I the box of the centroids
//     of the tile's row block.  So every ray of the tile lies within
//     R_t = max rad (+ the cull margin) of H.
//  2. The tile's list.  A breadth-first walk of the tree from the start
//     frontier drops every node whose box is farther than R_t from H (a
//     separating axis: the coordinate axes and the centroid direction crossed
//     with them) -- no ray of the tile can pass its slab test, so the
//     reference never tests its triangles -- and then every triangle farther
//     than R_t + M_T from H (16 axes: coordinate axes, the normal, and the
//     edges crossed with the centroid direction and the coordinate axes),
//     M_T being the bound on how far rounding moves a hit of the reference's
//     Moller-Trumbore test (the pair-list argument of kernels_wave.cu).
//     Triangles of the groups of both blocks (when each block has a single
//     group) are skipped, as the reference skips a ray's own groups
//     (src/GPUBVH.jl:239-240).  Both tests run in FP32 with the allowance
//     em = S 2^-16 of the pair lists.
//  3. The pair mask.  When the list is not empty, each pair keeps a bit iff
//     one listed triangle survives the pair-list kernel's own tests (its leaf
//     box against the pair's capsule, the group skip, the separating-axis
//     test against the capsule): the pair's rays may then be blocked and go
//     through the ray pipeline; every other pair's rays are certainly visible.
//
// Output per tile: a class byte (kClsSlow: some pair may be blocked, with
// its mask of 32 words, row li -> bit lj; kClsNear: some pair is near field
// for mixed precision; kClsTiny: some pair's points may nearly coincide).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_lists.cuh"
#include "kernels.h"

namespace rvf {

namespace {

constexpr int kCullWarps = 4;

// Pair masks: the capsule test over all 16 axes (1) or the pair lists' 4 (0).
#ifndef RVF_MASK_FULL_AXES
#define RVF_MASK_FULL_AXES 0
#endif

// Position of the n-th (from 0) set bit of m (n < popc(m)): binary search
// over halves by population count.
__device__ __forceinline__ int nth_set_bit(uint32_t m, int n) {
  int pos = 0;
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const int c = __popc(m & ((1u << s) - 1u));
    if (n >= c) {
      n -= c;
      m >>= s;
      pos += s;
    }
  }
  return pos;
}

// H = conv(B_1 u B_2) of two boxes (FP32 centres c and half extents h).
struct HullF {
  float c[2][3], h[2][3];
  float d[3];  // c[1] - c[0]
};

// Projection interval of the hull on w.
__device__ __forceinline__ void hull_proj(const HullF& H, float wx, float wy, float wz, float& lo, float& hi) {
  const float aw0 = fabsf(wx), aw1 = fabsf(wy), aw2 = fabsf(wz);
  const float m0 = fmaf(H.c[0][0], wx, fmaf(H.c[0][1], wy, H.c[0][2] * wz));
  const float r0 = fmaf(H.h[0][0], aw0, fmaf(H.h[0][1], aw1, H.h[0][2] * aw2));
  const float m1 = fmaf(H.c[1][0], wx, fmaf(H.c[1][1], wy, H.c[1][2] * wz));
  const float r1 = fmaf(H.h[1][0], aw0, fmaf(H.h[1][1], aw1, H.h[1][2] * aw2));
  lo = fminf(m0 - r0, m1 - r1);
  hi = fmaxf(m0 + r0, m1 + r1);
}

// True when the interval [qlo, qhi] lies farther than m |w| from the hull
// along w (squares avoid the square root; m > 0).
__device__ __forceinline__ bool hull_gap(const HullF& H, float wx, float wy, float wz, float qlo, float qhi,
                                         float m) {
  float lo, hi;
  hull_proj(H, wx, wy, wz, lo, hi);
  const float gap = fmaxf(qlo - hi, lo - qhi);
  return gap > 0.0f && gap * gap > m * m * fmaf(wx, wx, fmaf(wy, wy, wz * wz));
}

// True when every point of the box lies farther than m from the hull.
__device__ __forceinline__ bool hull_misses_box(const HullF& H, const NodeF& nd, float m) {
  // coordinate axes
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float lo = fminf(H.c[0][k] - H.h[0][k], H.c[1][k] - H.h[1][k]);
    const float hi = fmaxf(H.c[0][k] + H.h[0][k], H.c[1][k] + H.h[1][k]);
    if (nd.lo[k] - hi > m || lo - nd.hi[k] > m) return true;
  }
  // the centroid direction crossed with each coordinate axis
  const float bc[3] = {0.5f * (nd.lo[0] + nd.hi[0]), 0.5f * (nd.lo[1] + nd.hi[1]), 0.5f * (nd.lo[2] + nd.hi[2])};
  const float bh[3] = {0.5f * (nd.hi[0] - nd.lo[0]), 0.5f * (nd.hi[1] - nd.lo[1]), 0.5f * (nd.hi[2] - nd.lo[2])};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float w[3] = {0.f, 0.f, 0.f};  // d x e_k
    w[(k + 1) % 3] = H.d[(k + 2) % 3];
    w[(k + 2) % 3] = -H.d[(k + 1) % 3];
    const float bm = fmaf(bc[0], w[0], fmaf(bc[1], w[1], bc[2] * w[2]));
    const float br = fmaf(bh[0], fabsf(w[0]), fmaf(bh[1], fabsf(w[1]), bh[2] * fabsf(w[2])));
    if (hull_gap(H, w[0], w[1], w[2], bm - br, bm + br, m)) return true;
  }
  return false;
}

__device__ __forceinline__ void tri_proj(const float4& p0, const float4& p1, const float4& p2, float wx, float wy,
                                         float wz, float& lo, float& hi) {
  const float q0 = fmaf(p0.x, wx, fmaf(p0.y, wy, p0.z * wz));
  const float q1 = fmaf(p1.x, wx, fmaf(p1.y, wy, p1.z * wz));
  const float q2 = fmaf(p2.x, wx, fmaf(p2.y, wy, p2.z * wz));
  lo = fminf(q0, fminf(q1, q2));
  hi = fmaxf(q0, fmaxf(q1, q2));
}

// True when the triangle lies farther than m from the hull.
__device__ __forceinline__ bool hull_misses_tri(const HullF& H, const float4& p0, const float4& p1, const float4& p2,
                                                float m) {
  float lo, hi;
  // coordinate axes
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float w[3] = {k == 0 ? 1.f : 0.f, k == 1 ? 1.f : 0.f, k == 2 ? 1.f : 0.f};
    tri_proj(p0, p1, p2, w[0], w[1], w[2], lo, hi);
    if (hull_gap(H, w[0], w[1], w[2], lo, hi, m)) return true;
  }
  const float e[3][3] = {{p1.x - p0.x, p1.y - p0.y, p1.z - p0.z},
                         {p2.x - p0.x, p2.y - p0.y, p2.z - p0.z},
                         {p2.x - p1.x, p2.y - p1.y, p2.z - p1.z}};
  // the normal
  {
    const float nx = e[0][1] * e[1][2] - e[0][2] * e[1][1];
    const float ny = e[0][2] * e[1][0] - e[0][0] * e[1][2];
    const float nz = e[0][0] * e[1][1] - e[0][1] * e[1][0];
    tri_proj(p0, p1, p2, nx, ny, nz, lo, hi);
    if (hull_gap(H, nx, ny, nz, lo, hi, m)) return true;
  }
  // the edges crossed with the centroid direction and with the coordinate axes
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float* f = e[a];
    {
      const float* d = H.d;
      const float wx = d[1] * f[2] - d[2] * f[1], wy = d[2] * f[0] - d[0] * f[2], wz = d[0] * f[1] - d[1] * f[0];
      tri_proj(p0, p1, p2, wx, wy, wz, lo, hi);
      if (hull_gap(H, wx, wy, wz, lo, hi, m)) return true;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float w[3] = {0.f, 0.f, 0.f};  // e_k x f
      w[(k + 1) % 3] = -f[(k + 2) % 3];
      w[(k + 2) % 3] = f[(k + 1) % 3];
      tri_proj(p0, p1, p2, w[0], w[1], w[2], lo, hi);
      if (hull_gap(H, w[0], w[1], w[2], lo, hi, m)) return true;
    }
  }
  return false;
}

}  // namespace

// One warp per tile, grid-stride over the tiles of one request.
// resident blocks per SM the classification is compiled for
#ifndef RVF_CULL_MIN_BLOCKS
#define RVF_CULL_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(kCullWarps * 32, RVF_CULL_MIN_BLOCKS) k_tile_class(const TileClassArgs a) {
  __shared__ int s_front[kCullWarps][2 * kTileFront];
  __shared__ int s_leaf[kCullWarps][kTileLeaves];
  __shared__ int s_list[kCullWarps][kTileTris];
  __shared__ int s_rleaf[kCullWarps][kTileLeaves];  // runs of the list: leaf node
  __shared__ int s_rspan[kCullWarps][kTileLeaves];  //   first list entry * 16 + count
  __shared__ int s_row[kCullWarps][kTileLeaves];    // a row's runs
  __shared__ float s_cap[kCullWarps][32][12];        // a row's pairs: capsule start, end, direction, R, group
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* front = s_front[warp];
  int* leaves = s_leaf[warp];
  int* list = s_list[warp];
  int* rleaf = s_rleaf[warp];
  int* rspan = s_rspan[warp];
  int* rowl = s_row[warp];
  const int64_t N = a.N;
  uint32_t n_culled = 0, n_masked = 0, n_over = 0;
  for (;;) {
    // tiles claimed one at a time: their costs differ by orders of magnitude
    unsigned long long tc = 0;
    if (lane == 0) tc = atomicAdd(a.claim, 1ull);
    const int64_t t = (int64_t)__shfl_sync(kFull, tc, 0);
    if (t >= a.n_tiles) break;
    int64_t bi, bj;
    tile_coords(t, a.nT, bi, bj);
    const int64_t ei = bi * kTile + lane, ej = bj * kTile + lane;
    const bool oki = ei < N, okj = ej < N;
    double ci[3] = {0.0, 0.0, 0.0}, cj[3] = {0.0, 0.0, 0.0};
    double ri = 0.0, rj = 0.0, di = 0.0, dj = 0.0;
    int32_t gi = 0, gj = 0;
    if (oki) {
      ci[0] = a.cen[3 * ei]; ci[1] = a.cen[3 * ei + 1]; ci[2] = a.cen[3 * ei + 2];
      ri = a.rad ? a.rad[ei] : 0.0;
      di = a.diam[ei];
      gi = a.group[ei];
    }
    if (okj) {
      cj[0] = a.cen[3 * ej]; cj[1] = a.cen[3 * ej + 1]; cj[2] = a.cen[3 * ej + 2];
      rj = a.rad ? a.rad[ej] : 0.0;
      dj = a.diam[ej];
      gj = a.group[ej];
    }
    // near-field and nearly coincident pairs (lane = j, loop over the row block)
    bool near = false, tiny = false;
    const bool classify_near = a.near_factor >= 0.0 || a.tiny_gap >= 0.0;  // mixed precision only
    for (int li = 0; li < (classify_near ? kTile : 0); ++li) {
      const double x0 = __shfl_sync(kFull, ci[0], li), x1 = __shfl_sync(kFull, ci[1], li),
                   x2 = __shfl_sync(kFull, ci[2], li);
      const double rr = __shfl_sync(kFull, ri, li), dd = __shfl_sync(kFull, di, li);
      const int64_t i = bi * kTile + li;
      if (!(okj && i < N && i < ej)) continue;
      const double d0 = cj[0] - x0, d1 = cj[1] - x1, d2 = cj[2] - x2;
      const double q = d0 * d0 + d1 * d1 + d2 * d2;
      if (a.near_factor >= 0.0) {
        const double dm = fmax(dd, dj) * a.near_factor;
        near = near || q < dm * dm;
      }
      if (a.tiny_gap >= 0.0) {
        const double s = rr + rj + a.tiny_gap;
        tiny = tiny || q <= s * s;
      }
    }
    uint8_t cls = (__any_sync(kFull, near) ? kClsNear : 0) | (__any_sync(kFull, tiny) ? kClsTiny : 0);
    bool all_ones = false;  // occlusion the tile cannot classify: every pair keeps its rays
    int nl = 0;             // listed triangles
    int nrun = 0;           // leaves with listed triangles (runs of the list)
    HullF H;                // the tile's hull (occlusion, 3-D)
    float rmaxJ = 0.0f;     // largest point radius of the column block
    if (a.occ && !a.dim3) {
      all_ones = true;
    } else if (a.occ) {
      // the hull: centroid boxes of the two blocks, rounded outwards to FP32
      double lo[2][3], hi[2][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[0][c] = oki ? ci[c] : INFINITY;
        hi[0][c] = oki ? ci[c] : -INFINITY;
        lo[1][c] = okj ? cj[c] : INFINITY;
        hi[1][c] = okj ? cj[c] : -INFINITY;
      }
      double rmax = fmax(ri, rj);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            lo[b][c] = fmin(lo[b][c], __shfl_xor_sync(kFull, lo[b][c], o));
            hi[b][c] = fmax(hi[b][c], __shfl_xor_sync(kFull, hi[b][c], o));
          }
        rmax = fmax(rmax, __shfl_xor_sync(kFull, rmax, o));
      }
      // one group per block: its triangles are skipped by every ray of the tile
      const int32_t gi0 = __shfl_sync(kFull, gi, 0), gj0 = __shfl_sync(kFull, gj, 0);
      const bool g_same = a.skip_groups && __all_sync(kFull, (!oki || gi == gi0) && (!okj || gj == gj0));
      double rj_max = rj;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) rj_max = fmax(rj_max, __shfl_xor_sync(kFull, rj_max, o));
      rmaxJ = __double2float_ru(rj_max);
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float l = __double2float_rd(lo[b][c]), h = __double2float_ru(hi[b][c]);
          H.c[b][c] = 0.5f * (l + h);
          H.h[b][c] = 0.5f * (h - l);
        }
#pragma unroll
      for (int c = 0; c < 3; ++c) H.d[c] = H.c[1][c] - H.c[0][c];
      const float Rt = __double2float_ru(rmax + a.cull_margin);
      const float mbox = Rt + a.sat_em;
      // breadth-first walk from the start frontier
      int* cur = front;
      int* nxt = front + kTileFront;
      if (lane < a.n_frontier) cur[lane] = a.frontier[lane];
      __syncwarp();
      int ncur = a.n_frontier, nleaf = 0;
      bool over = false;
      while (ncur > 0 && !over) {  // one tree level per round
        int nnext = 0;
        for (int b = 0; b < ncur; b += 32) {
          const int q = b + lane;
          bool pass = false, leaf = false;
          int k = 0, right = 0;
          if (q < ncur && cur[q] < a.n_nodes) {
            k = cur[q];
            const NodeF nd = a.nodesf[k];
            pass = !hull_misses_box(H, nd, mbox);
            leaf = (nd.ab & 15) > 0;
            if (pass && !leaf) right = a.nodesf[k + 1].miss;
          }
          const uint32_t ml = __ballot_sync(kFull, pass && leaf), mi = __ballot_sync(kFull, pass && !leaf);
          const int pl = nleaf + __popc(ml & lanemask_lt());
          if (pass && leaf && pl < kTileLeaves) leaves[pl] = k;
          nleaf += __popc(ml);
          const int pi = nnext + 2 * __popc(mi & lanemask_lt());
          if (pass && !leaf && pi + 1 < kTileFront) {
            nxt[pi] = k + 1;
            nxt[pi + 1] = right;
          }
          nnext += 2 * __popc(mi);
        }
        __syncwarp();
        if (nleaf > kTileLeaves || nnext > kTileFront) over = true;
        int* tmp = cur;
        cur = nxt;
        nxt = tmp;
        ncur = nnext;
      }
      // triangles of the candidate leaves, four leaves of up to 8 per round
      for (int b = 0; b < nleaf && !over; b += 4) {
        const int li = b + (lane >> 3), u8 = lane & 7;
        bool keep = false;
        int u = 0;
        if (li < nleaf) {
          const int32_t ab = a.nodesf[leaves[li]].ab;
          if (u8 < (ab & 15)) {
            u = (ab >> 4) + u8;
            const float4 p0 = a.sat[3 * u], p1 = a.sat[3 * u + 1], p2 = a.sat[3 * u + 2];
            const int32_t g = __float_as_int(p1.w);
            keep = !(g_same && (g == gi0 || g == gj0)) && !hull_misses_tri(H, p0, p1, p2, Rt + p0.w + a.sat_em);
          }
        }
        const uint32_t m = __ballot_sync(kFull, keep);
        const int pos = nl + __popc(m & lanemask_lt());
        if (keep && pos < kTileTris) list[pos] = u;
        // one run per leaf of this round that kept triangles
        if (lane < 4 && b + lane < nleaf) {
          const uint32_t lm = (m >> (8 * lane)) & 0xffu;
          if (lm) {
            int before = 0;
            for (int k = 0; k < lane; ++k) before += ((m >> (8 * k)) & 0xffu) ? 1 : 0;
            const int r = nrun + before;
            rleaf[r] = leaves[b + lane];
            rspan[r] = (nl + __popc(m & ((1u << (8 * lane)) - 1u))) * 16 + __popc(lm);
          }
        }
        int nnew = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) nnew += ((m >> (8 * k)) & 0xffu) ? 1 : 0;
        nrun += nnew;
        nl += __popc(m);
        if (nl > kTileTris) over = true;
        __syncwarp();
      }
      __syncwarp();
      all_ones = over;
    }
    if (all_ones) {
      cls |= kClsSlow;
      a.mask[t * kTile + lane] = 0xffffffffu;
      n_masked += 32;
      n_over += lane == 0 ? 1 : 0;
    } else if (nl > 0) {
      // per pair: some listed triangle survives the pair-list tests.  Row by
      // row, the warp first keeps the runs (leaves with listed triangles)
      // whose box the row's own hull (its centroid and the column block's box,
      // radius max(rad_i, rad_J)) can reach, 32 at a time; each lane then
      // tests its pair against those leaves and their triangles.
      cls |= kClsSlow;
      for (int li = 0; li < kTile; ++li) {
        const int64_t i = bi * kTile + li;
        const double x0 = __shfl_sync(kFull, ci[0], li), x1 = __shfl_sync(kFull, ci[1], li),
                     x2 = __shfl_sync(kFull, ci[2], li);
        const double rr = __shfl_sync(kFull, ri, li);
        const int32_t g_i = __shfl_sync(kFull, gi, li);
        if (i >= N) {
          if (lane == 0) a.mask[t * kTile + li] = 0u;
          continue;
        }
        HullF Hr;
        const double xr[3] = {x0, x1, x2};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float l = __double2float_rd(xr[c]), h = __double2float_ru(xr[c]);
          Hr.c[0][c] = 0.5f * (l + h);
          Hr.h[0][c] = 0.5f * (h - l);
          Hr.c[1][c] = H.c[1][c];
          Hr.h[1][c] = H.h[1][c];
          Hr.d[c] = Hr.c[1][c] - Hr.c[0][c];
        }
        const float Rr = fmaxf(__double2float_ru(rr), rmaxJ) + __double2float_ru(a.cull_margin) + a.sat_em;
        int nr = 0;
        for (int b = 0; b < nrun; b += 32) {
          const int r = b + lane;
          const bool keep = r < nrun && !hull_misses_box(Hr, a.nodesf[rleaf[r]], Rr);
          const uint32_t m = __ballot_sync(kFull, keep);
          if (keep) rowl[nr + __popc(m & lanemask_lt())] = r;
          nr += __popc(m);
        }
        __syncwarp();
        const bool valid = okj && i < ej;
        CapsuleF cap{};
        float bf[3] = {0.f, 0.f, 0.f}, df[3] = {0.f, 0.f, 0.f};
        float Rf = 0.0f;
        if (valid && nr > 0) {
          const double R = fmax(rr, rj) + a.cull_margin;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double dd = cj[c] - xr[c];
            cap.A[c] = (float)xr[c];
            bf[c] = (float)cj[c];
            cap.zero[c] = dd == 0.0;
            cap.inv[c] = cap.zero[c] ? 0.0f : (float)(1.0 / dd);
          }
          cap.R = (float)R + a.sat_em;
#pragma unroll
          for (int c = 0; c < 3; ++c) df[c] = bf[c] - cap.A[c];
          Rf = (float)R;
        }
        // Each pair's capsule against each run's leaf (lanes are pairs), then
        // the (pair, triangle) tests of each run dealt out to the lanes --
        // lane w of a round takes test w: pair w / count, triangle w % count
        // -- so the lanes stay busy however few pairs reach a leaf.  A pair
        // leaves once one of its triangles survives.
        float* cd = s_cap[warp][lane];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cd[c] = cap.A[c];
          cd[3 + c] = bf[c];
          cd[6 + c] = df[c];
        }
        cd[9] = Rf;
        cd[10] = __int_as_float(gj);
        const uint32_t none = __ballot_sync(kFull, !valid);
        // the pairs reaching each run's leaf, in the walk's leaf array (not
        // needed once the runs are recorded)
        uint32_t* pms = reinterpret_cast<uint32_t*>(leaves);
        for (int e = 0; e < nr; ++e) {
          const bool pass = valid && !capsule_misses_box(cap, a.nodesf[rleaf[rowl[e]]]);
          const uint32_t pm = __ballot_sync(kFull, pass);
          if (lane == 0) pms[e] = pm;
        }
        __syncwarp();
        uint32_t hit = 0;
        for (int e = 0; e < nr; ++e) {
          const uint32_t pm = pms[e] & ~hit & ~none;
          if (pm == 0) continue;  // warp-uniform
          const int span = rspan[rowl[e]], k0 = span >> 4, cnt = span & 15;
          const int total = __popc(pm) * cnt;
          uint32_t h = 0;
          for (int w = lane; w < total; w += 32) {
            const int pi = w / cnt, ti = w - pi * cnt;
            const int p = nth_set_bit(pm, pi);
            const float* q = s_cap[warp][p];
            const int u = list[k0 + ti];
            const float4 p0 = a.sat[3 * u], p1 = a.sat[3 * u + 1], p2 = a.sat[3 * u + 2];
            const int32_t g = __float_as_int(p1.w);
            if (a.skip_groups && (g == g_i || g == __float_as_int(q[10]))) continue;
            const float qa[3] = {q[0], q[1], q[2]}, qb[3] = {q[3], q[4], q[5]}, qd[3] = {q[6], q[7], q[8]};
            const bool miss = RVF_MASK_FULL_AXES ? pair_misses_tri_full(qa, qb, qd, q[9], a.sat_em, p0, p1, p2)
                                                 : pair_misses_tri(qa, qb, qd, q[9], a.sat_em, p0, p1, p2);
            if (!miss) h |= 1u << p;
          }
          hit |= __reduce_or_sync(kFull, h);
        }
        const bool bit = (hit >> lane) & 1u;
        __syncwarp();
        const uint32_t m = __ballot_sync(kFull, bit);
        if (lane == 0) {
          a.mask[t * kTile + li] = m;
          n_masked += __popc(m);
        }
      }
    } else if (a.occ) {
      ++n_culled;
    }
    if (lane == 0) a.cls[t] = cls;
  }
  if (a.counters) {
    const uint64_t s_c = warp_sum_u64(lane == 0 ? n_culled : 0), s_m = warp_sum_u64(n_masked),
                   s_o = warp_sum_u64(n_over);
    if (lane == 0) {
      atomicAdd(a.counters + 0, s_c);
      atomicAdd(a.counters + 1, s_m);
      atomicAdd(a.counters + 2, s_o);
    }
  }
}

cudaError_t launch_tile_class(const TileClassArgs& a, int sm_count, cudaStream_t st) {
  if (a.n_tiles <= 0) return cudaSuccess;
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_class, kCullWarps * 32, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const int64_t want = (a.n_tiles + kCullWarps - 1) / kCullWarps;
  const int grid = (int)std::min<int64_t>(want, (int64_t)sm_count * per_sm);
  const cudaError_t e = cudaMemsetAsync(a.claim, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  k_tile_class<<<(unsigned)grid, kCullWarps * 32, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace rvf
