// device_trace.cuh -- compacted shadow-ray batches traced one ray per lane.
//
// The pair kernels do not trace a ray when they form it.  A ray whose
// segment misses the root box of the obstruction BVH is visible (the
// reference's walk, src/GPUBVH.jl:216-282, ends at the root); every other ray
// is appended to a per-warp buffer, and a full buffer of 32 rays is traced at
// once, one ray per lane:
//   * interior phase: each lane walks its own ray through the pre-order tree
//     (slab test, descend to node+1 on a pass, jump to the miss link on a
//     miss), collecting the leaves whose boxes it passes, until the end
//     (up to kLeafSlots of them per round, so that lanes which reach a leaf
//     early keep walking while the others catch up);
//   * leaf phase: the primitives of all collected leaves of the warp are
//     dealt out to the 32 lanes (a lane may test another lane's ray, read from
//     the warp's shared-memory ray bank), so a leaf of 8 triangles costs one
//     primitive test per lane instead of eight on one lane.
// The (ray, triangle) tests are the reference walk's tests up to its first
// hit plus at most the rest of that round's collected leaves, so the any-hit
// answer is the reference's.
#pragma once

#include "device_mixed.cuh"

namespace rvf {

// Per-warp shared-memory scratch: the ray bank with the leaf-phase work
// lists (RayBank) and, for the fused kernel, the compaction buffers.  3D FP64 rays use o/d/tmax; 2-D segments store
// their two end points in o (x, y) and d (x, y); FP32 rays use the *f arrays.
constexpr int kLeafSlots = 4;     // passed leaves a lane collects per round (FP64 traversal)
constexpr int kLeafSlotsF = 4;    // same, FP32 traversal (more slots cost more occupancy than they save)

// Per-warp ray bank and leaf-phase work lists for L collected leaves per lane.
template <int L>
struct RayBankT {
  union {
    struct {
      double o[3][32];
      double d[3][32];
      double tmax[32];
    } r64;  // FP64 rays; 2-D segments keep their end points in o (x, y) and d (x, y)
    struct {
      float o[3][32];
      float d[3][32];
      float tmax[32];
      float delta[32];
    } r32;
  };
  int32_t gi[32], gj[32];
  const void* prims[32];         // each ray's primitive array (rays of one warp may come from different meshes)
  int32_t first[L][32];          // collected leaves: first primitive
  uint16_t item[32 * L * 8];     // leaf phase: (lane, leaf slot, offset) per test
  uint8_t hit[32];
  uint8_t unsure[32];
};
using RayBank = RayBankT<kLeafSlots>;
using RayBankF = RayBankT<kLeafSlotsF>;

struct WarpScratch {
  RayBank bank;
  double contrib[2][64];  // [0] FP64 / main buffer, [1] FP32 buffer (mixed)
  uint32_t meta[2][64];
};

// ---------------------------------------------------------------------------
// Node sources for the traversal.  In shared memory the 16-byte chunks of
// each node are XOR-swizzled: lanes of a warp walk different nodes, and with
// the plain layout chunk c of every 64-byte node falls into one of only two
// of the eight 16-byte bank groups (one of four for 32-byte nodes), so a
// warp's node load needs up to 4x the ideal shared-memory wavefronts.
// Chunk c of node k is stored at chunk 4k + (c ^ ((k >> 1) & 3)) (FP64) or
// 2k + (c ^ ((k >> 2) & 1)) (FP32), which spreads any chunk over all eight
// groups as k varies.
// ---------------------------------------------------------------------------
template <typename Node>
struct GlobalNodes {
  const Node* p;
  __device__ __forceinline__ Node operator()(int k) const { return p[k]; }
};

template <typename Node>
struct SwizNodes {
  static constexpr int C = sizeof(Node) / 16;  // 16-byte chunks per node (4 or 2)
  const int4* p;
  __device__ static __forceinline__ int slot(int k, int c) {
    return C == 4 ? 4 * k + (c ^ ((k >> 1) & 3)) : 2 * k + (c ^ ((k >> 2) & 1));
  }
  __device__ __forceinline__ Node operator()(int k) const {
    union {
      int4 v[C];
      Node n;
    } u;
#pragma unroll
    for (int c = 0; c < C; ++c) u.v[c] = p[slot(k, c)];
    return u.n;
  }
  // block-cooperative copy of n nodes from global memory into dst
  __device__ static void fill(int4* dst, const Node* src, int n) {
    const int4* s4 = reinterpret_cast<const int4*>(src);
    for (int t = threadIdx.x; t < n * C; t += blockDim.x) dst[slot(t / C, t % C)] = s4[t];
  }
};

// buffer entry: owner lane (5 bits), swapped (1 bit), source point p (6 bits),
// destination point q (6 bits)
__device__ __forceinline__ uint32_t enc_entry(int lane, bool sw, int p, int q) {
  return (uint32_t)lane | ((uint32_t)sw << 5) | ((uint32_t)p << 6) | ((uint32_t)q << 12);
}
__device__ __forceinline__ int ent_lane(uint32_t e) { return (int)(e & 31u); }
__device__ __forceinline__ bool ent_sw(uint32_t e) { return ((e >> 5) & 1u) != 0; }
__device__ __forceinline__ int ent_p(uint32_t e) { return (int)((e >> 6) & 63u); }
__device__ __forceinline__ int ent_q(uint32_t e) { return (int)((e >> 12) & 63u); }

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Appends the lanes with `push` to buffer b (count n, warp-uniform).
__device__ __forceinline__ void buf_push(WarpScratch& ws, int b, int& n, bool push, uint32_t meta, double contrib) {
  const uint32_t m = __ballot_sync(kFull, push);
  if (m == 0) return;
  if (push) {
    const int pos = n + __popc(m & lanemask_lt());
    ws.meta[b][pos] = meta;
    ws.contrib[b][pos] = contrib;
  }
  n += __popc(m);
  __syncwarp();
}

// After the first `used` entries (used <= 32) were consumed: move the rest down.
__device__ __forceinline__ void buf_shift(WarpScratch& ws, int b, int& n, int used) {
  const int rest = n - used;
  const int lane = threadIdx.x & 31;
  uint32_t m = 0;
  double c = 0.0;
  if (lane < rest) {
    m = ws.meta[b][used + lane];
    c = ws.contrib[b][used + lane];
  }
  __syncwarp();
  if (lane < rest) {
    ws.meta[b][lane] = m;
    ws.contrib[b][lane] = c;
  }
  n = rest;
  __syncwarp();
}

// Owners add the contributions of their visible entries, in entry order.
__device__ __forceinline__ void buf_collect(const WarpScratch& ws, int b, int n, uint32_t visible, double& acc) {
  const int lane = threadIdx.x & 31;
  for (int t = 0; t < n; ++t) {
    const uint32_t e = ws.meta[b][t];
    if (ent_lane(e) == lane && ((visible >> t) & 1u)) acc += ws.contrib[b][t];
  }
}

// ---------------------------------------------------------------------------
// Generic batch traversal.  Pol provides
//   node(const Node&) -> int   kHit / kMiss / kUnsure for the lane's own ray
// (nodes(k) returns node k: GlobalNodes or SwizNodes)
//   leaf(const Node&, int& first, int& count)
//   prim(ws, owner, k) -> int  kHit / kMiss / kUnsure for owner's ray
// Returns kHit (blocked), kMiss (visible) or kUnsure (FP32 only: some
// decision of the walk was not certain and no certain hit was found).
// ---------------------------------------------------------------------------
template <typename Src, typename Pol, int L>
__device__ __forceinline__ int trace_batch(bool have, const Src& nodes, int n_nodes, RayBankT<L>& ws, Pol& pol,
                                           TravCount& cnt) {
  static_assert(L <= 8, "leaf slot index is 3 bits");
  const int lane = threadIdx.x & 31;
  ws.hit[lane] = 0;
  ws.unsure[lane] = 0;
  __syncwarp();
  int k = 0;
  bool done = !have;
  bool unsure = false;
  for (;;) {
    // interior phase: walk until kLeafSlots passed leaves are collected or the walk ends
    int nl = 0, total_own = 0;
    uint32_t counts = 0;  // 4 bits per collected leaf
    while (!done && nl < L) {
      const auto nd = nodes(k);
      ++cnt.nodes;
      const int s = pol.node(nd);
      int first, count;
      pol.leaf(nd, first, count);
      if (s == kUnsure) {
        unsure = true;
        ++cnt.unsure_slab;
        done = true;
      } else if (s == kHit && count > 0) {
        ws.first[nl][lane] = first;
        counts |= (uint32_t)count << (4 * nl);
        total_own += count;
        ++nl;
        k = pol.miss(nd);
      } else {
        // miss links point forward (checked when the tree is uploaded), so k grows
        k = (s == kHit) ? k + 1 : pol.miss(nd);
      }
      if (k >= n_nodes) done = true;
    }
    // leaf phase: deal the collected (ray, primitive) tests out to the lanes
    int incl = total_own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(kFull, incl, 31);
    if (total == 0) {
      if (!__any_sync(kFull, !done)) break;
      continue;
    }
    int pos = incl - total_own;
    for (int sl = 0; sl < nl; ++sl) {
      const int c = (int)((counts >> (4 * sl)) & 15u);
      for (int u = 0; u < c; ++u) ws.item[pos++] = (uint16_t)((lane << 6) | (sl << 3) | u);
    }
    __syncwarp();
    for (int base = 0; base < total; base += 32) {
      const int t = base + lane;
      if (t < total) {
        const int it = ws.item[t];
        const int o = it >> 6;
        const int r = pol.prim(ws, o, ws.first[(it >> 3) & 7][o] + (it & 7), cnt);
        if (r == kHit) ws.hit[o] = 1;
        else if (r == kUnsure) ws.unsure[o] = 1;
      }
    }
    __syncwarp();
    if (ws.hit[lane]) done = true;
    if (!__any_sync(kFull, !done)) break;
  }
  __syncwarp();
  const bool hit = ws.hit[lane] != 0;
  unsure = unsure || ws.unsure[lane] != 0;
  __syncwarp();
  if (!have) return kMiss;
  if (hit) return kHit;
  return unsure ? kUnsure : kMiss;
}

// FP64 3D rays, reference arithmetic (slab_d / mt_d).
struct PolD3 {
  RayD R;
  const TriD* tris;
  template <typename B>
  __device__ __forceinline__ void store(B& ws, int lane, int32_t gi, int32_t gj) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ws.r64.o[c][lane] = R.o[c];
      ws.r64.d[c][lane] = R.d[c];
    }
    ws.r64.tmax[lane] = R.tmax;
    ws.gi[lane] = gi;
    ws.gj[lane] = gj;
    ws.prims[lane] = tris;
  }
  __device__ __forceinline__ int node(const NodeD& nd) const { return slab_d(nd, R) ? kHit : kMiss; }
  __device__ __forceinline__ void leaf(const NodeD& nd, int& first, int& count) const {
    first = nd.a;
    count = nd.b;
  }
  __device__ __forceinline__ int miss(const NodeD& nd) const { return nd.miss; }
  template <typename B>
  __device__ __forceinline__ int prim(const B& ws, int o, int k, TravCount& cnt) const {
    const TriD tr = static_cast<const TriD*>(ws.prims[o])[k];
    if (tr.group == ws.gi[o] || tr.group == ws.gj[o]) return kMiss;
    ++cnt.prims;
    RayD Q;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Q.o[c] = ws.r64.o[c][o];
      Q.d[c] = ws.r64.d[c][o];
    }
    Q.tmax = ws.r64.tmax[o];
    return mt_d(tr, Q) ? kHit : kMiss;
  }
  // the lane's own ray against a triangle (pair lists: groups already excluded)
  __device__ __forceinline__ int prim_direct(const TriD& tr) const { return mt_d(tr, R) ? kHit : kMiss; }
};

// FP64 2-D segments (src/BVH.jl:265-322): a = first end point, b = second,
// exactly as seg_blocks receives them.
struct PolD2 {
  double a[2], b[2];
  const SegD* segs;
  template <typename B>
  __device__ __forceinline__ void store(B& ws, int lane, int32_t gi, int32_t gj) const {
    ws.r64.o[0][lane] = a[0];
    ws.r64.o[1][lane] = a[1];
    ws.r64.d[0][lane] = b[0];
    ws.r64.d[1][lane] = b[1];
    ws.gi[lane] = gi;
    ws.gj[lane] = gj;
    ws.prims[lane] = segs;
  }
  __device__ __forceinline__ int node(const NodeD& nd) const {
    const double xlo = fmin(a[0], b[0]), xhi = fmax(a[0], b[0]);
    const double ylo = fmin(a[1], b[1]), yhi = fmax(a[1], b[1]);
    return (nd.lo[0] > xhi || nd.hi[0] < xlo || nd.lo[1] > yhi || nd.hi[1] < ylo) ? kMiss : kHit;
  }
  __device__ __forceinline__ void leaf(const NodeD& nd, int& first, int& count) const {
    first = nd.a;
    count = nd.b;
  }
  __device__ __forceinline__ int miss(const NodeD& nd) const { return nd.miss; }
  template <typename B>
  __device__ __forceinline__ int prim(const B& ws, int o, int k, TravCount& cnt) const {
    const SegD sg = static_cast<const SegD*>(ws.prims[o])[k];
    if (sg.group == ws.gi[o] || sg.group == ws.gj[o]) return kMiss;
    ++cnt.prims;
    const double xa[2] = {ws.r64.o[0][o], ws.r64.o[1][o]}, xb[2] = {ws.r64.d[0][o], ws.r64.d[1][o]};
    return seg_blocks(sg, xa, xb) ? kHit : kMiss;
  }
};

// FP32 3D rays with certified decisions (slab_f / mt_f).
struct PolF3 {
  RayF R;
  const TriF* tris;
  template <typename B>
  __device__ __forceinline__ void store(B& ws, int lane, int32_t gi, int32_t gj) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ws.r32.o[c][lane] = R.o[c];
      ws.r32.d[c][lane] = R.d[c];
    }
    ws.r32.tmax[lane] = R.tmax;
    ws.r32.delta[lane] = R.delta;
    ws.gi[lane] = gi;
    ws.gj[lane] = gj;
    ws.prims[lane] = tris;
  }
  __device__ __forceinline__ int node(const NodeF& nd) const { return slab_f(nd, R); }
  __device__ __forceinline__ void leaf(const NodeF& nd, int& first, int& count) const {
    first = nd.ab >> 4;
    count = nd.ab & 15;
  }
  __device__ __forceinline__ int miss(const NodeF& nd) const { return nd.miss; }
  template <typename B>
  __device__ __forceinline__ int prim(const B& ws, int o, int k, TravCount& cnt) const {
    const TriF tr = static_cast<const TriF*>(ws.prims[o])[k];
    if (tr.group == ws.gi[o] || tr.group == ws.gj[o]) return kMiss;
    ++cnt.prims;
    RayF Q;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Q.o[c] = ws.r32.o[c][o];
      Q.d[c] = ws.r32.d[c][o];
    }
    Q.tmax = ws.r32.tmax[o];
    Q.delta = ws.r32.delta[o];
    const int r = mt_f(tr, Q);
    if (r == kUnsure) ++cnt.unsure_prim;
    return r;
  }
  // the lane's own ray against a triangle (pair lists: groups already excluded)
  __device__ __forceinline__ int prim_direct(const TriF& tr) const { return mt_f(tr, R); }
};

}  // namespace rvf
