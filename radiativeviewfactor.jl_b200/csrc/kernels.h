// kernels.h -- launch arguments and launchers of the librvf_b200 kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rvf_host.h"

namespace rvf {

// Wavefront pipeline state (kernels_wave.cu).
enum : int {
  kCtrTile = 0,    // tile claims
  kCtrResv = 1,    // reserved queue records (low 38 bits) and pending-pair slots (high bits)
  kCtrSpare = 2,
  kCtrRec64 = 3,   // records in the FP64 queue
  kCtrRec32 = 4,   // records in the FP32 queue
  kCtrSlots = 5,   // pending-pair slots in use
  kCtrHead64 = 6,  // traversal progress, FP64 queue
  kCtrHead32 = 7,  // traversal progress, FP32 queue
  kCtrPool = 8,    // pair-list pool entries taken
  kCtrCount = 9
};

// A pair with queued rays: its request (mesh) within the launch, internal
// element indices and the sum of its immediately decided terms.
struct PendSlot {
  int32_t i, j;
  int32_t req, pad;
  double acc;
};

// Per pending pair (3-D triangles): the triangles a shadow ray of the pair
// can hit under the reference's FP64 tests (primitive indices in leaf order),
// built by the list kernel after the generation into a pool: entries
// pool[off, off + n).  n = -1: no list (too long, or the pool is full); the
// pair's rays walk the tree.
constexpr int kListCap = 256;    // longest list kept
constexpr int kListFront = 64;   // breadth-first frontier of the list kernel's walk
constexpr int kListLeaves = 64;  // candidate leaves per pair
struct PairList {
  int32_t n;
  int32_t off;
};

// Tile classes (kernels_cull.cu): per 32 x 32 tile of the upper triangle a
// class byte and, for kClsSlow tiles, 32 mask words (row li of the tile ->
// bit lj set when some shadow ray of the pair may be blocked).
enum : uint8_t {
  kClsSlow = 1,  // some pair's rays may be blocked: the ray pipeline, with the mask
  kClsNear = 2,  // some pair is near field (mixed precision integrates it in FP64)
  kClsTiny = 4,  // some pair's points may nearly coincide (mixed precision: FP64)
};
constexpr int kTileLeaves = 256;  // candidate leaves of a tile's walk
constexpr int kTileFront = 256;   // breadth-first frontier of a tile's walk
constexpr int kTileTris = 1024;   // listed triangles of a tile (more: every pair keeps its rays)

struct TileClassArgs {
  int64_t N, nT, n_tiles;
  const double* cen;
  const double* rad;
  const double* diam;
  const int32_t* group;
  double near_factor;  // < 0: no near-field classification
  double tiny_gap;     // pairs closer than rad_i + rad_j + tiny_gap are kClsTiny
  double cull_margin;
  bool occ, dim3;
  bool skip_groups;  // rays skip the triangles of their elements' groups (false: a ray may hit any triangle)
  const NodeF* nodesf;
  int n_nodes;
  const int32_t* frontier;
  int n_frontier;
  const int32_t* leaf_of;
  const float4* sat;
  float sat_em;
  uint8_t* cls;    // n_tiles
  uint32_t* mask;  // n_tiles x 32
  unsigned long long* claim;  // zeroed tile counter (warps claim tiles one at a time)
  unsigned long long* counters;  // [culled tiles, masked pairs, tiles left unclassified]
};

struct WaveQ {
  uint64_t* rec64;  // FP64 ray queue
  uint64_t* rec32;  // FP32 ray queue (mixed precision)
  int64_t cap;      // records per queue
  PendSlot* slots;
  unsigned long long* vis;  // slots x vis_words visibility bits, bit p*pmax+q
  PairList* plist;          // per-slot lists, or null (every ray walks the tree)
  int32_t* pool;            // list entries
  int64_t pool_cap;
  int64_t scap;
  int vis_words;
  unsigned long long* ctr;  // kCtrCount counters
};

struct PrepArgs {
  int64_t N;
  int pmax;
  const double* coords;   // 3 x n_nodes
  const int32_t* enodes;  // N x 8, 0-based node ids
  const int8_t* fam;
  // rules (device pointers)
  const double *qx, *qe, *qw, *tx, *te, *tw, *lx, *lw;
  int nquadpts, ntripts, nline;
  const int32_t* orig;  // internal -> caller's element index (null: identity)
  // outputs
  double* tab;     // tiles x kComp x pmax x 32
  double* area;
  double* area_orig;    // areas in the caller's order (or null)
  int8_t* np;
  uint8_t* flat;
  double* nrm;     // 3N
  double* cen;     // 3N
  double* diam;    // N
  double* rad;     // N: largest distance of a quadrature point from the centroid (or null)
  int* err;
};

struct PairArgs {
  int64_t N;
  int64_t nT;       // tiles per side
  int64_t n_tiles;  // nT (nT + 1) / 2
  int pmax;
  bool dim3;
  const double* tab;
  const int8_t* np;
  const double* area;
  const uint8_t* flat;
  const double* nrm;
  const int32_t* group;
  const int32_t* orig;  // internal -> caller's element index (null: identity)
  const double* cen;    // pair culling: element centroids and point radii (or null)
  const double* rad;
  double cull_margin;
  double* F;        // N x N column-major, caller's element order
  // occlusion (n_nodes == 0: none)
  const NodeD* nodes;
  int n_nodes;
  bool nodes_in_smem;
  const TriD* tris;
  const SegD* segs;
  unsigned long long* tile_counter;
  unsigned long long* counters;  // [point pairs, rays, node visits, primitive tests]
  int* err;
  uint8_t* ray_log;              // device, or null
  int log_pm;
  WaveQ q;                       // wavefront queues (the fused kernel ignores them)
  int64_t tile0;                 // batched generation: first tile of this request in the launch
  const uint8_t* tcls;           // tile classes and masks (kernels_cull.cu), or null
  const uint32_t* tmask;
  bool fast_done;                // tiles without ray work were integrated by k_fast_fp64: skip them
  int fast_groups;               // k_fast_fp64 tasks per tile (1, 2 or 4 row groups)
  const int32_t* work;           // the tiles of the chunked pipeline in order (null: every tile)
};

struct RedArgs {
  int64_t N;
  int G;
  int n_chunks;
  const double* F;
  const double* area;
  const int64_t* member_off;  // G+1
  const int32_t* members;     // element ids grouped by group (ascending within a group)
  double* part;               // n_chunks x G x N
  double* rowgroup;           // G x N
  double* rowsum;             // N
  double* Fgroup;             // G x G column-major
  double* Agroup;             // G
};

struct PrepF32Args {
  int64_t N;
  int pmax;
  const double* tab;
  float* tabf;
  const int8_t* np;
  const double* cen;
};

struct MixedArgs {
  int64_t N, nT, n_tiles;
  int pmax;
  const double* tab;   // FP64 table (near field, grazing, re-tests)
  const float* tabf;   // FP32 table (offsets from the element centroid)
  const int8_t* np;
  const double* area;
  const uint8_t* flat;
  const double* nrm;
  const double* cen;
  const double* diam;
  double near_factor;
  const double* rad;
  double cull_margin;
  double tiny_gap;  // pairs closer than rad_i + rad_j + tiny_gap run in FP64 (as near-field pairs)
  const int32_t* group;
  const int32_t* orig;
  double* F;
  const NodeD* nodes;
  const NodeF* nodesf;
  int n_nodes;
  bool nodesf_in_smem;
  const TriD* tris;
  const TriF* trisf;
  float delta;  // absolute FP32 position error allowance (2^-20 x scene extent)
  unsigned long long* tile_counter;
  unsigned long long* counters;  // [-, rays, node tests, prim tests, FP64 rays, near pairs, grazing pp, unsure rays]
  int* err;
  uint8_t* ray_log;
  int log_pm;
  WaveQ q;
  int64_t tile0;
  const uint8_t* tcls;  // tile classes and masks (kernels_cull.cu), or null
  const uint32_t* tmask;
  bool fast_done;       // tiles without ray work were integrated by k_fast_mixed: skip them
  int fast_groups;      // k_fast_mixed tasks per tile (1, 2 or 4 row groups)
  const int32_t* work;  // the tiles of the chunked pipeline in order (null: every tile)
};

struct TraceArgs {
  int64_t N;
  int pmax;
  bool dim3;
  const double* tab;
  const float* tabf;
  const double* cen;
  const int32_t* group;
  const int32_t* orig;
  const NodeD* nodes;
  const NodeF* nodesf;
  int n_nodes;
  bool nodes_in_smem;
  const TriD* tris;
  const TriF* trisf;
  const SegD* segs;
  float delta;
  // pair lists (3-D): leaf node of each primitive (leaf order), its corners
  // in FP32 with its margin (sat), the generation's capsule radius and
  // margin, and the FP32 rounding allowance of the separating-axis test
  const int32_t* leaf_of;
  const float4* sat;
  const int32_t* frontier;  // start nodes of the list walk (<= 32)
  int n_frontier;
  const double* rad;
  double cull_margin;
  float sat_em;
  WaveQ q;
  unsigned long long* counters;
  uint8_t* ray_log;
  int log_pm;
};

struct ResolveArgs {
  int64_t N;
  int pmax;
  bool dim3;
  const double* tab;
  const float* tabf;
  const double* cen;
  const double* diam;
  double near_factor;
  const double* area;
  const int32_t* orig;
  double* F;
  WaveQ q;
};

// One launch of the pair pipeline over the tiles of one or more requests
// (meshes): global tile t belongs to request r when tile_base[r] <= t <
// tile_base[r+1], and is tile t - tile_base[r] + tile0 of that request.
// The launch blocks live in device memory so that a captured CUDA graph can
// be replayed with new contents.
constexpr int kMaxBatch = 64;  // requests per launch

struct GenBatch {
  const PairArgs* reqs;    // FP64 generation
  const MixedArgs* mreqs;  // mixed generation
  const int64_t* tile_base;
  int n_req;
  int pmax_max;            // shared-memory layout and queue reservation
  int64_t total_tiles;
  int claim_retries;       // compare-and-swap attempts of a tile claim before it gives up
  WaveQ q;
  unsigned long long* counters;
  int* err;
};

struct TraceBatch {
  const TraceArgs* reqs;
  int n_req;
  // one request only: its BVH staged in shared memory, per traversal precision
  bool nodes64_in_smem, nodes32_in_smem;
  const NodeD* smem_nodes64;
  const NodeF* smem_nodes32;
  int n_nodes_smem;
  WaveQ q;
  unsigned long long* counters;
};

struct ResolveBatch {
  const ResolveArgs* reqs;
  int n_req;
  WaveQ q;
};

// Kernel shapes of one launch class (fixed within a captured graph).
struct WaveShape {
  bool mixed, dim3, occ;
  int pmax_max;
  bool trace64_nodes_smem, trace32_nodes_smem;
  int n_nodes_smem;
  int gen_bps, trace_bps;  // blocks per SM of the generation / traversal grids (0 = occupancy limit)
};

size_t gen_smem_bytes(bool mixed, int pmax, bool occ);
size_t trace_smem_bytes(bool fp32, int n_nodes_smem);
// Generation, traversal and resolve of one chunk; the batch structs are
// device pointers.
cudaError_t launch_gen(const WaveShape& sh, const GenBatch* g, int sm_count, cudaStream_t st);
cudaError_t launch_trace(const WaveShape& sh, const TraceBatch* t, bool fp32, int sm_count, cudaStream_t st);
cudaError_t launch_resolve(const WaveShape& sh, const ResolveBatch* r, int sm_count, cudaStream_t st);
// Pair lists of the chunk's pending pairs (3-D triangles with occlusion).
cudaError_t launch_plist(const TraceBatch* t, int sm_count, cudaStream_t st);
// Tile classes and masks of one request (before its first chunk).
cudaError_t launch_tile_class(const TileClassArgs& a, int sm_count, cudaStream_t st);
// Every tile of one request that needs no shadow-ray work (its class), one
// warp per task (a.fast_groups tasks per tile), before the request's chunks;
// qb points of the destination element per lane block (fast_qb_default: by
// the rule's size; fast_qb_supported: the compiled blocks); task_ctr: a
// zeroed counter.
int fast_qb_default(bool mixed, int pmax);
cudaError_t preload_fast();  // loads every compiled shape (before timing them)
bool fast_qb_supported(bool mixed, int qb);
cudaError_t launch_fast(bool mixed, bool dim3, bool occ, int qb, const PairArgs& a, const MixedArgs& m,
                        unsigned long long* task_ctr, unsigned long long* counters, int sm_count, cudaStream_t st);

// A Quad8 pair sharing corner nodes (src/DuffyKernel.jl:95-115), i < j in the
// caller's order (the reference integrates with elem_i = the lower index).
struct DuffyPair {
  int32_t i, j;      // caller's element indices
  int32_t ii, jj;    // internal positions (node table rows)
  int32_t stype;     // 1 = common vertex, 2 = common edge
  int32_t ci0, cj0;  // first shared corner on each element (1-based)
  int32_t edge_i, edge_j;  // _corners_to_edge of the first two shared corners
  int32_t gi, gj;
  int32_t pad;
};

struct DuffyArgs {
  int64_t N;
  int nq;
  const double* p01;  // Gauss-Legendre points on [0,1]
  const double* w01;
  const DuffyPair* pairs;
  int64_t n_pairs;
  const double* coords;
  const int32_t* enodes;  // internal order, 0-based
  const double* area_orig;
  double* F;
  const NodeD* nodes;
  int n_nodes;
  const TriD* tris;
  unsigned long long* counters;
};

cudaError_t launch_duffy(const DuffyArgs& a, cudaStream_t st);

// Self view factors: F[i,i] for every element, one warp per element, with the
// FP64 pair arguments of the solve (kernels_self.cu).
cudaError_t launch_self(const PairArgs& a, cudaStream_t st);

struct McArgs {
  int64_t N, nT, n_tiles;
  int64_t tile0, tile_count;  // this launch integrates tiles [tile0, tile0 + tile_count)
  bool area_pass;             // also run the area rule (first launch of a solve)
  int n_samples;
  uint64_t seed;
  bool exclude;  // skip source / destination groups in the traversal
  bool dim3;
  const double* coords;
  const int32_t* enodes;  // internal order, 0-based
  const int8_t* fam;      // internal order
  const int32_t* group;   // internal order
  const int32_t* orig;    // internal -> caller's index
  const int32_t* inv;     // caller's index -> internal
  double* area_orig;      // written by the area-rule kernel
  double* F;
  const NodeD* nodes;
  int n_nodes;
  const TriD* tris;
  const SegD* segs;
  double cand_margin;  // curves: distance beyond which rounding cannot let a segment block a ray
  const uint8_t* tcls;    // surfaces with occlusion: tile classes and masks (kernels_cull.cu) for the
  const uint32_t* tmask;  //   elements' whole extent, or null (every sample ray walks the tree)
  unsigned long long* tile_counter;
  unsigned long long* counters;
  uint8_t* ray_log;  // [(i*N + j) * n_samples + k] for caller indices i < j
};

// Centres (of the nodes) and radii bounding every point of each surface
// element, for the tile classification of Monte Carlo solves.
struct McBoundsArgs {
  int64_t N;
  const double* coords;
  const int32_t* enodes;
  const int8_t* fam;
  double* cen;  // 3 x N
  double* rad;  // N
};
cudaError_t launch_mc_bounds(const McBoundsArgs& a, cudaStream_t st);
// Blocks of the Monte Carlo kernel resident at once (its persistent grid).
int mc_resident_blocks(const McArgs& a, int sm_count);
cudaError_t launch_mc(const McArgs& a, int sm_count, cudaStream_t st);
cudaError_t launch_prep(const PrepArgs& a, cudaStream_t st);
cudaError_t launch_prep_f32(const PrepF32Args& a, cudaStream_t st);
size_t pair_smem_bytes(int pmax, int n_nodes_smem, bool occ);
cudaError_t launch_pairs_fp64(const PairArgs& a, int sm_count, cudaStream_t st);
cudaError_t launch_reduce(const RedArgs& a, cudaStream_t st);

}  // namespace rvf
