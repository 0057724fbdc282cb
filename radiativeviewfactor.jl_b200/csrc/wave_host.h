// wave_host.h -- host side of the wavefront pair pipeline (wave_host.cpp).
#pragma once

#include <vector>

#include <functional>

#include "kernels.h"
#include "rvf_internal.h"

namespace rvf {

// One request's kernel arguments and progress through its tiles.
struct WaveReq {
  PairArgs pa{};
  MixedArgs ma{};
  TraceArgs ta{};
  ResolveArgs ra{};
  bool mixed = false, occ = false, dim3 = true;
  int pmax = 0;
  int64_t n_tiles = 0;  // tiles of the chunked pipeline (every upper-triangle tile, or the listed ones)
  std::vector<int64_t> row_end;  // with a tile list: listed tiles in tile rows 0..r (for the F download)
  int64_t claimed = 0;  // tiles integrated so far
  int claim_retries = 4096;  // compare-and-swap attempts of a tile claim (0: every claim gives up)
  int fast_qb = 0;           // quadrature-only kernel shape: points per lane block (0: by the rule)
  int fast_groups = 0;       //   and warp tasks per tile (0: fast_groups_auto)
  int64_t n_fast_tiles = 0;  // tiles of the quadrature-only kernel
  const NodeD* nodes_d = nullptr;
  const NodeF* nodes_f = nullptr;
  bool done() const { return claimed >= n_tiles; }
};

struct ChunkInfo {
  double ms_gen = 0, ms_trace = 0, ms_trace_fp64 = 0, ms_resolve = 0;  // CUDA events (eager launches only)
  double ms_lists = 0;                                                  // pair lists (inside ms_trace)
  int64_t rays_traced = 0;
  int kernels = 0;
  bool graph = false;  // replayed from a captured graph
};

int ensure_wave(Session* s, bool two_queues, bool occ, bool lists, int pmax, int64_t n_tiles, WaveQ& q);
// Fills w from a mesh, its tables and the options (builds the FP32 table on
// the first mixed-precision use).
int wave_prepare(Session* s, rvf_mesh* m, Tables* T, const rvf_options* o, uint8_t* ray_log, WaveReq& w,
                 int64_t* n_kernels);
WaveShape wave_shape(Session* s, WaveReq* const* reqs, int n);
// The request's tiles without shadow-ray work (by class), before its chunks;
// the chunks then skip them.  No-op without tile classes or with a ray log.
// Warp tasks per tile of the quadrature-only kernel when the caller names
// none: the fewest of 1, 2, 4, 8, 32 that give four tasks per resident warp.
int fast_groups_auto(int64_t n_tiles, int sm_count);
int wave_fast(Session* s, WaveReq& w, int64_t* n_kernels);
// One chunk over n requests of one shape (mixed, dim3, occ equal): claims
// tiles in request order while the queues have room, traces and resolves
// them, and advances each request's progress.  use_graph replays a CUDA
// graph captured per launch shape (eager launch when capture is refused).
// gen_bps / trace_bps: blocks per SM of the two grids (0 = occupancy limit);
// pp_budget > 0 caps the point pairs (worst case 32 x 32 x pmax^2 per tile)
// offered to the launch, given to the requests in order.
// on_launched (optional) runs on the host once the chunk's work is queued and
// before the host waits for it: host work that overlaps the chunk.
int wave_chunk(Session* s, WaveReq* const* reqs, int n, bool use_graph, ChunkInfo* info, int gen_bps = 0,
               int trace_bps = 0, double pp_budget = 0.0, const std::function<void()>* on_launched = nullptr);

}  // namespace rvf
