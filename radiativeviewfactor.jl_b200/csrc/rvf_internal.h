// rvf_internal.h -- session / mesh state behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/rvf_b200.h"
#include "rvf_host.h"
#include "kernels.h"

struct rvf_session;

namespace rvf {

using Session = ::rvf_session;

int set_err(int code, const char* fmt, ...);
int cuda_err(cudaError_t e, const char* what);
// Status of the exception being handled (call inside a catch block): every
// entry point of the C interface turns exceptions into a status this way.
int exception_status() noexcept;
extern thread_local std::string g_last_error;

// Device allocation charged against the session's HBM budget.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  Session* owner = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { free_(); }
  int alloc(Session* s, size_t n);
  void free_();
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

int upload(Session* s, DevBuf& b, const void* src, size_t n);
constexpr size_t kSpareMin = (size_t)4096;  // every buffer: cudaFree costs ~1 ms and synchronises the device
// Frees cached buffers, the oldest first, until `need` more bytes fit the
// budget (need = 0: all of them).
void release_spares(Session* s, size_t need = 0);

struct Tables {
  int nquad = 0, pmax = 0;
  DevBuf rules, tab, area, np, flat, nrm, cen, diam, rad;  // internal element order
  DevBuf area_orig;                                   // areas in the caller's element order
  DevBuf tabf;  // FP32 table, built on the first mixed-precision solve
  DevBuf tcls, tmask;  // tile classes and masks of the last solve (kernels_cull.cu)
  DevBuf twork;        // the tiles the chunked pipeline integrates (tile indices, row-major)
};

// Autotuner choices of the request server (server.cpp), kept by the session
// so that every server on it reuses them.  Chunk grids per launch class:
// candidate (generation, traversal) blocks per SM, ms per million point
// pairs of the claimed tiles.
struct GridTune {
  size_t next = 0;
  std::vector<double> score;
  int gen = 0, trace = 0;
  bool done = false;
};
// The quadrature-only kernel's shape per launch class, rule size and size
// class: ms per 1e9 point pairs of each candidate.
struct FastTune {
  double score[4] = {0, 0, 0, 0};
  int qb = 0, groups = 1;
  bool done = false;
};

}  // namespace rvf

struct rvf_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // downloads of finished F columns while later chunks compute
  size_t budget = 0, used = 0;
  int fail_alloc_in = 0;  // test hook: the n-th cudaMalloc from now fails once (0 = never)
  int sm_count = 0;
  size_t smem_optin = 0;
  std::mutex mu;
  // autotuner state: a lock of its own, always taken last (admission holds
  // mu while it reads it, rvf_server_stats_get holds the server's lock)
  std::mutex tune_mu;
  std::map<uint64_t, rvf::GridTune> grid_tune;
  std::map<uint64_t, rvf::FastTune> ftune;
  std::vector<uint64_t> ftune_done;  // keys in the order their sweeps ended
  rvf::DevBuf err;           // int
  rvf::DevBuf tile_counter;  // u64
  rvf::DevBuf counters;      // u64 x 8
  // wavefront pair pipeline (kernels_wave.cu, wave_host.cpp): queues,
  // device launch blocks, pinned counter readback, graphs per launch shape
  rvf::DevBuf wq_ctr, wq_rec64, wq_rec32, wq_slots, wq_vis, wq_plist, wq_pool;
  rvf::DevBuf fast_ctr;  // tile counter of the kernel for tiles without ray work
  rvf::DevBuf wl_pair, wl_mixed, wl_trace, wl_resolve, wl_tilebase, wl_gen, wl_tb, wl_rb;
  unsigned long long* h_ctr = nullptr;
  std::map<uint64_t, cudaGraphExec_t> graphs;
  std::set<rvf_mesh*> meshes;
  cudaEvent_t ev[8] = {};
  // Freed device buffers (all of them, in size classes from 4 KiB), kept for reuse and still
  // charged to the budget: solving one new mesh after another (an F of
  // 15 GB each) then skips cudaMalloc / cudaFree, whose mapping work costs
  // a few hundred milliseconds per mesh.  Dropped when an allocation would
  // exceed the budget, and at session destroy.
  std::mutex spare_mu;
  std::vector<std::pair<void*, size_t>> spares;
};

struct rvf_mesh {
  rvf_session* s = nullptr;
  int dim = 2;
  int64_t N = 0, Nn = 0;
  // host copies
  std::vector<int32_t> h_enodes;  // N x 8, 0-based, caller's element order
  std::vector<int32_t> h_orig;    // internal (Morton) position -> caller's element index
  std::vector<int8_t> h_fam;
  std::vector<int32_t> h_group;
  std::vector<int32_t> h_tags;
  std::vector<int64_t> h_member_off;
  std::vector<int32_t> h_members;
  std::vector<double> h_soup;
  std::vector<int32_t> h_obs_group;
  std::vector<rvf::NodeD> h_nodes;
  int G = 0;
  // device
  rvf::DevBuf coords, enodes, fam, group, member_off, members;  // per-element arrays in internal order
  rvf::DevBuf orig;                                             // int32 internal -> caller's index
  rvf::DevBuf inv;                                              // int32 caller's index -> internal
  rvf::DevBuf mc_area;                                          // Monte Carlo areas (caller's order)
  rvf::DevBuf mc_cen, mc_rad, mc_tcls, mc_tmask;                // Monte Carlo tile classes (surfaces)
  bool mc_cls_ready = false;                                    //   valid for the current options
  rvf::DevBuf nodes, tris_ref, tris_geo, segs;
  rvf::DevBuf nodesf, trisf_ref, trisf_geo;  // FP32 copies (mixed precision)
  rvf::DevBuf leaf_of;                        // int32 leaf node of each primitive (leaf order)
  rvf::DevBuf sat_ref, sat_geo;               // pair-list data per triangle (3 float4, leaf order)
  rvf::DevBuf frontier;                       // int32 start nodes of the pair-list walk
  int n_frontier = 0;
  float sat_em = 0.f;
  double extent = 1.0;                        // 1 + max |coordinate| of the mesh and the soup
  int n_nodes = 0;
  int64_t n_obs = 0;
  std::map<int, std::unique_ptr<rvf::Tables>> tables;
  // Quad8 pairs sharing corners (built on the first use_duffy solve)
  bool duffy_built = false;
  int64_t n_duffy = 0;       // pairs (i, j), i < j, sharing corners
  int64_t n_duffy_self = 0;  // the Quad8 pairs (i, i) of self_vf solves, after them in duffy_pairs
  rvf::DevBuf duffy_pairs;
  std::map<int, std::unique_ptr<rvf::DevBuf>> duffy_rules;  // nquad -> [p01 | w01]
  // results of the last solve
  rvf::DevBuf F, part, rowgroup, rowsum, Fgroup, Agroup;
  const double* result_area = nullptr;  // areas (caller's order) of the last result
  bool has_result = false;
};

namespace rvf {
int mesh_upload(Session* s, const rvf_mesh_desc* d, rvf_mesh** out);
int ensure_tables(Session* s, rvf_mesh* m, int nquad, Tables** out);
// solve.cpp helpers shared with the serving loop (callers hold s->mu)
int read_err(Session* s);
int validate_options(const rvf_mesh* m, const rvf_options* o);
int no_progress(Session* s);
int reduce_alloc(Session* s, rvf_mesh* m);  // the reductions' buffers (before any kernel runs)
int mc_classify(Session* s, rvf_mesh* m, const rvf_options* o);  // Monte Carlo tile classes (surfaces)
int run_reduce(Session* s, rvf_mesh* m, const double* area);
// The self pairs (i, i) of a quadrature solve with the pipeline's FP64
// arguments, counted in the session's counters.
cudaError_t launch_self_pairs(Session* s, const PairArgs& pa, cudaStream_t st);
int ensure_duffy(Session* s, rvf_mesh* m, int nquad, const double** p01, const double** w01);
void fill_mc_args(Session* s, rvf_mesh* m, const rvf_options* o, uint8_t* ray_log, McArgs& c);
}  // namespace rvf
