// solve.cpp -- extern "C" entry points of librvf_b200 (include/rvf_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/rvf_b200.h"
#include "kernels.h"
#include "wave_host.h"
#include "rvf_internal.h"

using namespace rvf;

namespace {

struct EvTimer {
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  explicit EvTimer(cudaStream_t s) : st(s) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
  double stop() {
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~EvTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace

namespace rvf {

int read_err(Session* s) {
  int herr = 0;
  cudaError_t e = cudaMemcpyAsync(&herr, s->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_err(e, "kernel execution");
  if (herr & kErrWaitTimeout) return set_err(RVF_ETIMEDOUT, "a bounded device wait gave up (shared-memory copy did not complete)");
  if (herr & kErrBadInput) return set_err(RVF_EINVAL, "kernel reported invalid input");
  return RVF_OK;
}

// A chunk that claimed no tile: its claims either gave up after their
// bounded retries (RVF_ETIMEDOUT) or found no queue room for one tile.
int no_progress(Session* s) {
  int herr = 0;
  if (cudaMemcpy(&herr, s->err.ptr, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && (herr & kErrClaimGaveUp))
    return set_err(RVF_ETIMEDOUT, "pair pipeline made no progress: every tile claim gave up after its bounded retries");
  return set_err(RVF_ENOMEM, "pair pipeline made no progress: ray queue too small for one tile");
}

int validate_options(const rvf_mesh* m, const rvf_options* o) {
  if (o->nquad < 1) return set_err(RVF_EINVAL, "nquad must be >= 1, got %d", o->nquad);
  if (o->method != RVF_METHOD_QUADRATURE && o->method != RVF_METHOD_MONTE_CARLO)
    return set_err(RVF_EINVAL, "unknown method %d", o->method);
  if (o->precision != RVF_PREC_FP64 && o->precision != RVF_PREC_MIXED)
    return set_err(RVF_EINVAL, "unknown precision %d", o->precision);
  if (o->method == RVF_METHOD_MONTE_CARLO && o->use_duffy)
    return set_err(RVF_EINVAL, "use_duffy and monte_carlo cannot both be true.");  // src/Assembly.jl:79-80
  if (o->method == RVF_METHOD_MONTE_CARLO && o->n_samples < 1)
    return set_err(RVF_EINVAL, "n_samples must be >= 1");
  if (o->ray_log && o->ray_log_pm < 1) return set_err(RVF_EINVAL, "ray_log needs ray_log_pm >= 1");
  if (o->fault_inject & ~(RVF_FAULT_CLAIM | RVF_FAULT_ALLOC))
    return set_err(RVF_EINVAL, "unknown fault_inject bits 0x%x", o->fault_inject);
  if (o->self_vf != 0 && o->self_vf != 1) return set_err(RVF_EINVAL, "self_vf must be 0 or 1, got %d", o->self_vf);
  if (o->fast_points &&
      !fast_qb_supported(o->precision == RVF_PREC_MIXED && m->dim == 2 && o->method == RVF_METHOD_QUADRATURE,
                         o->fast_points))
    return set_err(RVF_EINVAL, "fast_points %d is not a compiled block for this precision", o->fast_points);
  if (o->fast_row_groups != 0 && o->fast_row_groups != 1 && o->fast_row_groups != 2 && o->fast_row_groups != 4 &&
      o->fast_row_groups != 8 && o->fast_row_groups != 32)
    return set_err(RVF_EINVAL, "fast_row_groups must be 0, 1, 2, 4, 8 or 32, got %d", o->fast_row_groups);
  if (o->self_vf && o->method == RVF_METHOD_MONTE_CARLO)
    return set_err(RVF_EINVAL, "self_vf is supported with quadrature only");
  return RVF_OK;
}

// Monte Carlo launch arguments of a whole solve (src/GPUMCKernels.jl:295-328).
void fill_mc_args(Session* s, rvf_mesh* m, const rvf_options* o, uint8_t* ray_log, McArgs& c) {
  const int64_t N = m->N;
  const bool occ = o->occlusion && m->n_nodes > 0;
  c = McArgs{};
  c.N = N;
  c.nT = (N + kTile - 1) / kTile;
  c.n_tiles = c.nT * (c.nT + 1) / 2;
  c.tile0 = 0;
  c.tile_count = c.n_tiles;
  c.area_pass = true;
  c.n_samples = o->n_samples;
  c.seed = o->seed;
  c.exclude = o->mc_exclude_groups != 0 || m->dim == 1;
  c.dim3 = (m->dim == 2);
  c.coords = m->coords.as<double>();
  c.enodes = m->enodes.as<int32_t>();
  c.fam = m->fam.as<int8_t>();
  c.group = m->group.as<int32_t>();
  c.orig = m->orig.as<int32_t>();
  c.inv = m->inv.as<int32_t>();
  c.area_orig = m->mc_area.as<double>();
  c.F = m->F.as<double>();
  c.nodes = occ ? m->nodes.as<NodeD>() : nullptr;
  c.n_nodes = occ ? m->n_nodes : 0;
  c.tris = occ ? (o->geometric_soup ? m->tris_geo.as<TriD>() : m->tris_ref.as<TriD>()) : nullptr;
  c.segs = occ ? m->segs.as<SegD>() : nullptr;
  {
    // a computed hit of the reference's segment test (src/BVH.jl:265-322:
    // |den| >= 1e-8, parameters strictly inside (1e-8, 1 - 1e-8)) lies within
    // about 2e-7 S^3 of both segments (S bounds every length), so a segment
    // farther than this from a ray cannot block it
    const double S = 2.0 * m->extent;
    c.cand_margin = 1e-5 * S * S * S + std::ldexp(S, -16);
  }
  c.tcls = (occ && c.dim3 && m->mc_cls_ready) ? m->mc_tcls.as<uint8_t>() : nullptr;
  c.tmask = c.tcls ? m->mc_tmask.as<uint32_t>() : nullptr;
  c.tile_counter = s->tile_counter.as<unsigned long long>();
  c.counters = s->counters.as<unsigned long long>();
  c.ray_log = ray_log;
}

// Tile classes for a Monte Carlo solve of a surface mesh with occlusion:
// the quadrature pipeline's classification (kernels_cull.cu) with element
// centres and radii that bound every point of each element (a sample can lie
// anywhere on it), and, unless the solve skips the elements' own groups,
// every triangle a candidate.  A pair outside its row's mask has no sample
// ray that can be blocked.
int mc_classify(Session* s, rvf_mesh* m, const rvf_options* o) {
  m->mc_cls_ready = false;
  const int64_t N = m->N;
  const bool occ = o->occlusion && m->n_nodes > 0;
  if (o->disable_tile_cull || !occ || m->dim != 2 || N == 0 || !m->frontier.ptr) return RVF_OK;
  const int64_t nT = (N + kTile - 1) / kTile, nt = nT * (nT + 1) / 2;
  int rc = 0;
  if (m->mc_cen.bytes < sizeof(double) * 3 * N && (rc = m->mc_cen.alloc(s, sizeof(double) * 3 * N))) return rc;
  if (m->mc_rad.bytes < sizeof(double) * N && (rc = m->mc_rad.alloc(s, sizeof(double) * N))) return rc;
  if (m->mc_tcls.bytes < (size_t)nt && (rc = m->mc_tcls.alloc(s, (size_t)nt))) return rc;
  if (m->mc_tmask.bytes < sizeof(uint32_t) * kTile * nt && (rc = m->mc_tmask.alloc(s, sizeof(uint32_t) * kTile * nt)))
    return rc;
  if (!s->fast_ctr.ptr && (rc = s->fast_ctr.alloc(s, 256))) return rc;
  McBoundsArgs b{N, m->coords.as<double>(), m->enodes.as<int32_t>(), m->fam.as<int8_t>(), m->mc_cen.as<double>(),
                 m->mc_rad.as<double>()};
  cudaError_t e = launch_mc_bounds(b, s->stream);
  if (e != cudaSuccess) return cuda_err(e, "Monte Carlo bounds launch");
  TileClassArgs c{};
  c.N = N;
  c.nT = nT;
  c.n_tiles = nt;
  c.cen = m->mc_cen.as<double>();
  c.rad = m->mc_rad.as<double>();
  c.diam = c.rad;  // read only by the near-field pass, which is off
  c.group = m->group.as<int32_t>();
  c.near_factor = -1.0;
  c.tiny_gap = -1.0;
  c.cull_margin = std::ldexp(m->extent, -30);
  c.occ = true;
  c.dim3 = true;
  c.skip_groups = o->mc_exclude_groups != 0;  // otherwise the rays skip group 0 only: test every triangle
  c.nodesf = m->nodesf.as<NodeF>();
  c.n_nodes = m->n_nodes;
  c.frontier = m->frontier.as<int32_t>();
  c.n_frontier = m->n_frontier;
  c.leaf_of = m->leaf_of.as<int32_t>();
  c.sat = o->geometric_soup ? m->sat_geo.as<float4>() : m->sat_ref.as<float4>();
  c.sat_em = m->sat_em;
  c.cls = m->mc_tcls.as<uint8_t>();
  c.mask = m->mc_tmask.as<uint32_t>();
  c.claim = s->fast_ctr.as<unsigned long long>() + 1;
  c.counters = s->counters.as<unsigned long long>() + 13;
  if ((e = launch_tile_class(c, s->sm_count, s->stream)) != cudaSuccess)
    return cuda_err(e, "Monte Carlo tile classification launch");
  m->mc_cls_ready = true;
  return RVF_OK;
}

cudaError_t launch_self_pairs(Session* s, const PairArgs& pa, cudaStream_t st) {
  PairArgs a = pa;
  a.counters = s->counters.as<unsigned long long>();
  return launch_self(a, st);
}

// The reductions' buffers, allocated before the pair pipeline starts: an
// allocation while kernels and F copies are in flight can wait for them.
int reduce_alloc(Session* s, rvf_mesh* m) {
  const int64_t N = m->N;
  if (N == 0 || m->G == 0) return RVF_OK;
  const int n_chunks = (int)std::min<int64_t>(256, std::max<int64_t>(1, (1 << 20) / std::max<int64_t>(N, 1)));
  int rc;
  if (m->part.bytes < sizeof(double) * n_chunks * m->G * N)
    if ((rc = m->part.alloc(s, sizeof(double) * n_chunks * m->G * N))) return rc;
  if (m->rowgroup.bytes < sizeof(double) * m->G * N)
    if ((rc = m->rowgroup.alloc(s, sizeof(double) * m->G * N))) return rc;
  if (m->rowsum.bytes < sizeof(double) * N)
    if ((rc = m->rowsum.alloc(s, sizeof(double) * N))) return rc;
  if (m->Fgroup.bytes < sizeof(double) * m->G * m->G)
    if ((rc = m->Fgroup.alloc(s, sizeof(double) * m->G * m->G))) return rc;
  if (m->Agroup.bytes < sizeof(double) * m->G)
    if ((rc = m->Agroup.alloc(s, sizeof(double) * m->G))) return rc;
  return RVF_OK;
}

int run_reduce(Session* s, rvf_mesh* m, const double* area) {
  const int64_t N = m->N;
  if (N == 0 || m->G == 0) return RVF_OK;
  const int n_chunks = (int)std::min<int64_t>(256, std::max<int64_t>(1, (1 << 20) / std::max<int64_t>(N, 1)));
  int rc = reduce_alloc(s, m);
  if (rc) return rc;
  RedArgs r{};
  r.N = N;
  r.G = m->G;
  r.n_chunks = n_chunks;
  r.F = m->F.as<double>();
  r.area = area;  // reductions work in the caller's element order
  r.member_off = m->member_off.as<int64_t>();
  r.members = m->members.as<int32_t>();
  r.part = m->part.as<double>();
  r.rowgroup = m->rowgroup.as<double>();
  r.rowsum = m->rowsum.as<double>();
  r.Fgroup = m->Fgroup.as<double>();
  r.Agroup = m->Agroup.as<double>();
  cudaError_t e = launch_reduce(r, s->stream);
  return e == cudaSuccess ? RVF_OK : cuda_err(e, "reduction kernels");
}

// Quad8 pairs that share corner nodes, in the reference's classification
// (singularity_type, src/DuffyKernel.jl:95-115): corners 1-4 compared by node
// index, ci outer / cj inner, the first two matches kept.
int ensure_duffy(Session* s, rvf_mesh* m, int nquad, const double** p01, const double** w01) {
  if (!m->duffy_built) {
    const int64_t N = m->N;
    std::vector<int32_t> inv(N);
    for (int64_t e = 0; e < N; ++e) inv[m->h_orig[e]] = (int32_t)e;
    std::map<int32_t, std::vector<int32_t>> by_node;
    for (int64_t e = 0; e < N; ++e)
      if (m->h_fam[e] == 0)
        for (int c = 0; c < 4; ++c) by_node[m->h_enodes[(size_t)e * 8 + c]].push_back((int32_t)e);
    auto corners_to_edge = [](int c1, int c2) {  // src/DuffyKernel.jl:411-419
      int a = std::min(c1, c2), b = std::max(c1, c2);
      if (a == 1 && b == 2) return 1;
      if (a == 2 && b == 3) return 2;
      if (a == 3 && b == 4) return 3;
      if (a == 1 && b == 4) return 4;
      return 1;
    };
    std::vector<DuffyPair> pairs;
    // singularity_type (src/DuffyKernel.jl:95-115): corners equal by node
    // index, in the reference's loop order (corner of i outer, of j inner)
    auto classify = [&](int64_t i, int32_t j) {
      const int32_t* a = &m->h_enodes[(size_t)i * 8];
      const int32_t* b = &m->h_enodes[(size_t)j * 8];
      int n = 0, ci[2] = {0, 0}, cj[2] = {0, 0};
      for (int x = 0; x < 4; ++x)
        for (int y = 0; y < 4; ++y)
          if (a[x] == b[y]) {
            if (n < 2) { ci[n] = x + 1; cj[n] = y + 1; }
            ++n;
          }
      if (n == 0) return;
      DuffyPair P{};
      P.i = (int32_t)i; P.j = j; P.ii = inv[i]; P.jj = inv[j];
      P.stype = n == 1 ? 1 : 2;
      P.ci0 = ci[0]; P.cj0 = cj[0];
      P.edge_i = n >= 2 ? corners_to_edge(ci[0], ci[1]) : 1;
      P.edge_j = n >= 2 ? corners_to_edge(cj[0], cj[1]) : 1;
      P.gi = m->h_group[i]; P.gj = m->h_group[j];
      pairs.push_back(P);
    };
    for (int64_t i = 0; i < N; ++i) {
      if (m->h_fam[i] != 0) continue;
      std::vector<int32_t> cand;
      for (int c = 0; c < 4; ++c)
        for (int32_t j : by_node[m->h_enodes[(size_t)i * 8 + c]])
          if (j > i) cand.push_back(j);
      std::sort(cand.begin(), cand.end());
      cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
      for (int32_t j : cand) classify(i, j);
    }
    const size_t n_regular = pairs.size();
    // then the self pairs (i, i) of self_vf solves: an element shares every
    // corner with itself, so the reference treats it as a common-edge pair on
    // the first two matches, (1, 1) and (2, 2)
    for (int64_t i = 0; i < N; ++i)
      if (m->h_fam[i] == 0) classify(i, (int32_t)i);
    int rc;
    if (!pairs.empty() && (rc = upload(s, m->duffy_pairs, pairs.data(), sizeof(DuffyPair) * pairs.size()))) return rc;
    m->n_duffy = (int64_t)n_regular;
    m->n_duffy_self = (int64_t)(pairs.size() - n_regular);
    m->duffy_built = true;
  }
  auto it = m->duffy_rules.find(nquad);
  if (it == m->duffy_rules.end()) {
    std::vector<double> p, w;
    gl1d(nquad, p, w);
    std::vector<double> buf(2 * nquad);
    for (int k = 0; k < nquad; ++k) {  // src/DuffyKernel.jl:226-229
      buf[k] = (p[k] + 1.0) / 2.0;
      buf[nquad + k] = w[k] / 2.0;
    }
    auto b = std::make_unique<DevBuf>();
    int rc;
    if ((rc = upload(s, *b, buf.data(), sizeof(double) * buf.size()))) return rc;
    it = m->duffy_rules.emplace(nquad, std::move(b)).first;
  }
  *p01 = it->second->as<double>();
  *w01 = *p01 + nquad;
  return RVF_OK;
}

}  // namespace rvf

extern "C" {

const char* rvf_version(void) { return "rvf_b200 0.1.0 (sm_100a)"; }
int rvf_abi_version(void) { return RVF_ABI_VERSION; }

int rvf_last_error(char* buf, size_t n) {
  if (!buf || n == 0) return (int)g_last_error.size();
  size_t k = std::min(n - 1, g_last_error.size());
  std::memcpy(buf, g_last_error.data(), k);
  buf[k] = 0;
  return (int)g_last_error.size();
}

void rvf_default_options(rvf_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->nquad = 4;  // src/Assembly.jl:65
  o->method = RVF_METHOD_QUADRATURE;
  o->n_samples = 10000;  // src/Assembly.jl:70
  o->seed = 0;
  o->precision = RVF_PREC_FP64;
  o->occlusion = 1;
  o->near_field_factor = 2.0;
}

int rvf_session_create(const rvf_session_opts* opts, rvf_session** out) try {
  if (!out) return set_err(RVF_EINVAL, "null out");
  *out = nullptr;
  int dev = opts ? opts->device : 0;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_err(RVF_ENODEV, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= n) return set_err(RVF_ENODEV, "device %d out of range (%d devices)", dev, n);
  cudaDeviceProp p;
  if ((e = cudaGetDeviceProperties(&p, dev)) != cudaSuccess) return cuda_err(e, "cudaGetDeviceProperties");
  if (p.major < 10) return set_err(RVF_ENODEV, "device %d is sm_%d%d; this library is built for sm_100a", dev, p.major, p.minor);
  if ((e = cudaSetDevice(dev)) != cudaSuccess) return cuda_err(e, "cudaSetDevice");
  auto s = std::make_unique<rvf_session>();
  s->device = dev;
  s->sm_count = p.multiProcessorCount;
  s->smem_optin = p.sharedMemPerBlockOptin;
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_err(e, "cudaStreamCreate");
  if ((e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_err(e, "cudaStreamCreate");
  for (cudaEvent_t& v : s->ev)
    if ((e = cudaEventCreate(&v)) != cudaSuccess) return cuda_err(e, "cudaEventCreate");
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  s->budget = (opts && opts->hbm_budget_bytes) ? opts->hbm_budget_bytes : (size_t)(0.9 * (double)fr);
  int rc;
  if ((rc = s->err.alloc(s.get(), 256))) return rc;
  if ((rc = s->tile_counter.alloc(s.get(), 256))) return rc;
  if ((rc = s->counters.alloc(s.get(), 256))) return rc;
  *out = s.release();
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_session_destroy(rvf_session* s) try {
  if (!s) return RVF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    for (rvf_mesh* m : s->meshes) delete m;
    s->meshes.clear();
    s->err.free_();
    s->tile_counter.free_();
    s->counters.free_();
    s->fast_ctr.free_();
    s->wq_ctr.free_(); s->wq_rec64.free_(); s->wq_rec32.free_(); s->wq_slots.free_(); s->wq_vis.free_(); s->wq_plist.free_(); s->wq_pool.free_();
    for (rvf::DevBuf* b : {&s->wl_pair, &s->wl_mixed, &s->wl_trace, &s->wl_resolve, &s->wl_tilebase, &s->wl_gen,
                           &s->wl_tb, &s->wl_rb})
      b->free_();
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    rvf::release_spares(s);
    if (s->h_ctr) cudaFreeHost(s->h_ctr);
    s->h_ctr = nullptr;
    for (cudaEvent_t v : s->ev)
      if (v) cudaEventDestroy(v);
    cudaStreamDestroy(s->stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  }
  delete s;
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_device_info(rvf_session* s, int* sm_count, uint64_t* hbm_total, uint64_t* hbm_free) {
  if (!s) return set_err(RVF_EINVAL, "null session");
  cudaSetDevice(s->device);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  if (sm_count) *sm_count = s->sm_count;
  if (hbm_total) *hbm_total = tot;
  if (hbm_free) *hbm_free = fr;
  return RVF_OK;
}

int rvf_mesh_upload(rvf_session* s, const rvf_mesh_desc* d, rvf_mesh** out) try {
  if (!s) return set_err(RVF_EINVAL, "null session");
  std::lock_guard<std::mutex> lk(s->mu);
  cudaSetDevice(s->device);
  int rc = mesh_upload(s, d, out);
  if (rc == RVF_OK) s->meshes.insert(*out);
  return rc;
} catch (...) {
  return exception_status();
}

int rvf_mesh_release(rvf_session* s, rvf_mesh* m) try {
  if (!s || !m) return set_err(RVF_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->meshes.count(m)) return set_err(RVF_EINVAL, "mesh does not belong to this session");
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  s->meshes.erase(m);
  delete m;
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_mesh_n_elems(const rvf_mesh* m, int64_t* n) {
  if (!m || !n) return set_err(RVF_EINVAL, "null argument");
  *n = m->N;
  return RVF_OK;
}

namespace {

// Download of F overlapped with the pair pipeline.  Tiles are claimed in
// row-major order over (bi <= bj); internal column j of F is final once tile
// row floor(j / 32) is done -- later tiles (bi', bj') with bi' > bi write only
// columns of internal elements in blocks >= bi' -- so after each chunk the
// caller's columns orig[j] of the newly finished rows go to the host on the
// copy stream while the next chunk computes (contiguous caller columns in
// one copy).  A pageable destination makes the copies synchronous: still
// correct, without the overlap.
#ifndef RVF_DL_CHUNKS
#define RVF_DL_CHUNKS 16
#endif
#ifndef RVF_DL_MIN_PP
#define RVF_DL_MIN_PP 2.5e8  // point pairs of a download chunk at least
#endif
constexpr int kDownloadChunks = RVF_DL_CHUNKS;

struct ColumnDownload {
  Session* s = nullptr;
  const rvf_mesh* m = nullptr;
  double* host = nullptr;
  int64_t N = 0, nT = 0, rows_done = 0;
  bool issued = false;
  std::vector<int32_t> cols;
  std::vector<int64_t> listed;  // the pipeline's tile list: listed tiles through each row (a copy: the
                                // pipeline's request ends before the last download)

  // one past the last tile of row bi (in the pipeline's claim order)
  int64_t row_end(int64_t bi) const {
    if (!listed.empty()) return listed[(size_t)bi];
    return (bi + 1) * nT - bi * (bi + 1) / 2;
  }

  cudaError_t advance(int64_t claimed_tiles) {
    cols.clear();
    while (rows_done < nT && row_end(rows_done) <= claimed_tiles) {
      const int64_t j1 = std::min<int64_t>(N, (rows_done + 1) * kTile);
      for (int64_t j = rows_done * kTile; j < j1; ++j) cols.push_back(m->h_orig[j]);
      ++rows_done;
    }
    std::sort(cols.begin(), cols.end());
    const double* dev = m->F.as<double>();
    for (size_t a = 0; a < cols.size();) {
      size_t b = a + 1;
      while (b < cols.size() && cols[b] == cols[b - 1] + 1) ++b;
      const int64_t c0 = cols[a], nc = (int64_t)(b - a);
      const cudaError_t e = cudaMemcpyAsync(host + c0 * N, dev + c0 * N, sizeof(double) * N * nc,
                                            cudaMemcpyDeviceToHost, s->copy_stream);
      if (e != cudaSuccess) return e;
      issued = true;
      a = b;
    }
    return cudaSuccess;
  }
  // copies still in flight must end before the caller's buffer can be reused
  ~ColumnDownload() {
    if (issued) cudaStreamSynchronize(s->copy_stream);
  }
};

}  // namespace

int rvf_solve(rvf_session* s, rvf_mesh* m, const rvf_options* o, double* F_elem, double* A_elem, double* F_group,
              double* A_group, double* row_sums, rvf_stats* st) try {
  if (!s || !m || !o) return set_err(RVF_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->meshes.count(m)) return set_err(RVF_EINVAL, "mesh does not belong to this session");
  cudaSetDevice(s->device);
  int rc = validate_options(m, o);
  if (rc) return rc;
  // test hook: the first device allocation of this call fails; disarmed on return
  struct FaultGuard {
    Session* s;
    ~FaultGuard() { s->fail_alloc_in = 0; }
  } fault_guard{s};
  s->fail_alloc_in = (o->fault_inject & RVF_FAULT_ALLOC) ? 1 : 0;
  const bool mc = (o->method == RVF_METHOD_MONTE_CARLO);
  // mixed precision covers quadrature on surface meshes; curve meshes and
  // Monte Carlo (which reproduces the reference's streams) run in FP64
  const bool mixed = (o->precision == RVF_PREC_MIXED) && (m->dim == 2) && !mc;
  if (mixed && !(o->near_field_factor >= 0.0)) return set_err(RVF_EINVAL, "near_field_factor must be >= 0");
  rvf_stats S{};
  int64_t n_kernels = 0;  // kernels of this library launched by this call
  EvTimer total(s->stream);
  const int64_t N = m->N;
  Tables* T = nullptr;
  const double* area_res = nullptr;  // element areas of this result, caller's order
  if (!mc) {
    EvTimer t(s->stream);
    const bool fresh = m->tables.find(o->nquad) == m->tables.end();
    if ((rc = ensure_tables(s, m, o->nquad, &T))) return rc;
    if ((rc = reduce_alloc(s, m))) return rc;
    if (fresh && N > 0) n_kernels += 1;
    S.ms_prep = t.stop();
    area_res = T->area_orig.as<double>();
  } else {
    if (m->mc_area.bytes < sizeof(double) * std::max<int64_t>(N, 1))
      if ((rc = m->mc_area.alloc(s, sizeof(double) * std::max<int64_t>(N, 1)))) return rc;
    if ((rc = reduce_alloc(s, m))) return rc;
    area_res = m->mc_area.as<double>();
  }
  if (m->F.bytes < sizeof(double) * N * N)
    if ((rc = m->F.alloc(s, sizeof(double) * std::max<int64_t>(N * N, 1)))) return rc;
  m->has_result = false;
  cudaMemsetAsync(s->tile_counter.ptr, 0, 8, s->stream);
  cudaMemsetAsync(s->counters.ptr, 0, 256, s->stream);
  cudaMemsetAsync(s->err.ptr, 0, sizeof(int), s->stream);
  DevBuf log;
  ColumnDownload dl;    // quadrature with a host F: columns go down as their tile rows finish
  int64_t w_tiles = 0;  // tiles done by the pair pipeline
  size_t log_bytes = 0;  // the caller's log size (a reused device buffer may be larger)
  if (o->ray_log) {
    if (!mc && o->ray_log_pm < T->pmax)
      return set_err(RVF_EINVAL, "ray_log_pm %d < points per element %d", o->ray_log_pm, T->pmax);
    // quadrature: [(i*N + j) * pm + p] * pm + q; Monte Carlo: (i*N + j) * n_samples + k
    size_t lb = (size_t)N * N * (mc ? (size_t)o->n_samples : (size_t)o->ray_log_pm * o->ray_log_pm);
    if ((rc = log.alloc(s, lb))) return rc;
    cudaMemsetAsync(log.ptr, 0, lb, s->stream);
    log_bytes = lb;
  }
  if (mc) {  // src/GPUMCKernels.jl:295-328
    {
      EvTimer tc(s->stream);
      if ((rc = mc_classify(s, m, o))) return rc;
      S.ms_cull = tc.stop();
    }
    McArgs c{};
    fill_mc_args(s, m, o, o->ray_log ? log.as<uint8_t>() : nullptr, c);
    if (N > 0) {
      EvTimer t(s->stream);
      cudaError_t e = launch_mc(c, s->sm_count, s->stream);
      if (e != cudaSuccess) return cuda_err(e, "Monte Carlo kernel launch");
      n_kernels += 2;
      S.ms_pairs = t.stop();
      if ((rc = read_err(s))) return rc;
    }
  } else {
  if (N > 0) {
    if (N == 1) {
      cudaMemsetAsync(m->F.ptr, 0, sizeof(double), s->stream);
    }
    cudaError_t e = cudaSuccess;
    WaveReq w;
    {
      EvTimer tc(s->stream);
      if ((rc = wave_prepare(s, m, T, o, o->ray_log ? log.as<uint8_t>() : nullptr, w, &n_kernels))) return rc;
      S.ms_cull = tc.stop();
    }
    {
      EvTimer tf(s->stream);
      if ((rc = wave_fast(s, w, &n_kernels))) return rc;
      S.ms_gen += tf.stop();
    }
    // Duffy and self pairs overwrite F after the pipeline: no early columns then
    if (F_elem && N > 1 && !(o->use_duffy && m->dim == 2) && !o->self_vf) {
      dl.s = s;
      dl.m = m;
      dl.host = F_elem;
      dl.N = N;
      dl.nT = (N + kTile - 1) / kTile;
      dl.listed = w.row_end;
      // rows without listed tiles are final once the quadrature-only kernel
      // ends: their columns may go out before any chunk, on the copy stream
      if ((e = cudaEventRecord(s->ev[7], s->stream)) != cudaSuccess ||
          (e = cudaStreamWaitEvent(s->copy_stream, s->ev[7], 0)) != cudaSuccess)
        return cuda_err(e, "download ordering");
    }
    EvTimer t(s->stream);
    WaveReq* one = &w;
    // the columns finished by earlier chunks are queued for download while
    // the next chunk runs
    cudaError_t dl_err = cudaSuccess;
    int64_t dl_upto = 0;
    const std::function<void()> queue_columns = [&]() {
      if (dl.host && dl_err == cudaSuccess) dl_err = dl.advance(dl_upto);
    };
    // With a host F the pipeline runs in up to kDownloadChunks chunks (none
    // below RVF_DL_MIN_PP point pairs), so that the columns of finished tile
    // rows go down while later chunks compute (the last chunk's rows hold
    // about 1/sqrt(chunks) of the columns); without, one chunk as far as the
    // ray queues allow.
    double pp_budget = 0.0;
    if (dl.host && w.n_tiles > 0)
      pp_budget = std::max((double)RVF_DL_MIN_PP, (double)w.n_tiles * kTile * kTile * w.pmax * w.pmax / kDownloadChunks);
    while (!w.done()) {  // chunks: each claims tiles while the ray queues have room
      ChunkInfo ci;
      const int64_t before = w.claimed;
      dl_upto = before;
      if ((rc = wave_chunk(s, &one, 1, false, &ci, 0, 0, pp_budget, &queue_columns))) return rc;
      if (dl_err != cudaSuccess) return cuda_err(dl_err, "F column download");
      if ((rc = read_err(s))) return rc;
      n_kernels += ci.kernels;
      S.n_chunks += 1;
      S.ms_gen += ci.ms_gen;
      S.ms_trace += ci.ms_trace;
      S.ms_trace_fp64 += ci.ms_trace_fp64;
      S.ms_resolve += ci.ms_resolve;
      S.ms_lists += ci.ms_lists;
      S.n_rays_traced += ci.rays_traced;
      if (w.claimed == before) return no_progress(s);
    }
    w_tiles = w.claimed;
    if (o->self_vf) {  // the pairs (i, i), before Duffy (which replaces the Quad8 ones)
      if ((e = launch_self_pairs(s, w.pa, s->stream)) != cudaSuccess) return cuda_err(e, "self-pair kernel launch");
      n_kernels += 1;
    }
    S.ms_pairs = t.stop();
    if ((rc = read_err(s))) return rc;
    // Duffy integrals overwrite the singular Quad8 pairs (Duffy for
    // Quad8-Quad8 surface pairs only, src/DuffyKernel.jl:461-463)
    if (o->use_duffy && m->dim == 2) {
      EvTimer td(s->stream);
      DuffyArgs d{};
      if ((rc = ensure_duffy(s, m, o->nquad, &d.p01, &d.w01))) return rc;
      d.N = N;
      d.nq = o->nquad;
      d.pairs = m->duffy_pairs.as<DuffyPair>();
      d.n_pairs = m->n_duffy + (o->self_vf ? m->n_duffy_self : 0);
      d.coords = m->coords.as<double>();
      d.enodes = m->enodes.as<int32_t>();
      d.area_orig = T->area_orig.as<double>();
      d.F = m->F.as<double>();
      d.nodes = w.pa.nodes;
      d.n_nodes = w.pa.n_nodes;
      d.tris = w.pa.tris;
      d.counters = s->counters.as<unsigned long long>();
      if (d.n_pairs > 0) {
        if ((e = launch_duffy(d, s->stream)) != cudaSuccess) return cuda_err(e, "Duffy kernel launch");
        n_kernels += 1;
      }
      S.ms_duffy = td.stop();
      S.n_duffy_pairs = m->n_duffy;
      if ((rc = read_err(s))) return rc;
    }
    if (N == 1) {  // raw 1x1 zero, area 0 -> F = 0/0 (the reference's result for one element)
      double nanv = std::nan("");
      cudaMemcpyAsync(m->F.ptr, &nanv, sizeof(double), cudaMemcpyHostToDevice, s->stream);
    }
  }
  }  // quadrature
  {
    EvTimer t(s->stream);
    if ((rc = run_reduce(s, m, area_res))) return rc;
    if (N > 0 && m->G > 0) n_kernels += 3;
    S.ms_reduce = t.stop();
  }
  m->has_result = true;
  m->result_area = area_res;
  {
    EvTimer t(s->stream);
    cudaError_t e = cudaSuccess;
    if (F_elem && N > 0 && !dl.host)
      e = cudaMemcpyAsync(F_elem, m->F.ptr, sizeof(double) * N * N, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && dl.host) {
      e = dl.advance(w_tiles);  // every row: nothing left unless a chunk was cut short
      if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy_stream);
    }
    if (e == cudaSuccess && A_elem && N > 0) e = cudaMemcpyAsync(A_elem, area_res, sizeof(double) * N, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && F_group && m->G > 0 && N > 0)
      e = cudaMemcpyAsync(F_group, m->Fgroup.ptr, sizeof(double) * m->G * m->G, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && A_group && m->G > 0 && N > 0)
      e = cudaMemcpyAsync(A_group, m->Agroup.ptr, sizeof(double) * m->G, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && row_sums && N > 0)
      e = cudaMemcpyAsync(row_sums, m->rowsum.ptr, sizeof(double) * N, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && o->ray_log)
      e = cudaMemcpyAsync(o->ray_log, log.ptr, log_bytes, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_err(e, "device->host copy");
    S.ms_download = t.stop();
  }
  if (st) {
    unsigned long long c[16] = {};
    cudaMemcpy(c, s->counters.ptr, sizeof c, cudaMemcpyDeviceToHost);
    S.n_pairs = N * (N - 1) / 2;
    S.n_point_pairs = (int64_t)c[0];
    S.n_rays = (int64_t)c[1];
    S.n_rays_fp64 = mixed ? (int64_t)c[4] : (int64_t)c[1];
    S.n_pairs_fp64 = mixed ? (int64_t)c[5] : S.n_pairs;
    S.n_node_visits = (int64_t)c[2];
    S.n_prim_tests = (int64_t)c[3];
    S.n_kernels = n_kernels;
    S.n_graze_fp64 = mixed ? (int64_t)c[6] : 0;
    S.n_unsure_rays = mixed ? (int64_t)c[7] : 0;
    S.n_unsure_slab = mixed ? (int64_t)c[8] : 0;
    S.n_unsure_prim = mixed ? (int64_t)c[9] : 0;
    S.n_unsure_dir = mixed ? (int64_t)c[10] : 0;
    S.n_list_pairs = (int64_t)c[11];
    S.n_walk_pairs = (int64_t)c[12];
    S.n_tiles_culled = (int64_t)c[13];
    S.n_pairs_masked = (int64_t)c[14];
    S.n_tiles_unclassified = (int64_t)c[15];
    if (N > 0 && m->G > 0) {
      std::vector<double> rs(N);
      cudaMemcpy(rs.data(), m->rowsum.ptr, sizeof(double) * N, cudaMemcpyDeviceToHost);
      double mx = 0.0;
      for (double v : rs) mx = std::max(mx, std::fabs(v - 1.0));
      S.max_row_sum_dev = mx;
    }
    S.ms_total = total.stop();
    *st = S;
  }
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_result_copy(rvf_session* s, rvf_mesh* m, double* F_elem, double* A_elem) try {
  if (!s || !m) return set_err(RVF_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (!m->has_result) return set_err(RVF_EINVAL, "no result on this mesh yet");
  cudaSetDevice(s->device);
  cudaError_t e = cudaSuccess;
  if (F_elem) e = cudaMemcpyAsync(F_elem, m->F.ptr, sizeof(double) * m->N * m->N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && A_elem) e = cudaMemcpyAsync(A_elem, m->result_area, sizeof(double) * m->N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e == cudaSuccess ? RVF_OK : cuda_err(e, "rvf_result_copy");
} catch (...) {
  return exception_status();
}

int rvf_result_device(rvf_mesh* m, const double** F_dev, const double** A_dev) {
  if (!m) return set_err(RVF_EINVAL, "null mesh");
  if (!m->has_result) return set_err(RVF_EINVAL, "no result on this mesh yet");
  if (F_dev) *F_dev = m->F.as<double>();
  if (A_dev) *A_dev = m->result_area;
  return RVF_OK;
}

int rvf_host_alloc(size_t bytes, void** p) {
  if (!p) return set_err(RVF_EINVAL, "null out");
  cudaError_t e = cudaHostAlloc(p, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_err(RVF_ENOMEM, "cudaHostAlloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return RVF_OK;
}

int rvf_host_free(void* p) {
  if (p) cudaFreeHost(p);
  return RVF_OK;
}

int rvf_quadrature_rule(int32_t family, int32_t nquad, double* pts, double* wts, int32_t* n_pts) try {
  if (family < 0 || family > 5 || nquad < 1) return set_err(RVF_EINVAL, "bad family/nquad");
  Rule r = (family == 0 || family == 2) ? gl2d(nquad) : (family == 1 || family == 3) ? tri_rule(nquad) : line_rule(nquad);
  if (n_pts) *n_pts = r.size();
  for (int k = 0; k < r.size(); ++k) {
    if (pts) { pts[2 * k] = r.xi[k]; pts[2 * k + 1] = r.eta[k]; }
    if (wts) wts[k] = r.w[k];
  }
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_bvh_build_host(const double* soup, int32_t nv, int64_t n_prims, double* lo, double* hi, int32_t* meta,
                       int32_t* tri_idx, int64_t* n_nodes) try {
  if (!soup || n_prims <= 0 || (nv != 2 && nv != 3)) return set_err(RVF_EINVAL, "bad soup");
  HostBVH b = build_bvh(soup, nv, n_prims);
  if (n_nodes) *n_nodes = (int64_t)b.nodes.size();
  if (!lo) return RVF_OK;
  for (size_t k = 0; k < b.nodes.size(); ++k) {
    const HostBVH::Node& n = b.nodes[k];
    for (int c = 0; c < 3; ++c) {
      lo[3 * k + c] = n.lo[c];
      if (hi) hi[3 * k + c] = n.hi[c];
    }
    if (meta) {
      meta[5 * k + 0] = (int32_t)n.left;
      meta[5 * k + 1] = (int32_t)n.right;
      meta[5 * k + 2] = (int32_t)n.tri_start;
      meta[5 * k + 3] = (int32_t)n.tri_count;
      meta[5 * k + 4] = (int32_t)n.miss;
    }
  }
  if (tri_idx)
    for (int64_t t = 0; t < n_prims; ++t) tri_idx[t] = (int32_t)b.tri_idx[t];
  return RVF_OK;
} catch (...) {
  return exception_status();
}

}  // extern "C"
