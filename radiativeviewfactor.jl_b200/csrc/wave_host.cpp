// wave_host.cpp -- host side of the wavefront pair pipeline (kernels_wave.cu):
// per-request kernel arguments, queue sizing, and chunked launches over one
// or more requests of one launch shape, optionally replayed from a CUDA graph
// captured per shape.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.h"
#include "wave_host.h"

namespace rvf {

// Ray queues of the pipeline, kept by the session and grown on demand.
// Capacity: every point pair of every tile when that is small, otherwise up
// to 2^29 records per queue (4 GiB) within the HBM budget, and never below a
// few tiles' worst case.
int ensure_wave(Session* s, bool two_queues, bool occ, bool lists, int pmax, int64_t n_tiles, WaveQ& q) {
  int rc = 0;
  if (!s->wq_ctr.ptr && (rc = s->wq_ctr.alloc(s, sizeof(unsigned long long) * kCtrCount))) return rc;
  q = WaveQ{};
  q.ctr = s->wq_ctr.as<unsigned long long>();
  q.vis_words = (pmax * pmax + 63) / 64;
  if (!occ) return 0;
  const int64_t per_tile = (int64_t)kTile * kTile * pmax * pmax;
  const int64_t want = std::min<int64_t>(n_tiles * per_tile, (int64_t)1 << 29);
  const int64_t floor_recs = std::min<int64_t>(n_tiles * per_tile, 4 * per_tile);
  const int64_t want_s = std::min<int64_t>(n_tiles * kTile * kTile, (int64_t)1 << 25);
  const int64_t floor_s = std::min<int64_t>(n_tiles * kTile * kTile, 4 * kTile * kTile);
  const int nq = two_queues ? 2 : 1;
  // pair lists: 8 B per slot and a pool of kPoolPerSlot entries per slot
  constexpr int64_t kPoolPerSlot = 24;
  const size_t slot_bytes = sizeof(PendSlot) + sizeof(unsigned long long) * q.vis_words +
                            (lists ? sizeof(PairList) + sizeof(int32_t) * kPoolPerSlot : 0);
  auto have = [&](int64_t recs, int64_t slots) {
    return s->wq_rec64.bytes >= sizeof(uint64_t) * recs &&
           (!two_queues || s->wq_rec32.bytes >= sizeof(uint64_t) * recs) &&
           s->wq_slots.bytes >= sizeof(PendSlot) * slots &&
           s->wq_vis.bytes >= sizeof(unsigned long long) * q.vis_words * slots &&
           (!lists || (s->wq_plist.bytes >= sizeof(PairList) * slots &&
                       s->wq_pool.bytes >= sizeof(int32_t) * kPoolPerSlot * slots));
  };
  int64_t recs = want, slots = want_s;
  if (!have(recs, slots)) {
    // release and size against the budget left
    s->wq_rec64.free_();
    s->wq_rec32.free_();
    s->wq_slots.free_();
    s->wq_vis.free_();
    s->wq_plist.free_();
    s->wq_pool.free_();
    const size_t left = s->budget > s->used ? s->budget - s->used : 0;
    while ((size_t)(recs * 8 * nq) + (size_t)slots * slot_bytes > left / 2 && (recs > floor_recs || slots > floor_s)) {
      recs = std::max<int64_t>(floor_recs, recs / 2);
      slots = std::max<int64_t>(floor_s, slots / 2);
    }
    if ((rc = s->wq_rec64.alloc(s, sizeof(uint64_t) * recs))) return rc;
    if (two_queues && (rc = s->wq_rec32.alloc(s, sizeof(uint64_t) * recs))) return rc;
    if ((rc = s->wq_slots.alloc(s, sizeof(PendSlot) * slots))) return rc;
    if ((rc = s->wq_vis.alloc(s, sizeof(unsigned long long) * q.vis_words * slots))) return rc;
    if (lists && (rc = s->wq_plist.alloc(s, sizeof(PairList) * slots))) return rc;
    if (lists && (rc = s->wq_pool.alloc(s, sizeof(int32_t) * kPoolPerSlot * slots))) return rc;
  }
  q.rec64 = s->wq_rec64.as<uint64_t>();
  q.rec32 = two_queues ? s->wq_rec32.as<uint64_t>() : nullptr;
  q.cap = (int64_t)(s->wq_rec64.bytes / sizeof(uint64_t));
  if (two_queues) q.cap = std::min<int64_t>(q.cap, (int64_t)(s->wq_rec32.bytes / sizeof(uint64_t)));
  q.slots = s->wq_slots.as<PendSlot>();
  q.vis = s->wq_vis.as<unsigned long long>();
  q.scap = std::min<int64_t>((int64_t)(s->wq_slots.bytes / sizeof(PendSlot)),
                             (int64_t)(s->wq_vis.bytes / (sizeof(unsigned long long) * q.vis_words)));
  q.plist = lists ? s->wq_plist.as<PairList>() : nullptr;
  q.pool = lists ? s->wq_pool.as<int32_t>() : nullptr;
  q.pool_cap = lists ? (int64_t)(s->wq_pool.bytes / sizeof(int32_t)) : 0;
  if (lists) q.scap = std::min<int64_t>(q.scap, (int64_t)(s->wq_plist.bytes / sizeof(PairList)));
  return 0;
}

int wave_prepare(Session* s, rvf_mesh* m, Tables* T, const rvf_options* o, uint8_t* ray_log, WaveReq& w,
                 int64_t* n_kernels) {
  const int64_t N = m->N;
  const bool occ = o->occlusion && m->n_nodes > 0;
  w = WaveReq{};
  w.mixed = (o->precision == RVF_PREC_MIXED) && (m->dim == 2);
  w.occ = occ;
  w.dim3 = (m->dim == 2);
  w.pmax = T->pmax;
  if (o->fault_inject & RVF_FAULT_CLAIM) w.claim_retries = 0;
  w.fast_qb = o->fast_points;
  w.fast_groups = o->fast_row_groups;  // 0: by the tile count (wave_fast)
  PairArgs& a = w.pa;
  a.N = N;
  a.nT = (N + kTile - 1) / kTile;
  a.n_tiles = a.nT * (a.nT + 1) / 2;
  a.pmax = T->pmax;
  a.dim3 = w.dim3;
  a.tab = T->tab.as<double>();
  a.np = T->np.as<int8_t>();
  a.area = T->area.as<double>();
  a.flat = T->flat.as<uint8_t>();
  a.nrm = T->nrm.as<double>();
  a.group = m->group.as<int32_t>();
  a.orig = m->orig.as<int32_t>();
  a.cen = T->cen.as<double>();
  a.rad = T->rad.as<double>();
  a.cull_margin = std::ldexp(m->extent, -30);
  a.F = m->F.as<double>();
  a.nodes = occ ? m->nodes.as<NodeD>() : nullptr;
  a.n_nodes = occ ? m->n_nodes : 0;
  a.tris = occ ? (o->geometric_soup ? m->tris_geo.as<TriD>() : m->tris_ref.as<TriD>()) : nullptr;
  a.segs = occ ? m->segs.as<SegD>() : nullptr;
  a.ray_log = ray_log;
  a.log_pm = o->ray_log_pm;
  w.n_tiles = a.n_tiles;
  if (w.mixed) {
    if (!T->tabf.ptr) {
      int rc = 0;
      if ((rc = T->tabf.alloc(s, sizeof(float) * a.nT * kComp * T->pmax * kTile))) return rc;
      cudaMemsetAsync(T->tabf.ptr, 0, T->tabf.bytes, s->stream);
      PrepF32Args pf{N, T->pmax, T->tab.as<double>(), T->tabf.as<float>(), T->np.as<int8_t>(), T->cen.as<double>()};
      const cudaError_t e = launch_prep_f32(pf, s->stream);
      if (e != cudaSuccess) return cuda_err(e, "FP32 table kernel launch");
      if (n_kernels) *n_kernels += 1;
    }
    MixedArgs& x = w.ma;
    x.N = N; x.nT = a.nT; x.n_tiles = a.n_tiles; x.pmax = a.pmax;
    x.tab = a.tab; x.tabf = T->tabf.as<float>(); x.np = a.np; x.area = a.area; x.flat = a.flat; x.nrm = a.nrm;
    x.cen = T->cen.as<double>(); x.diam = T->diam.as<double>(); x.near_factor = o->near_field_factor;
    x.rad = a.rad; x.cull_margin = a.cull_margin; x.tiny_gap = std::ldexp(m->extent, -16);
    x.group = a.group; x.orig = a.orig; x.F = a.F;
    x.nodes = a.nodes; x.n_nodes = a.n_nodes;
    x.nodesf = occ ? m->nodesf.as<NodeF>() : nullptr;
    x.tris = a.tris;
    x.trisf = occ ? (o->geometric_soup ? m->trisf_geo.as<TriF>() : m->trisf_ref.as<TriF>()) : nullptr;
    x.delta = (float)std::ldexp(m->extent, -20);
    x.ray_log = a.ray_log; x.log_pm = a.log_pm;
  }
  // Tile classes: which pairs' shadow rays may be blocked, which tiles are
  // near field (kernels_cull.cu); recomputed by every solve.
  if (!o->disable_tile_cull && N > 0) {
    int rc = 0;
    const size_t nt = (size_t)a.n_tiles;
    if (T->tcls.bytes < nt && (rc = T->tcls.alloc(s, nt))) return rc;
    if (T->tmask.bytes < nt * kTile * sizeof(uint32_t) && (rc = T->tmask.alloc(s, nt * kTile * sizeof(uint32_t))))
      return rc;
    TileClassArgs c{};
    c.N = N;
    c.nT = a.nT;
    c.n_tiles = a.n_tiles;
    c.cen = a.cen;
    c.rad = a.rad;
    c.diam = T->diam.as<double>();
    c.group = a.group;
    c.near_factor = w.mixed ? o->near_field_factor : -1.0;
    c.tiny_gap = w.mixed ? std::ldexp(m->extent, -16) : -1.0;
    c.cull_margin = a.cull_margin;
    c.occ = occ;
    c.skip_groups = true;
    c.dim3 = w.dim3;
    if (occ && w.dim3) {
      c.nodesf = m->nodesf.as<NodeF>();
      c.n_nodes = m->n_nodes;
      c.frontier = m->frontier.as<int32_t>();
      c.n_frontier = m->n_frontier;
      c.leaf_of = m->leaf_of.as<int32_t>();
      c.sat = o->geometric_soup ? m->sat_geo.as<float4>() : m->sat_ref.as<float4>();
      c.sat_em = m->sat_em;
    }
    c.cls = T->tcls.as<uint8_t>();
    c.mask = T->tmask.as<uint32_t>();
    if (!s->fast_ctr.ptr && (rc = s->fast_ctr.alloc(s, 256))) return rc;
    c.claim = s->fast_ctr.as<unsigned long long>() + 1;
    c.counters = s->counters.as<unsigned long long>() + 13;
    const cudaError_t e = launch_tile_class(c, s->sm_count, s->stream);
    if (e != cudaSuccess) return cuda_err(e, "tile classification launch");
    if (n_kernels) *n_kernels += 1;
    a.tcls = c.cls;
    a.tmask = c.mask;
    w.ma.tcls = c.cls;
    w.ma.tmask = c.mask;
    if (!ray_log) {
      // The chunked pipeline's tiles: those with ray work (or near-field /
      // nearly coincident pairs in mixed precision), in row-major order; the
      // others go to the quadrature-only kernel (wave_fast).
      std::vector<uint8_t> cls(nt);
      cudaError_t e2 = cudaMemcpyAsync(cls.data(), c.cls, nt, cudaMemcpyDeviceToHost, s->stream);
      if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s->stream);
      if (e2 != cudaSuccess) return cuda_err(e2, "tile classes");
      const uint8_t need = w.mixed ? (uint8_t)(kClsSlow | kClsNear | kClsTiny) : (uint8_t)kClsSlow;
      std::vector<int32_t> work;
      w.row_end.assign((size_t)a.nT, 0);
      int64_t t = 0;
      for (int64_t bi = 0; bi < a.nT; ++bi) {
        for (int64_t bj = bi; bj < a.nT; ++bj, ++t)
          if (cls[(size_t)t] & need) work.push_back((int32_t)t);
        w.row_end[(size_t)bi] = (int64_t)work.size();
      }
      if (!work.empty()) {
        if (T->twork.bytes < sizeof(int32_t) * work.size() &&
            (rc = T->twork.alloc(s, sizeof(int32_t) * work.size())))
          return rc;
        e2 = cudaMemcpyAsync(T->twork.ptr, work.data(), sizeof(int32_t) * work.size(), cudaMemcpyHostToDevice,
                             s->stream);
        if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(s->stream);  // the host vector goes out of scope
        if (e2 != cudaSuccess) return cuda_err(e2, "tile list upload");
      }
      a.work = T->twork.as<int32_t>();
      w.ma.work = a.work;
      w.n_tiles = (int64_t)work.size();
      w.n_fast_tiles = a.n_tiles - w.n_tiles;
    }
  }
  TraceArgs& ta = w.ta;
  ta.N = N; ta.pmax = a.pmax; ta.dim3 = a.dim3; ta.tab = a.tab; ta.tabf = w.ma.tabf; ta.cen = a.cen;
  ta.group = a.group; ta.orig = a.orig; ta.nodes = a.nodes; ta.nodesf = occ ? m->nodesf.as<NodeF>() : nullptr; ta.n_nodes = a.n_nodes;
  ta.tris = a.tris; ta.trisf = w.ma.trisf; ta.segs = a.segs; ta.delta = w.ma.delta;
  ta.leaf_of = (occ && w.dim3 && !o->disable_pair_lists) ? m->leaf_of.as<int32_t>() : nullptr;
  ta.sat = (occ && w.dim3) ? (o->geometric_soup ? m->sat_geo.as<float4>() : m->sat_ref.as<float4>()) : nullptr;
  ta.sat_em = m->sat_em;
  ta.frontier = (occ && w.dim3) ? m->frontier.as<int32_t>() : nullptr;
  ta.n_frontier = (occ && w.dim3) ? m->n_frontier : 0;
  ta.rad = a.rad;
  ta.cull_margin = a.cull_margin;
  ta.ray_log = a.ray_log; ta.log_pm = a.log_pm;
  ResolveArgs& ra = w.ra;
  ra.N = N; ra.pmax = a.pmax; ra.dim3 = a.dim3; ra.tab = a.tab; ra.tabf = w.ma.tabf; ra.cen = a.cen;
  ra.diam = T->diam.as<double>(); ra.near_factor = o->near_field_factor; ra.area = a.area; ra.orig = a.orig;
  ra.F = a.F;
  w.nodes_d = a.nodes;
  w.nodes_f = w.ma.nodesf;
  return 0;
}

int fast_groups_auto(int64_t n_tiles, int sm_count) {
  const int64_t want = (int64_t)4 * 16 * std::max(sm_count, 1);  // four tasks per resident warp (16 per SM)
  int g = 1;
  while (g < 32 && n_tiles * g < want) g = g == 8 ? 32 : 2 * g;
  return g;
}

int wave_fast(Session* s, WaveReq& w, int64_t* n_kernels) {
  if (!w.pa.tcls || w.pa.ray_log || w.pa.n_tiles == 0) return 0;
  int rc = 0;
  if (!s->fast_ctr.ptr && (rc = s->fast_ctr.alloc(s, 256))) return rc;
  w.pa.fast_groups = w.ma.fast_groups =
      w.fast_groups > 0 ? w.fast_groups : fast_groups_auto(w.n_fast_tiles > 0 ? w.n_fast_tiles : w.pa.n_tiles,
                                                           s->sm_count);
  const int qb = w.fast_qb > 0 ? w.fast_qb : fast_qb_default(w.mixed, w.pmax);
  cudaError_t e = cudaMemsetAsync(s->fast_ctr.ptr, 0, sizeof(unsigned long long), s->stream);
  if (e == cudaSuccess)
    e = launch_fast(w.mixed, w.dim3, w.occ, qb, w.pa, w.ma, s->fast_ctr.as<unsigned long long>(),
                    s->counters.as<unsigned long long>(), s->sm_count, s->stream);
  if (e != cudaSuccess) return cuda_err(e, "quadrature-only tiles launch");
  if (n_kernels) *n_kernels += 1;
  w.pa.fast_done = true;
  w.ma.fast_done = true;
  return 0;
}

// Shared-memory shape of a launch over reqs.
WaveShape wave_shape(Session* s, WaveReq* const* reqs, int n) {
  WaveShape sh{};
  sh.mixed = reqs[0]->mixed;
  sh.dim3 = reqs[0]->dim3;
  sh.occ = reqs[0]->occ;
  for (int r = 0; r < n; ++r) sh.pmax_max = std::max(sh.pmax_max, reqs[r]->pmax);
  if (n == 1 && sh.occ) {
    sh.n_nodes_smem = reqs[0]->pa.n_nodes;
    sh.trace64_nodes_smem = trace_smem_bytes(false, sh.n_nodes_smem) <= (size_t)72 * 1024;
    sh.trace32_nodes_smem = sh.mixed && trace_smem_bytes(true, sh.n_nodes_smem) <= (size_t)80 * 1024;
    if (!sh.trace64_nodes_smem && !sh.trace32_nodes_smem) sh.n_nodes_smem = 0;
  }
  return sh;
}

namespace {

int ensure_blocks(Session* s) {
  int rc = 0;
  if (!s->wl_pair.ptr) {
    if ((rc = s->wl_pair.alloc(s, sizeof(PairArgs) * kMaxBatch))) return rc;
    if ((rc = s->wl_mixed.alloc(s, sizeof(MixedArgs) * kMaxBatch))) return rc;
    if ((rc = s->wl_trace.alloc(s, sizeof(TraceArgs) * kMaxBatch))) return rc;
    if ((rc = s->wl_resolve.alloc(s, sizeof(ResolveArgs) * kMaxBatch))) return rc;
    if ((rc = s->wl_tilebase.alloc(s, sizeof(int64_t) * (kMaxBatch + 1)))) return rc;
    if ((rc = s->wl_gen.alloc(s, sizeof(GenBatch)))) return rc;
    if ((rc = s->wl_tb.alloc(s, sizeof(TraceBatch)))) return rc;
    if ((rc = s->wl_rb.alloc(s, sizeof(ResolveBatch)))) return rc;
  }
  if (!s->h_ctr) {
    const cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&s->h_ctr), sizeof(unsigned long long) * kCtrCount, 0);
    if (e != cudaSuccess) return cuda_err(e, "cudaHostAlloc");
  }
  return 0;
}

uint64_t shape_key(const WaveShape& sh) {
  return (uint64_t)sh.mixed | ((uint64_t)sh.dim3 << 1) | ((uint64_t)sh.occ << 2) |
         ((uint64_t)sh.trace64_nodes_smem << 4) | ((uint64_t)sh.trace32_nodes_smem << 5) |
         ((uint64_t)sh.pmax_max << 8) | ((uint64_t)sh.gen_bps << 16) | ((uint64_t)sh.trace_bps << 20) |
         ((uint64_t)sh.n_nodes_smem << 24);
}

// The chunk's device work: counters reset, generation, traversal(s), resolve
// and the counters' copy to pinned host memory (with timing events when
// launched eagerly).
cudaError_t enqueue_chunk(Session* s, const WaveShape& sh, bool events) {
  cudaStream_t st = s->stream;
  cudaError_t e = cudaMemsetAsync(s->wq_ctr.ptr, 0, sizeof(unsigned long long) * kCtrCount, st);
  if (e != cudaSuccess) return e;
  if (events) cudaEventRecord(s->ev[0], st);
  if ((e = launch_gen(sh, s->wl_gen.as<GenBatch>(), s->sm_count, st)) != cudaSuccess) return e;
  if (events) cudaEventRecord(s->ev[1], st);
  if (sh.occ) {
    // the pair lists count as traversal time (the first traversal phase)
    const bool lists = sh.dim3;
    auto plist = [&]() -> cudaError_t {
      if (events) cudaEventRecord(s->ev[5], st);
      const cudaError_t el = launch_plist(s->wl_tb.as<TraceBatch>(), s->sm_count, st);
      if (events) cudaEventRecord(s->ev[6], st);
      return el;
    };
    if (lists && sh.mixed && (e = plist()) != cudaSuccess) return e;
    if (sh.mixed && (e = launch_trace(sh, s->wl_tb.as<TraceBatch>(), true, s->sm_count, st)) != cudaSuccess) return e;
    if (events) cudaEventRecord(s->ev[2], st);
    if (lists && !sh.mixed && (e = plist()) != cudaSuccess) return e;
    if ((e = launch_trace(sh, s->wl_tb.as<TraceBatch>(), false, s->sm_count, st)) != cudaSuccess) return e;
    if (events) cudaEventRecord(s->ev[3], st);
    if ((e = launch_resolve(sh, s->wl_rb.as<ResolveBatch>(), s->sm_count, st)) != cudaSuccess) return e;
    if (events) cudaEventRecord(s->ev[4], st);
  }
  return cudaMemcpyAsync(s->h_ctr, s->wq_ctr.ptr, sizeof(unsigned long long) * kCtrCount, cudaMemcpyDeviceToHost, st);
}

}  // namespace

int wave_chunk(Session* s, WaveReq* const* reqs_in, int n_in, bool use_graph, ChunkInfo* info, int gen_bps,
               int trace_bps, double pp_budget, const std::function<void()>* on_launched) {
  if (n_in < 1 || n_in > kMaxBatch) return set_err(RVF_EINVAL, "batch of %d requests (1..%d)", n_in, kMaxBatch);
  int rc = 0;
  if ((rc = ensure_blocks(s))) return rc;
  // tiles offered to this launch, in request order: all that remain, or as
  // many as the point-pair budget allows (the oldest requests first)
  std::vector<WaveReq*> reqs;
  std::vector<int64_t> offer;
  double left = pp_budget > 0 ? pp_budget : 1e300;
  for (int r = 0; r < n_in && left > 0; ++r) {
    const int64_t rem = reqs_in[r]->n_tiles - reqs_in[r]->claimed;
    if (rem <= 0) continue;
    const double per = (double)kTile * kTile * reqs_in[r]->pmax * reqs_in[r]->pmax;
    const int64_t take = (left >= per * (double)rem) ? rem : std::max<int64_t>(1, (int64_t)std::ceil(left / per));
    reqs.push_back(reqs_in[r]);
    offer.push_back(take);
    left -= per * (double)take;
  }
  if (reqs.empty()) return RVF_OK;
  const int n = (int)reqs.size();
  WaveShape sh = wave_shape(s, reqs.data(), n);
  sh.gen_bps = gen_bps;
  sh.trace_bps = trace_bps;
  std::vector<int64_t> base(n + 1, 0);
  for (int r = 0; r < n; ++r) base[r + 1] = base[r] + offer[r];
  WaveQ q{};
  if ((rc = ensure_wave(s, sh.mixed && sh.occ, sh.occ, sh.occ && sh.dim3, sh.pmax_max, base[n], q))) return rc;
  std::vector<PairArgs> pa(n);
  std::vector<MixedArgs> ma(n);
  std::vector<TraceArgs> ta(n);
  std::vector<ResolveArgs> ra(n);
  for (int r = 0; r < n; ++r) {
    pa[r] = reqs[r]->pa;
    ma[r] = reqs[r]->ma;
    ta[r] = reqs[r]->ta;
    ra[r] = reqs[r]->ra;
    pa[r].tile0 = ma[r].tile0 = reqs[r]->claimed;
    pa[r].q = ma[r].q = ta[r].q = q;
  }
  GenBatch g{};
  g.reqs = s->wl_pair.as<PairArgs>();
  g.mreqs = s->wl_mixed.as<MixedArgs>();
  g.tile_base = s->wl_tilebase.as<int64_t>();
  g.n_req = n;
  g.pmax_max = sh.pmax_max;
  g.total_tiles = base[n];
  g.claim_retries = reqs[0]->claim_retries;
  for (int r = 1; r < n; ++r) g.claim_retries = std::min(g.claim_retries, reqs[r]->claim_retries);
  g.q = q;
  g.counters = s->counters.as<unsigned long long>();
  g.err = s->err.as<int>();
  TraceBatch tb{};
  tb.reqs = s->wl_trace.as<TraceArgs>();
  tb.n_req = n;
  tb.nodes64_in_smem = sh.trace64_nodes_smem;
  tb.nodes32_in_smem = sh.trace32_nodes_smem;
  tb.smem_nodes64 = reqs[0]->nodes_d;
  tb.smem_nodes32 = reqs[0]->nodes_f;
  tb.n_nodes_smem = sh.n_nodes_smem;
  tb.q = q;
  tb.counters = g.counters;
  ResolveBatch rb{};
  rb.reqs = s->wl_resolve.as<ResolveArgs>();
  rb.n_req = n;
  rb.q = q;
  cudaStream_t st = s->stream;
  cudaError_t e = cudaSuccess;
  auto up = [&](DevBuf& d, const void* h, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.ptr, h, bytes, cudaMemcpyHostToDevice, st);
  };
  up(s->wl_pair, pa.data(), sizeof(PairArgs) * n);
  up(s->wl_mixed, ma.data(), sizeof(MixedArgs) * n);
  up(s->wl_trace, ta.data(), sizeof(TraceArgs) * n);
  up(s->wl_resolve, ra.data(), sizeof(ResolveArgs) * n);
  up(s->wl_tilebase, base.data(), sizeof(int64_t) * (n + 1));
  up(s->wl_gen, &g, sizeof g);
  up(s->wl_tb, &tb, sizeof tb);
  up(s->wl_rb, &rb, sizeof rb);
  if (e != cudaSuccess) return cuda_err(e, "launch block upload");
  bool replayed = false;
  if (use_graph) {
    const uint64_t key = shape_key(sh);
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const cudaError_t e1 = enqueue_chunk(s, sh, false);
        const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
        if (e1 == cudaSuccess && e2 == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess)
          it = s->graphs.emplace(key, exec).first;
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();  // a refused capture falls back to eager launches
      }
    }
    if (it != s->graphs.end()) {
      if ((e = cudaGraphLaunch(it->second, st)) != cudaSuccess) return cuda_err(e, "graph launch");
      replayed = true;
    }
  }
  if (!replayed && (e = enqueue_chunk(s, sh, info != nullptr)) != cudaSuccess) return cuda_err(e, "pair pipeline launch");
  if (on_launched) (*on_launched)();
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_err(e, "pair pipeline");
  if (info) {
    *info = ChunkInfo{};
    info->graph = replayed;
    info->kernels = 1 + (sh.occ ? (sh.mixed ? 3 : 2) + (sh.dim3 ? 1 : 0) : 0);
    if (!replayed) {
      float t = 0.f;
      cudaEventElapsedTime(&t, s->ev[0], s->ev[1]);
      info->ms_gen = t;
      if (sh.occ) {
        float t12 = 0.f, t23 = 0.f, t34 = 0.f;
        cudaEventElapsedTime(&t12, s->ev[1], s->ev[2]);
        cudaEventElapsedTime(&t23, s->ev[2], s->ev[3]);
        cudaEventElapsedTime(&t34, s->ev[3], s->ev[4]);
        info->ms_trace = sh.mixed ? t12 : t23;
        info->ms_trace_fp64 = sh.mixed ? t23 : 0.0;
        info->ms_resolve = t34;
        if (sh.dim3) {
          float tl = 0.f;
          cudaEventElapsedTime(&tl, s->ev[5], s->ev[6]);
          info->ms_lists = tl;
        }
      }
    }
    info->rays_traced = (int64_t)(sh.mixed ? s->h_ctr[kCtrRec32] : s->h_ctr[kCtrRec64]);
  }
  // tiles are claimed in launch order: request r got min(claimed - base[r], its remaining tiles)
  const int64_t got = (int64_t)s->h_ctr[kCtrTile];
  for (int r = 0; r < n; ++r) {
    const int64_t take = std::max<int64_t>(0, std::min<int64_t>(got - base[r], base[r + 1] - base[r]));
    reqs[r]->claimed += take;
  }
  return 0;
}

}  // namespace rvf
