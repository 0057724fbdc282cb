// server.cpp -- the continuous-batching request loop (include/rvf_b200.h,
// "Serving").  One worker thread per server: FIFO admission by device
// footprint, batched chunks of the wavefront pipeline over every admitted
// quadrature request of one launch class, CUDA-graph replay per launch shape,
// a grid-size sweep per class, Monte Carlo requests between chunks.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/rvf_b200.h"
#include "kernels.h"
#include "rvf_internal.h"
#include "wave_host.h"

using namespace rvf;

namespace {

using Clock = std::chrono::steady_clock;

// Owned copy of a mesh description (the caller may free its buffers once
// rvf_submit returns).
struct MeshCopy {
  std::vector<double> coords, soup;
  std::vector<int8_t> fam;
  std::vector<int32_t> idx, group, tags, obs_group;
  std::vector<int32_t> nodes[6];
  rvf_mesh_desc d{};

  void take(const rvf_mesh_desc* s) {
    d = *s;
    coords.assign(s->coords, s->coords + (s->coords ? 3 * s->n_nodes : 0));
    fam.assign(s->elem_family, s->elem_family + (s->elem_family ? s->n_elems : 0));
    idx.assign(s->elem_node_idx, s->elem_node_idx + (s->elem_node_idx ? s->n_elems : 0));
    group.assign(s->elem_group, s->elem_group + (s->elem_group ? s->n_elems : 0));
    static const int k[6] = {8, 6, 4, 3, 3, 2};
    for (int f = 0; f < 6; ++f) {
      if (s->nodes[f]) nodes[f].assign(s->nodes[f], s->nodes[f] + k[f] * s->n_family[f]);
      else nodes[f].clear();
      d.nodes[f] = s->nodes[f] ? nodes[f].data() : nullptr;
    }
    if (s->n_obs > 0 && s->obs_soup) {
      soup.assign(s->obs_soup, s->obs_soup + (size_t)3 * s->obs_nv * s->n_obs);
      obs_group.assign(s->obs_group, s->obs_group + s->n_obs);
      d.obs_soup = soup.data();
      d.obs_group = obs_group.data();
    } else {
      d.obs_soup = nullptr;
      d.obs_group = nullptr;
    }
    tags.assign(s->group_tags, s->group_tags + (s->group_tags ? s->n_groups : 0));
    d.coords = coords.data();
    d.elem_family = fam.data();
    d.elem_node_idx = idx.data();
    d.elem_group = group.data();
    d.group_tags = tags.data();
  }
  void drop() { *this = MeshCopy{}; }
};

struct Req {
  int64_t id = 0;
  int state = RVF_REQ_QUEUED;
  int status = RVF_OK;
  MeshCopy mesh;
  rvf_options opts{};
  uint64_t footprint = 0;
  int64_t n_elems = 0;
  bool quad = true;
  bool cancel = false;
  rvf_mesh* m = nullptr;
  Tables* T = nullptr;
  WaveReq w;
  double t_submit = 0, t_admit = -1, t_done = -1;
  int64_t n_chunks = 0;
  // Monte Carlo progress (tiles of the upper triangle)
  int64_t mc_tiles = 0, mc_claimed = 0;
  bool mc_area_done = false;
};

// points per element of the quadrature rules (upper bound over the families present)
int pmax_of(const rvf_mesh_desc* d, int nquad) {
  int pm = 1;
  const int tri = nquad <= 1 ? 1 : nquad == 2 ? 3 : nquad == 3 ? 7 : 13;  // src/GPUKernels.jl:414-439
  for (int f = 0; f < 6; ++f) {
    if (d->n_family[f] <= 0) continue;
    const int p = (f == RVF_QUAD8 || f == RVF_QUAD4) ? nquad * nquad : (f == RVF_TRI6 || f == RVF_TRI3) ? tri : nquad;
    pm = std::max(pm, p);
  }
  return pm;
}

// Device memory a request holds from admission to release: F, the
// quadrature tables (FP64, plus FP32 in mixed mode), per-element arrays,
// BVH, reductions.
uint64_t footprint_of(const rvf_mesh_desc* d, const rvf_options* o) {
  const uint64_t N = (uint64_t)std::max<int64_t>(d->n_elems, 0);
  const uint64_t tiles = (N + kTile - 1) / kTile;
  const uint64_t pm = (uint64_t)pmax_of(d, o->nquad);
  const uint64_t G = (uint64_t)std::max(d->n_groups, 1);
  uint64_t b = (uint64_t)(8.0 * 1.19 * (double)std::max<uint64_t>(N * N, 1));  // F, in its size class
  b += tiles * kTile * kComp * pm * 8;                                     // FP64 table
  if (o->precision == RVF_PREC_MIXED) b += tiles * kTile * kComp * pm * 4;  // FP32 table
  b += N * 256 + 24 * (uint64_t)std::max<int64_t>(d->n_nodes, 0);          // per-element arrays, coordinates
  b += (uint64_t)std::max<int64_t>(d->n_obs, 0) * 400;                    // BVH nodes and primitives, both precisions
  b += (uint64_t)std::min<uint64_t>(256, std::max<uint64_t>(1, (1u << 20) / std::max<uint64_t>(N, 1))) * G * N * 8;
  b += (G * N + G * G + G + N) * 8;                                        // row-group, group and row sums
  b += tiles * (tiles + 1) / 2 * (1 + kTile * 4);                          // tile classes and masks
  return b + (1u << 20);
}

}  // namespace

struct rvf_server {
  rvf_session* s = nullptr;
  rvf_server_opts o{};
  uint64_t admit_budget = 0, admitted = 0, admitted_peak = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int64_t> finished_ids;  // finished requests not yet returned by rvf_wait_any
  std::deque<Req*> queue;
  std::vector<Req*> active;
  std::map<int64_t, std::unique_ptr<Req>> reqs;
  std::vector<rvf_mesh*> to_free;  // meshes of released requests, freed by the worker
  int64_t next_id = 1;
  bool closing = false;
  std::thread worker;
  Clock::time_point t0;
  // statistics
  int64_t submitted = 0, completed = 0, failed = 0, canceled = 0;
  int64_t chunks = 0, graph_replays = 0, batched = 0, pairs_done = 0;
  double ms_admit = 0, ms_quad = 0, ms_mc = 0, ms_free = 0, ms_idle = 0;  // worker time by activity
  double share_mc = 0, share_quad = 0;           // the same while both kinds wait (time sharing)
  std::vector<double> latencies;
  double first_submit = -1, last_done = 0;
  double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
};

namespace {

// Work offered to one launch: tens of milliseconds, so that arrivals join
// and the oldest requests finish at short intervals (quadrature point pairs
// of the mixed pipeline; Monte Carlo sample pairs, each of which evaluates
// both elements' geometry).
constexpr double kChunkPointPairs = 6e9;
constexpr double kChunkSamplePairs = 2e9;

const int kCand[][2] = {{0, 0}, {2, 0}, {0, 2}, {2, 2}};
constexpr int kNCand = 4;

// Candidate shapes of the quadrature-only kernel: the default (points by the
// rule, tasks per tile by the tile count), about half the points per lane
// block (fewer registers, more resident warps), and the next finer and the
// next coarser split of a tile into warp tasks (1, 2, 4, 8, 32).
constexpr int kNFastCand = 4;
void fast_cand(bool mixed, int pmax, int64_t n_tiles, int sm_count, size_t c, int& qb, int& groups) {
  static const int steps[5] = {1, 2, 4, 8, 32};
  const int d = fast_qb_default(mixed, pmax);
  const int ga = fast_groups_auto(n_tiles, sm_count);
  int k = 0;
  while (steps[k] != ga) ++k;
  qb = d;
  groups = ga;
  if (c == 1) qb = std::max(2, (d + 1) / 2);
  if (c == 2) groups = steps[k < 4 ? k + 1 : 2];
  if (c == 3) groups = steps[k > 0 ? k - 1 : 2];
}

// launch class: precision, surface or curve mesh, occlusion
uint64_t class_key(const Req* r) {
  return (uint64_t)r->w.mixed | ((uint64_t)r->w.dim3 << 1) | ((uint64_t)r->w.occ << 2);
}

// launch class and size class (4^k <= quadrature-only tiles < 4^(k+1))
uint64_t fast_key(uint64_t class_key, int64_t n_fast_tiles) {
  int k = 0;
  while (k < 15 && ((int64_t)1 << (2 * (k + 1))) <= n_fast_tiles) ++k;
  return class_key | ((uint64_t)k << 8);
}

void finish(rvf_server* sv, Req* r, int state, int status) {  // sv->mu held
  r->state = state;
  r->status = status;
  r->t_done = sv->now_ms();
  if (state == RVF_REQ_DONE) {
    ++sv->completed;
    sv->latencies.push_back(r->t_done - r->t_submit);
    sv->last_done = std::max(sv->last_done, r->t_done);
    sv->pairs_done += r->n_elems * (r->n_elems - 1) / 2;
  } else if (state == RVF_REQ_FAILED) {
    ++sv->failed;
  } else if (state == RVF_REQ_CANCELED) {
    ++sv->canceled;
  }
  sv->finished_ids.push_back(r->id);
  sv->cv_done.notify_all();
}

// Hands a request's device memory to the worker, which frees it before its
// next admission, and drops the request's admission charge (sv->mu held).
// The caller -- rvf_release on a client thread -- thus never waits for the
// session lock, which the worker holds while a chunk runs.
void drop_device(rvf_server* sv, Req* r) {
  if (r->m) {
    sv->to_free.push_back(r->m);
    r->m = nullptr;
    r->T = nullptr;
  }
  if (r->footprint && r->t_admit >= 0) {
    sv->admitted -= std::min(sv->admitted, r->footprint);
    r->footprint = 0;
  }
  sv->cv_work.notify_all();
}

// Upload and tables of an admitted request (no server lock held).
int admit_one(rvf_server* sv, Req* r) {
  Session* s = sv->s;
  int rc = rvf_mesh_upload(s, &r->mesh.d, &r->m);
  if (rc) return rc;
  r->mesh.drop();
  std::lock_guard<std::mutex> lk(s->mu);
  cudaSetDevice(s->device);
  rvf_mesh* m = r->m;
  if ((rc = validate_options(m, &r->opts))) return rc;
  if (!r->quad) {
    const int64_t N = m->N, nT = (N + kTile - 1) / kTile;
    if (m->mc_area.bytes < sizeof(double) * std::max<int64_t>(N, 1))
      if ((rc = m->mc_area.alloc(s, sizeof(double) * std::max<int64_t>(N, 1)))) return rc;
    if (m->F.bytes < sizeof(double) * N * N)
      if ((rc = m->F.alloc(s, sizeof(double) * std::max<int64_t>(N * N, 1)))) return rc;
    if ((rc = reduce_alloc(s, m))) return rc;
    if ((rc = mc_classify(s, m, &r->opts))) return rc;
    m->has_result = false;
    r->mc_tiles = nT * (nT + 1) / 2;
    const cudaError_t e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? RVF_OK : cuda_err(e, "request set-up");
  }
  if (r->opts.precision == RVF_PREC_MIXED && !(r->opts.near_field_factor >= 0.0))
    return set_err(RVF_EINVAL, "near_field_factor must be >= 0");
  if ((rc = ensure_tables(s, m, r->opts.nquad, &r->T))) return rc;
  const int64_t N = m->N;
  if (m->F.bytes < sizeof(double) * N * N)
    if ((rc = m->F.alloc(s, sizeof(double) * std::max<int64_t>(N * N, 1)))) return rc;
  if ((rc = reduce_alloc(s, m))) return rc;
  m->has_result = false;
  if (N == 1) cudaMemsetAsync(m->F.ptr, 0, sizeof(double), s->stream);
  if ((rc = wave_prepare(s, m, r->T, &r->opts, nullptr, r->w, nullptr))) return rc;
  // the quadrature-only kernel's shape: the caller's, the tuned one, or --
  // on the first request of its launch class and size class -- the fastest
  // candidate, every candidate run on this request (each forms the same F)
  const bool own = r->opts.fast_points != 0 || r->opts.fast_row_groups != 0;
  const uint64_t fkey = fast_key(class_key(r), r->w.n_fast_tiles) | ((uint64_t)r->w.pmax << 16);
  bool sweep = false;
  if (!own && r->w.n_fast_tiles > 0) {
    std::lock_guard<std::mutex> lk2(s->tune_mu);
    const auto it = s->ftune.find(fkey);
    if (it != s->ftune.end() && it->second.done) {
      r->w.fast_qb = it->second.qb;
      r->w.fast_groups = it->second.groups;
    } else {
      sweep = sv->o.autotune >= 0;
    }
  }
  if (!sweep) {
    if ((rc = wave_fast(s, r->w, nullptr))) return rc;
    const cudaError_t e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? RVF_OK : cuda_err(e, "request set-up");
  }
  cudaError_t e = preload_fast();
  if (e != cudaSuccess) return cuda_err(e, "kernel load");
  FastTune t;
  const double gpp = (double)r->w.n_fast_tiles * kTile * kTile * r->w.pmax * r->w.pmax * 1e-9;
  for (int c = 0; c < kNFastCand; ++c) {
    fast_cand(r->w.mixed, r->w.pmax, r->w.n_fast_tiles, s->sm_count, (size_t)c, r->w.fast_qb, r->w.fast_groups);
    cudaEventRecord(s->ev[0], s->stream);
    if ((rc = wave_fast(s, r->w, nullptr))) return rc;
    cudaEventRecord(s->ev[1], s->stream);
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return cuda_err(e, "request set-up");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]);
    t.score[c] = (double)ms / gpp;
  }
  size_t b = 0;
  for (size_t c = 1; c < (size_t)kNFastCand; ++c)
    if (t.score[c] < t.score[b]) b = c;
  fast_cand(r->w.mixed, r->w.pmax, r->w.n_fast_tiles, s->sm_count, b, t.qb, t.groups);
  t.done = true;
  std::lock_guard<std::mutex> lk2(s->tune_mu);
  if (!s->ftune[fkey].done) {
    s->ftune[fkey] = t;
    s->ftune_done.push_back(fkey);
  }
  return RVF_OK;
}

// Self pairs, Duffy pairs, the one-element case and the reductions of a
// request whose tiles are all integrated (s->mu held) -- the tail of rvf_solve.
int finish_quad(Session* s, Req* r) {
  rvf_mesh* m = r->m;
  const rvf_options& o = r->opts;
  const int64_t N = m->N;
  int rc = 0;
  cudaError_t e = cudaSuccess;
  if (o.self_vf && N > 0 && (e = launch_self_pairs(s, r->w.pa, s->stream)) != cudaSuccess)
    return cuda_err(e, "self-pair kernel launch");
  if (o.use_duffy && m->dim == 2 && N > 0) {
    DuffyArgs d{};
    if ((rc = ensure_duffy(s, m, o.nquad, &d.p01, &d.w01))) return rc;
    d.N = N;
    d.nq = o.nquad;
    d.pairs = m->duffy_pairs.as<DuffyPair>();
    d.n_pairs = m->n_duffy + (o.self_vf ? m->n_duffy_self : 0);
    d.coords = m->coords.as<double>();
    d.enodes = m->enodes.as<int32_t>();
    d.area_orig = r->T->area_orig.as<double>();
    d.F = m->F.as<double>();
    d.nodes = r->w.pa.nodes;
    d.n_nodes = r->w.pa.n_nodes;
    d.tris = r->w.pa.tris;
    d.counters = s->counters.as<unsigned long long>();
    if (d.n_pairs > 0 && (e = launch_duffy(d, s->stream)) != cudaSuccess) return cuda_err(e, "Duffy kernel launch");
  }
  if (N == 1) {
    const double nanv = std::nan("");
    cudaMemcpyAsync(m->F.ptr, &nanv, sizeof(double), cudaMemcpyHostToDevice, s->stream);
  }
  if ((rc = run_reduce(s, m, r->T->area_orig.as<double>()))) return rc;
  if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return cuda_err(e, "request finish");
  if ((rc = read_err(s))) return rc;
  m->has_result = true;
  m->result_area = r->T->area_orig.as<double>();
  return RVF_OK;
}


// One batched chunk over reqs (same class); finishes the requests it completes.
void run_chunk(rvf_server* sv, std::vector<Req*>& batch) {
  Session* s = sv->s;
  const uint64_t key = class_key(batch[0]);
  int gen = 0, trace = 0;
  size_t cand = 0;
  bool tuning = false;
  {
    std::lock_guard<std::mutex> lk(s->tune_mu);
    GridTune& t = s->grid_tune[key];
    if (sv->o.autotune >= 0 && !t.done && batch[0]->w.occ) {
      tuning = true;
      cand = t.next;
      gen = kCand[cand][0];
      trace = kCand[cand][1];
    } else if (t.done) {
      gen = t.gen;
      trace = t.trace;
    }
  }
  std::vector<WaveReq*> w(batch.size());
  std::vector<int64_t> before(batch.size());
  int64_t pp = 0;
  for (size_t k = 0; k < batch.size(); ++k) {
    w[k] = &batch[k]->w;
    before[k] = w[k]->claimed;
  }
  int rc = 0;
  ChunkInfo info;
  const auto c0 = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    cudaSetDevice(s->device);
    cudaMemsetAsync(s->err.ptr, 0, sizeof(int), s->stream);
    rc = wave_chunk(s, w.data(), (int)w.size(), sv->o.use_graphs >= 0, &info, gen, trace, kChunkPointPairs);
    if (!rc) rc = read_err(s);
  }
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - c0).count();
  std::vector<Req*> done;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    ++sv->chunks;
    sv->graph_replays += info.graph ? 1 : 0;
    sv->batched += (int64_t)batch.size();
    int pm = 1;
    for (size_t k = 0; k < batch.size(); ++k) {
      Req* r = batch[k];
      r->n_chunks += 1;
      pp += w[k]->claimed - before[k];
      pm = std::max(pm, w[k]->pmax);
      if (rc) {
        finish(sv, r, RVF_REQ_FAILED, rc);
        drop_device(sv, r);
      } else if (w[k]->done()) {
        done.push_back(r);
      }
    }
    if (!rc && pp == 0) {  // the queues could not take one tile: fail the batch rather than spin
      rc = no_progress(s);
      for (Req* r : batch) {
        finish(sv, r, RVF_REQ_FAILED, rc);
        drop_device(sv, r);
      }
      done.clear();
    }
    if (rc) {
      sv->active.erase(std::remove_if(sv->active.begin(), sv->active.end(),
                                      [](Req* r) { return r->state != RVF_REQ_RUNNING; }),
                       sv->active.end());
    }
    if (tuning && !rc && pp > 0) {
      std::lock_guard<std::mutex> lk2(s->tune_mu);
      GridTune& t = s->grid_tune[key];
      t.score.resize(kNCand, 0.0);
      t.score[cand] = ms / ((double)pp * kTile * kTile * pm * pm * 1e-6);
      if (++t.next >= (size_t)kNCand) {
        size_t b = 0;
        for (size_t c = 1; c < (size_t)kNCand; ++c)
          if (t.score[c] < t.score[b]) b = c;
        t.gen = kCand[b][0];
        t.trace = kCand[b][1];
        t.done = true;
      }
    }
  }
  for (Req* r : done) {
    int frc;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      cudaSetDevice(s->device);
      frc = finish_quad(s, r);
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->active.erase(std::remove(sv->active.begin(), sv->active.end(), r), sv->active.end());
    if (frc) {
      finish(sv, r, RVF_REQ_FAILED, frc);
      drop_device(sv, r);
    } else {
      finish(sv, r, RVF_REQ_DONE, RVF_OK);
    }
  }
}

// One chunk of a Monte Carlo request (the area rule on its first chunk);
// finishes the request after its last tile.
void run_mc_chunk(rvf_server* sv, Req* r) {
  Session* s = sv->s;
  int rc = 0;
  bool fin = false;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    cudaSetDevice(s->device);
    McArgs c{};
    fill_mc_args(s, r->m, &r->opts, nullptr, c);
    // a whole number of waves of the persistent grid: no partial last wave
    const double per = (double)kTile * kTile * std::max(1, r->opts.n_samples);
    const int64_t grid = mc_resident_blocks(c, s->sm_count);
    const int64_t budget = grid * std::max<int64_t>(1, (int64_t)(kChunkSamplePairs / per) / grid);
    c.tile0 = r->mc_claimed;
    c.tile_count = std::min<int64_t>(r->mc_tiles - r->mc_claimed, budget);
    c.area_pass = !r->mc_area_done;
    cudaMemsetAsync(s->err.ptr, 0, sizeof(int), s->stream);
    cudaMemsetAsync(s->tile_counter.ptr, 0, 8, s->stream);
    cudaError_t e = launch_mc(c, s->sm_count, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    rc = (e != cudaSuccess) ? cuda_err(e, "Monte Carlo chunk") : read_err(s);
    if (!rc) {
      r->mc_claimed += std::max<int64_t>(c.tile_count, 0);
      r->mc_area_done = true;
      if (r->mc_claimed >= r->mc_tiles) {
        rc = run_reduce(s, r->m, r->m->mc_area.as<double>());
        if (!rc && (e = cudaStreamSynchronize(s->stream)) != cudaSuccess) rc = cuda_err(e, "Monte Carlo finish");
        if (!rc) {
          r->m->has_result = true;
          r->m->result_area = r->m->mc_area.as<double>();
          fin = true;
        }
      }
    }
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  ++sv->chunks;
  r->n_chunks += 1;
  if (rc || fin) sv->active.erase(std::remove(sv->active.begin(), sv->active.end(), r), sv->active.end());
  if (rc) {
    finish(sv, r, RVF_REQ_FAILED, rc);
    drop_device(sv, r);
  } else if (fin) {
    finish(sv, r, RVF_REQ_DONE, RVF_OK);
  }
}

void worker_loop(rvf_server* sv);

// The worker thread: an exception (a failed host allocation) fails the
// requests in progress, whose state is then unknown, and the loop goes on.
void worker_main(rvf_server* sv) {
  for (;;) {
    try {
      worker_loop(sv);
      return;
    } catch (...) {
      const int rc = exception_status();
      std::lock_guard<std::mutex> lk(sv->mu);
      for (auto& kv : sv->reqs) {
        Req* r = kv.second.get();
        if (r->state != RVF_REQ_RUNNING) continue;
        finish(sv, r, RVF_REQ_FAILED, rc);
        drop_device(sv, r);
      }
      sv->active.clear();
    }
  }
}

// Frees the meshes of released and failed requests (no lock held).
void free_released(rvf_server* sv) {
  std::vector<rvf_mesh*> fr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    fr.swap(sv->to_free);
  }
  if (fr.empty()) return;
  const auto f0 = Clock::now();
  for (rvf_mesh* m : fr) rvf_mesh_release(sv->s, m);
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->ms_free += std::chrono::duration<double, std::milli>(Clock::now() - f0).count();
}

void worker_loop(rvf_server* sv) {
  for (;;) {
    free_released(sv);
    std::vector<Req*> admit;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      // requests cancelled while running leave at a chunk boundary
      for (Req* r : sv->active)
        if (r->cancel) {
          finish(sv, r, RVF_REQ_CANCELED, RVF_ECANCELED);
          drop_device(sv, r);
        }
      sv->active.erase(std::remove_if(sv->active.begin(), sv->active.end(),
                                      [](Req* r) { return r->state != RVF_REQ_RUNNING; }),
                       sv->active.end());
      // FIFO admission while the footprints fit
      while (!sv->queue.empty()) {
        Req* r = sv->queue.front();
        if (r->cancel) {
          sv->queue.pop_front();
          finish(sv, r, RVF_REQ_CANCELED, RVF_ECANCELED);
          continue;
        }
        if (r->footprint > sv->admit_budget) {
          sv->queue.pop_front();
          r->mesh.drop();
          finish(sv, r, RVF_REQ_FAILED, RVF_EBUDGET);
          continue;
        }
        if (sv->admitted + r->footprint > sv->admit_budget) break;
        sv->queue.pop_front();
        sv->admitted += r->footprint;
        sv->admitted_peak = std::max(sv->admitted_peak, sv->admitted);
        r->state = RVF_REQ_RUNNING;
        r->t_admit = sv->now_ms();
        admit.push_back(r);
      }
      if (admit.empty() && sv->active.empty()) {
        if (sv->closing && sv->queue.empty()) return;
        const auto w0 = Clock::now();
        sv->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        sv->ms_idle += std::chrono::duration<double, std::milli>(Clock::now() - w0).count();
        continue;
      }
    }
    for (Req* r : admit) {
      const auto a0 = Clock::now();
      const int rc = admit_one(sv, r);
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->ms_admit += std::chrono::duration<double, std::milli>(Clock::now() - a0).count();
      if (rc) {
        finish(sv, r, RVF_REQ_FAILED, rc);
        drop_device(sv, r);
      } else if (r->quad && r->w.done()) {  // no tiles (empty mesh)
        std::lock_guard<std::mutex> lk2(sv->s->mu);
        const int frc = finish_quad(sv->s, r);
        if (frc) {
          finish(sv, r, RVF_REQ_FAILED, frc);
          drop_device(sv, r);
        } else {
          finish(sv, r, RVF_REQ_DONE, RVF_OK);
        }
      } else {
        sv->active.push_back(r);
      }
    }
    // next piece of work: a chunk of the oldest admitted Monte Carlo
    // request (alone), or of the oldest quadrature request together with
    // every request of its class.  While both kinds wait, each gets half of
    // the worker's time, so short quadrature requests do not queue behind a
    // long Monte Carlo one (a 40,000-element request takes ~20 s).
    Req* mc = nullptr;
    std::vector<Req*> batch;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      const int maxb = (sv->o.max_batch >= 1 && sv->o.max_batch <= kMaxBatch) ? sv->o.max_batch : kMaxBatch;
      Req* head_q = nullptr;
      Req* head_mc = nullptr;
      for (Req* r : sv->active) {
        if (r->cancel) continue;
        if (r->quad && !r->w.done() && !head_q) head_q = r;
        if (!r->quad && !head_mc) head_mc = r;
      }
      if (!head_q || !head_mc) sv->share_mc = sv->share_quad = 0.0;  // no contention: no debt either way
      const Req* head = nullptr;
      if (head_mc && (!head_q || sv->share_mc <= sv->share_quad)) head = head_mc;
      else head = head_q;
      if (head && !head->quad) {
        mc = const_cast<Req*>(head);
      } else if (head) {
        const uint64_t key = class_key(head);
        for (Req* r : sv->active)
          if (!r->cancel && r->quad && !r->w.done() && class_key(r) == key && (int)batch.size() < maxb)
            batch.push_back(r);
      }
    }
    const auto c0 = Clock::now();
    if (mc) run_mc_chunk(sv, mc);
    else if (!batch.empty()) run_chunk(sv, batch);
    const double ms = std::chrono::duration<double, std::milli>(Clock::now() - c0).count();
    std::lock_guard<std::mutex> lk(sv->mu);
    (mc ? sv->ms_mc : sv->ms_quad) += ms;
    (mc ? sv->share_mc : sv->share_quad) += ms;
  }
}

Req* find(rvf_server* sv, int64_t id) {
  auto it = sv->reqs.find(id);
  return it == sv->reqs.end() ? nullptr : it->second.get();
}

int report(const Req* r, rvf_request_info* info) {
  if (info) {
    *info = rvf_request_info{};
    info->state = r->state;
    info->status = r->status;
    info->n_elems = r->n_elems;
    info->footprint_bytes = r->footprint;
    info->t_submit_ms = r->t_submit;
    info->t_admit_ms = r->t_admit;
    info->t_done_ms = r->t_done;
    info->n_chunks = r->n_chunks;
  }
  switch (r->state) {
    case RVF_REQ_DONE: return RVF_OK;
    case RVF_REQ_FAILED: return r->status ? r->status : RVF_ECUDA;
    case RVF_REQ_CANCELED: return RVF_ECANCELED;
    default: return RVF_EBUSY;
  }
}

}  // namespace

extern "C" {

int rvf_server_create(rvf_session* s, const rvf_server_opts* o, rvf_server** out) try {
  if (!s || !out) return set_err(RVF_EINVAL, "null argument");
  auto sv = std::make_unique<rvf_server>();
  sv->s = s;
  if (o) sv->o = *o;
  if (sv->o.max_batch < 0 || sv->o.max_batch > kMaxBatch)
    return set_err(RVF_EINVAL, "max_batch %d outside 0..%d", sv->o.max_batch, kMaxBatch);
  sv->admit_budget = sv->o.admit_bytes ? sv->o.admit_bytes : (uint64_t)(0.7 * (double)s->budget);
  sv->t0 = Clock::now();
  sv->worker = std::thread(worker_main, sv.get());
  *out = sv.release();
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_server_destroy(rvf_server* sv) try {
  if (!sv) return RVF_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->closing = true;
    for (Req* r : sv->queue) r->cancel = true;
    for (Req* r : sv->active) r->cancel = true;
    sv->cv_work.notify_all();
  }
  if (sv->worker.joinable()) sv->worker.join();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (auto& kv : sv->reqs) drop_device(sv, kv.second.get());
    sv->reqs.clear();
  }
  free_released(sv);
  delete sv;
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_submit(rvf_server* sv, const rvf_mesh_desc* d, const rvf_options* o, int64_t* id) try {
  if (!sv || !d || !o || !id) return set_err(RVF_EINVAL, "null argument");
  if (o->ray_log) return set_err(RVF_EINVAL, "ray_log is not supported by the server");
  if (d->n_elems < 0 || d->n_elems > INT32_MAX) return set_err(RVF_EINVAL, "n_elems %lld out of range", (long long)d->n_elems);
  auto r = std::make_unique<Req>();
  r->mesh.take(d);
  r->opts = *o;
  r->n_elems = d->n_elems;
  r->quad = (o->method == RVF_METHOD_QUADRATURE);
  r->footprint = footprint_of(d, o);
  std::lock_guard<std::mutex> lk(sv->mu);
  if (sv->closing) return set_err(RVF_ECLOSED, "server is shutting down");
  r->id = sv->next_id++;
  r->t_submit = sv->now_ms();
  if (sv->first_submit < 0) sv->first_submit = r->t_submit;
  *id = r->id;
  sv->queue.push_back(r.get());
  sv->reqs.emplace(r->id, std::move(r));
  ++sv->submitted;
  sv->cv_work.notify_all();
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_poll(rvf_server* sv, int64_t id, rvf_request_info* info) try {
  if (!sv) return set_err(RVF_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  Req* r = find(sv, id);
  if (!r) return set_err(RVF_EINVAL, "unknown request %lld", (long long)id);
  return report(r, info);
} catch (...) {
  return exception_status();
}

int rvf_wait(rvf_server* sv, int64_t id, int64_t timeout_ms, rvf_request_info* info) try {
  if (!sv) return set_err(RVF_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(sv->mu);
  Req* r = find(sv, id);
  if (!r) return set_err(RVF_EINVAL, "unknown request %lld", (long long)id);
  auto ready = [&] { return r->state != RVF_REQ_QUEUED && r->state != RVF_REQ_RUNNING; };
  if (timeout_ms < 0) sv->cv_done.wait(lk, ready);
  else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    report(r, info);
    return set_err(RVF_ETIMEDOUT, "request %lld still in progress after %lld ms", (long long)id, (long long)timeout_ms);
  }
  const int rc = report(r, info);
  if (rc == RVF_ECANCELED) return set_err(rc, "request %lld was cancelled", (long long)id);
  if (rc != RVF_OK) return set_err(rc, "request %lld failed (status %d)", (long long)id, rc);
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_wait_any(rvf_server* sv, int64_t timeout_ms, int64_t* id) try {
  if (!sv || !id) return set_err(RVF_EINVAL, "null argument");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto ready = [&] { return !sv->finished_ids.empty(); };
  if (timeout_ms < 0) sv->cv_done.wait(lk, ready);
  else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return set_err(RVF_ETIMEDOUT, "no request finished within %lld ms", (long long)timeout_ms);
  *id = sv->finished_ids.front();
  sv->finished_ids.pop_front();
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_cancel(rvf_server* sv, int64_t id) try {
  if (!sv) return set_err(RVF_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  Req* r = find(sv, id);
  if (!r) return set_err(RVF_EINVAL, "unknown request %lld", (long long)id);
  if (r->state == RVF_REQ_QUEUED || r->state == RVF_REQ_RUNNING) r->cancel = true;
  sv->cv_work.notify_all();
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_request_result_device(rvf_server* sv, int64_t id, const double** F_dev, const double** A_dev) try {
  if (!sv) return set_err(RVF_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  Req* r = find(sv, id);
  if (!r) return set_err(RVF_EINVAL, "unknown request %lld", (long long)id);
  if (r->state != RVF_REQ_DONE || !r->m) return set_err(RVF_EBUSY, "request %lld has no result", (long long)id);
  if (F_dev) *F_dev = r->m->F.as<double>();
  if (A_dev) *A_dev = r->m->result_area;
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_request_result(rvf_server* sv, int64_t id, double* F_elem, double* A_elem, double* F_group,
                       double* A_group, double* row_sums) try {
  if (!sv) return set_err(RVF_EINVAL, "null server");
  rvf_mesh* m = nullptr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    Req* r = find(sv, id);
    if (!r) return set_err(RVF_EINVAL, "unknown request %lld", (long long)id);
    if (r->state != RVF_REQ_DONE || !r->m) return set_err(RVF_EBUSY, "request %lld has no result", (long long)id);
    m = r->m;
  }
  Session* s = sv->s;
  std::lock_guard<std::mutex> lk(s->mu);
  cudaSetDevice(s->device);
  const int64_t N = m->N;
  cudaError_t e = cudaSuccess;
  auto cp = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && dst && src && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream);
  };
  cp(F_elem, m->F.ptr, sizeof(double) * N * N);
  cp(A_elem, m->result_area, sizeof(double) * N);
  if (m->G > 0 && N > 0) {
    cp(F_group, m->Fgroup.ptr, sizeof(double) * m->G * m->G);
    cp(A_group, m->Agroup.ptr, sizeof(double) * m->G);
    cp(row_sums, m->rowsum.ptr, sizeof(double) * N);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e == cudaSuccess ? RVF_OK : cuda_err(e, "result copy");
} catch (...) {
  return exception_status();
}

int rvf_release(rvf_server* sv, int64_t id) try {
  if (!sv) return set_err(RVF_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  Req* r = find(sv, id);
  if (!r) return set_err(RVF_EINVAL, "unknown request %lld", (long long)id);
  if (r->state == RVF_REQ_QUEUED || r->state == RVF_REQ_RUNNING)
    return set_err(RVF_EBUSY, "request %lld is still in progress (cancel it first)", (long long)id);
  drop_device(sv, r);
  sv->reqs.erase(id);
  return RVF_OK;
} catch (...) {
  return exception_status();
}

int rvf_server_stats_get(rvf_server* sv, rvf_server_stats* st) try {
  if (!sv || !st) return set_err(RVF_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  *st = rvf_server_stats{};
  st->submitted = sv->submitted;
  st->completed = sv->completed;
  st->failed = sv->failed;
  st->canceled = sv->canceled;
  st->in_flight = (int64_t)(sv->queue.size() + sv->active.size());
  std::vector<double> l = sv->latencies;
  std::sort(l.begin(), l.end());
  if (!l.empty()) {
    auto pct = [&](double q) {
      const size_t k = (size_t)std::ceil(q * (double)l.size()) - 1;
      return l[std::min(k, l.size() - 1)];
    };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    double sum = 0;
    for (double v : l) sum += v;
    st->mean_ms = sum / (double)l.size();
  }
  st->wall_ms = sv->first_submit >= 0 ? sv->last_done - sv->first_submit : 0.0;
  st->pairs_done = sv->pairs_done;
  st->chunks = sv->chunks;
  st->graph_replays = sv->graph_replays;
  st->batched_requests = sv->batched;
  st->admitted_bytes_peak = sv->admitted_peak;
  st->ms_admit = sv->ms_admit;
  st->ms_quad_chunks = sv->ms_quad;
  st->ms_mc_chunks = sv->ms_mc;
  st->ms_free = sv->ms_free;
  st->ms_idle = sv->ms_idle;
  Session* s = sv->s;
  std::lock_guard<std::mutex> lk2(s->tune_mu);
  const size_t first = s->ftune_done.size() > 8 ? s->ftune_done.size() - 8 : 0;
  for (size_t n = first; n < s->ftune_done.size(); ++n) {
    const uint64_t key = s->ftune_done[n];
    const FastTune& f = s->ftune[key];
    rvf_tuned_shape& o = st->tuned[st->n_tuned++];
    o.mixed = (int32_t)(key & 1);
    o.dim3 = (int32_t)((key >> 1) & 1);
    o.occlusion = (int32_t)((key >> 2) & 1);
    o.size_class = (int32_t)((key >> 8) & 15);
    o.rule_points = (int32_t)(key >> 16);
    const auto g = s->grid_tune.find(key & 0xff);
    if (g != s->grid_tune.end() && g->second.done) {
      o.gen_blocks_per_sm = g->second.gen;
      o.trace_blocks_per_sm = g->second.trace;
    }
    o.fast_points = f.qb;
    o.fast_row_groups = f.groups;
    double best = f.score[0];
    for (int c = 1; c < kNFastCand; ++c) best = std::min(best, f.score[c]);
    o.fast_ms_per_gpp = best;
    o.fast_ms_per_gpp_default = f.score[0];
  }
  return RVF_OK;
} catch (...) {
  return exception_status();
}

}  // extern "C"
