// abi.cpp -- the C ABI of librvf_b200 (include/rvf_b200.h).
//
// compute_view_factors_gpu (src/GPUAssembly.jl:32-105) restated as a
// host driver: upload (build_gpu_arrays, src/GPUKernels.jl:336-412), BVH
// (build_flat_bvh_from_mesh, src/GPUBVH.jl:146-174), pair kernel, F = raw/A,
// aggregation (src/Results.jl:56-82) and the copies back to the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <new>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rvf_b200.h"
#include "kernels.h"
#include "rvf_internal.h"

namespace rvf {

thread_local std::string g_last_error;

int set_err(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_err(cudaError_t e, const char* what) {
  return set_err(RVF_ECUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

int exception_status() noexcept {
  int code = RVF_EINTERNAL;
  try {
    try {
      throw;
    } catch (const std::bad_alloc&) {
      code = RVF_ENOMEM;
      set_err(code, "host memory allocation failed");
    } catch (const std::exception& e) {
      set_err(code, "internal error: %s", e.what());
    } catch (...) {
      set_err(code, "internal error");
    }
  } catch (...) {  // recording the message failed too
  }
  return code;
}

// ---------------------------------------------------------------------------
// device buffers with budget accounting
// ---------------------------------------------------------------------------
int DevBuf::alloc(Session* s, size_t n) {
  free_();
  if (n == 0) return RVF_OK;
  // test hook: this allocation fails (before the cache could serve it)
  if (s->fail_alloc_in > 0 && --s->fail_alloc_in == 0)
    return set_err(RVF_ENOMEM, "cudaMalloc(%zu) failed: injected allocation failure (fault_inject)", n);
  if (n < kSpareMin) n = kSpareMin;  // the smallest size class
  if (n >= kSpareMin) {
    // the smallest cached buffer that holds n with at most a quarter to spare
    std::lock_guard<std::mutex> lk(s->spare_mu);
    size_t best = s->spares.size();
    for (size_t k = 0; k < s->spares.size(); ++k) {
      const size_t b = s->spares[k].second;
      if (b >= n && b - n <= n / 4 && (best == s->spares.size() || b < s->spares[best].second)) best = k;
    }
    if (best < s->spares.size()) {
      ptr = s->spares[best].first;
      bytes = s->spares[best].second;
      owner = s;
      s->spares.erase(s->spares.begin() + (std::ptrdiff_t)best);
      return RVF_OK;  // already charged to the budget
    }
  }
  // Buffers come in size classes 2^(1/4) apart from 4 KiB (at most 19%
  // spare), so that a freed one serves the next request of about the same
  // size -- mesh after mesh of different element counts, as a serving stream
  // sends them -- instead of a cudaMalloc / cudaFree each time (gigabytes of
  // mapping work for an F; about a millisecond and a device synchronisation
  // for any buffer).
  if (n >= kSpareMin) {
    size_t c = kSpareMin;
    while (c < n) {
      const size_t next = (size_t)((double)c * 1.189207115002721);  // 2^(1/4)
      c = (next + 4095) & ~(size_t)4095;
    }
    if (s->used + c <= s->budget || s->used + n > s->budget) n = c;  // the class when it fits the budget
  }
  if (s->used + n > s->budget) release_spares(s, n);
  if (s->used + n > s->budget)
    return set_err(RVF_EBUDGET, "HBM budget exceeded: need %zu more bytes, %zu of %zu in use", n, s->used,
                   s->budget);
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release_spares(s);
    e = cudaMalloc(&ptr, n);
  }
  if (e != cudaSuccess) {
    ptr = nullptr;
    cudaGetLastError();
    return set_err(RVF_ENOMEM, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  owner = s;
  s->used += n;
  return RVF_OK;
}
void DevBuf::free_() {
  if (ptr) {
    if (owner && bytes >= kSpareMin) {
      std::lock_guard<std::mutex> lk(owner->spare_mu);
      owner->spares.emplace_back(ptr, bytes);  // stays charged to the budget
    } else {
      cudaFree(ptr);
      if (owner) owner->used -= bytes;
    }
  }
  ptr = nullptr;
  bytes = 0;
  owner = nullptr;
}

void release_spares(Session* s, size_t need) {
  std::lock_guard<std::mutex> lk(s->spare_mu);
  // the oldest first (the front of the list), until `need` more bytes fit
  size_t k = 0;
  for (; k < s->spares.size() && (need == 0 || s->used + need > s->budget); ++k) {
    cudaFree(s->spares[k].first);
    s->used -= s->spares[k].second;
  }
  s->spares.erase(s->spares.begin(), s->spares.begin() + (std::ptrdiff_t)k);
}

int upload(Session* s, DevBuf& b, const void* src, size_t n) {
  int rc = b.alloc(s, n);
  if (rc) return rc;
  if (n == 0) return RVF_OK;
  cudaError_t e = cudaMemcpyAsync(b.ptr, src, n, cudaMemcpyHostToDevice, s->stream);
  return e == cudaSuccess ? RVF_OK : cuda_err(e, "cudaMemcpyAsync H2D");
}

// ---------------------------------------------------------------------------
// mesh upload
// ---------------------------------------------------------------------------
static const int kFamNodes[6] = {8, 6, 4, 3, 3, 2};
#ifndef RVF_ORDER_RUN
#define RVF_ORDER_RUN 8
#endif
static const int64_t kOrderRun = RVF_ORDER_RUN;  // caller-consecutive elements kept together in the internal order

int mesh_upload(Session* s, const rvf_mesh_desc* d, rvf_mesh** out) {
  if (!d || !out) return set_err(RVF_EINVAL, "null argument");
  if (d->mesh_dim != 1 && d->mesh_dim != 2) return set_err(RVF_EINVAL, "mesh_dim must be 1 or 2, got %d", d->mesh_dim);
  if (d->n_elems < 0 || d->n_nodes < 0) return set_err(RVF_EINVAL, "negative sizes");
  if (d->n_elems > 0 && (!d->coords || !d->elem_family || !d->elem_node_idx || !d->elem_group))
    return set_err(RVF_EINVAL, "missing mesh arrays");
  auto m = std::make_unique<rvf_mesh>();
  m->s = s;
  m->dim = d->mesh_dim;
  m->N = d->n_elems;
  m->Nn = d->n_nodes;
  const int64_t N = m->N;
  // padded, 0-based node table (element-major)
  m->h_enodes.assign((size_t)N * 8, 0);
  m->h_fam.assign(d->elem_family, d->elem_family + N);
  m->h_group.assign(d->elem_group, d->elem_group + N);
  for (int64_t e = 0; e < N; ++e) {
    int f = d->elem_family[e];
    if (f < 0 || f > 5) return set_err(RVF_EINVAL, "element %lld: unknown family code %d", (long long)e + 1, f);
    if ((d->mesh_dim == 2) != (f <= 3))
      return set_err(RVF_EINVAL, "element %lld: family %d does not match mesh_dim %d", (long long)e + 1, f,
                     d->mesh_dim);
    int64_t col = d->elem_node_idx[e];
    if (col < 1 || col > d->n_family[f] || !d->nodes[f])
      return set_err(RVF_EINVAL, "element %lld: elem_node_idx %lld outside the family table", (long long)e + 1,
                     (long long)col);
    int k = kFamNodes[f];
    for (int a = 0; a < k; ++a) {
      int32_t nid = d->nodes[f][(col - 1) * k + a];
      if (nid < 1 || nid > d->n_nodes)
        return set_err(RVF_EINVAL, "element %lld: node id %d outside 1..%lld", (long long)e + 1, nid,
                       (long long)d->n_nodes);
      m->h_enodes[(size_t)e * 8 + a] = nid - 1;
    }
  }
  // groups: sorted tags (src/Results.jl:59) -> member lists in element order
  std::vector<int32_t> tags;
  if (d->n_groups > 0 && d->group_tags) tags.assign(d->group_tags, d->group_tags + d->n_groups);
  else {
    tags = m->h_group;
    std::sort(tags.begin(), tags.end());
    tags.erase(std::unique(tags.begin(), tags.end()), tags.end());
  }
  for (size_t k = 1; k < tags.size(); ++k)
    if (!(tags[k - 1] < tags[k])) return set_err(RVF_EINVAL, "group_tags must be sorted ascending and distinct");
  m->G = (int)tags.size();
  m->h_tags = tags;
  m->h_member_off.assign(m->G + 1, 0);
  std::vector<std::vector<int32_t>> mem(m->G);
  for (int64_t e = 0; e < N; ++e) {
    auto it = std::lower_bound(tags.begin(), tags.end(), m->h_group[e]);
    if (it != tags.end() && *it == m->h_group[e]) mem[it - tags.begin()].push_back((int32_t)e);
  }
  for (int g = 0; g < m->G; ++g) {
    m->h_member_off[g + 1] = m->h_member_off[g] + (int64_t)mem[g].size();
    m->h_members.insert(m->h_members.end(), mem[g].begin(), mem[g].end());
  }

  // Internal element order: runs of kOrderRun consecutive elements of the
  // caller, ordered along a Morton (Z-order) curve of the runs' centroids, so
  // that 32 consecutive internal elements form a compact patch (the shadow
  // rays of one warp leave or reach neighbouring points) while the caller's
  // columns of F that finish together stay in runs of kOrderRun (one copy
  // each when F is downloaded during the solve).  Results do not depend on
  // this order; they stay in the caller's (orig[internal] = original index).
  m->h_orig.resize(N);
  {
    std::vector<double> cx(N), cy(N), cz(N);
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t e = 0; e < N; ++e) {
      const int k = kFamNodes[m->h_fam[e]] == 8 ? 4 : kFamNodes[m->h_fam[e]] == 6 ? 3 : kFamNodes[m->h_fam[e]];
      double c[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < k; ++a)
        for (int q = 0; q < 3; ++q) c[q] += d->coords[3 * (int64_t)m->h_enodes[(size_t)e * 8 + a] + q];
      cx[e] = c[0] / k; cy[e] = c[1] / k; cz[e] = c[2] / k;
      const double cc[3] = {cx[e], cy[e], cz[e]};
      for (int q = 0; q < 3; ++q) { lo[q] = std::min(lo[q], cc[q]); hi[q] = std::max(hi[q], cc[q]); }
    }
    auto spread = [](uint64_t v) {  // 21 bits -> every third bit
      v &= 0x1fffff;
      v = (v | v << 32) & 0x1f00000000ffffULL;
      v = (v | v << 16) & 0x1f0000ff0000ffULL;
      v = (v | v << 8) & 0x100f00f00f00f00fULL;
      v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
      v = (v | v << 2) & 0x1249249249249249ULL;
      return v;
    };
    const int64_t n_runs = (N + kOrderRun - 1) / kOrderRun;
    std::vector<std::pair<uint64_t, int32_t>> key(n_runs);
    for (int64_t r = 0; r < n_runs; ++r) {
      const int64_t e0 = r * kOrderRun, e1 = std::min<int64_t>(N, e0 + kOrderRun);
      double cc[3] = {0.0, 0.0, 0.0};
      for (int64_t e = e0; e < e1; ++e) { cc[0] += cx[e]; cc[1] += cy[e]; cc[2] += cz[e]; }
      uint64_t q3[3];
      for (int q = 0; q < 3; ++q) {
        cc[q] /= (double)(e1 - e0);
        const double span = hi[q] - lo[q];
        const double f = span > 0.0 ? (cc[q] - lo[q]) / span : 0.0;
        q3[q] = (uint64_t)std::min(2097151.0, std::max(0.0, f * 2097151.0));
      }
      key[r] = {spread(q3[0]) | (spread(q3[1]) << 1) | (spread(q3[2]) << 2), (int32_t)r};
    }
    std::stable_sort(key.begin(), key.end(),
                     [](const std::pair<uint64_t, int32_t>& a, const std::pair<uint64_t, int32_t>& b) {
                       return a.first < b.first;
                     });
    int64_t at = 0;
    for (int64_t k = 0; k < n_runs; ++k) {
      const int64_t e0 = (int64_t)key[k].second * kOrderRun, e1 = std::min<int64_t>(N, e0 + kOrderRun);
      for (int64_t e = e0; e < e1; ++e) m->h_orig[at++] = (int32_t)e;
    }
  }
  std::vector<int32_t> p_enodes((size_t)N * 8), p_group(N);
  std::vector<int8_t> p_fam(N);
  for (int64_t e = 0; e < N; ++e) {
    const int32_t o = m->h_orig[e];
    for (int a = 0; a < 8; ++a) p_enodes[(size_t)e * 8 + a] = m->h_enodes[(size_t)o * 8 + a];
    p_fam[e] = m->h_fam[o];
    p_group[e] = m->h_group[o];
  }

  int rc;
  if ((rc = upload(s, m->coords, d->coords, sizeof(double) * 3 * d->n_nodes))) return rc;
  if ((rc = upload(s, m->enodes, p_enodes.data(), sizeof(int32_t) * 8 * N))) return rc;
  if ((rc = upload(s, m->fam, p_fam.data(), N))) return rc;
  if ((rc = upload(s, m->group, p_group.data(), sizeof(int32_t) * N))) return rc;
  if ((rc = upload(s, m->orig, m->h_orig.data(), sizeof(int32_t) * N))) return rc;
  {
    std::vector<int32_t> inv(N);
    for (int64_t e = 0; e < N; ++e) inv[m->h_orig[e]] = (int32_t)e;
    if ((rc = upload(s, m->inv, inv.data(), sizeof(int32_t) * N))) return rc;
  }
  if ((rc = upload(s, m->member_off, m->h_member_off.data(), sizeof(int64_t) * (m->G + 1)))) return rc;
  if ((rc = upload(s, m->members, m->h_members.data(), sizeof(int32_t) * m->h_members.size()))) return rc;

  {
    double mx = 0.0;
    for (int64_t k = 0; k < 3 * d->n_nodes; ++k) {
      if (!std::isfinite(d->coords[k])) return set_err(RVF_EINVAL, "node %lld has a non-finite coordinate", (long long)(k / 3 + 1));
      mx = std::max(mx, std::fabs(d->coords[k]));
    }
    m->extent = 1.0 + mx;
  }

  // obstruction BVH (exact tree of src/BVH.jl over the merged soup)
  if (d->n_obs > 0) {
    if (!d->obs_soup || !d->obs_group) return set_err(RVF_EINVAL, "obstruction soup arrays missing");
    const int nv = d->obs_nv;
    if ((d->mesh_dim == 2 && nv != 3) || (d->mesh_dim == 1 && nv != 2))
      return set_err(RVF_EINVAL, "obs_nv %d does not match mesh_dim %d", nv, d->mesh_dim);
    m->h_soup.assign(d->obs_soup, d->obs_soup + (size_t)3 * nv * d->n_obs);
    m->h_obs_group.assign(d->obs_group, d->obs_group + d->n_obs);
    for (double v : m->h_soup)
      if (!std::isfinite(v)) return set_err(RVF_EINVAL, "obstruction soup holds a non-finite coordinate");
    HostBVH b = build_bvh(m->h_soup.data(), nv, d->n_obs);
    const int M = (int)b.nodes.size();
    std::vector<NodeD> nodes(M);
    for (int k = 0; k < M; ++k) {
      const HostBVH::Node& h = b.nodes[k];
      NodeD& n = nodes[k];
      for (int c = 0; c < 3; ++c) { n.lo[c] = h.lo[c]; n.hi[c] = h.hi[c]; }
      if (h.left != 0 && h.left != k + 2) return set_err(RVF_EINVAL, "internal: BVH is not in pre-order");
      n.a = h.tri_count > 0 ? (int32_t)(h.tri_start - 1) : 0;
      n.b = (int32_t)h.tri_count;
      // the batched traversal deals at most 32 x 8 leaf tests out per round
      if (n.b > 8) return set_err(RVF_EINVAL, "internal: BVH leaf holds more than 8 primitives");
      n.miss = h.miss == 0 ? M : (int32_t)(h.miss - 1);
      n.pad = 0;
      // every walk of the tree moves forward: miss links and first children lie ahead
      if (n.miss <= k || n.miss > M || (n.b == 0 && k + 1 >= M))
        return set_err(RVF_EINVAL, "internal: BVH node %d has a link that does not point forward", k);
    }
    m->n_nodes = M;
    m->h_nodes = nodes;
    if ((rc = upload(s, m->nodes, nodes.data(), sizeof(NodeD) * M))) return rc;
    std::vector<int32_t> leaf_of((size_t)d->n_obs, -1);
    for (int k = 0; k < M; ++k)
      for (int u = 0; u < nodes[k].b; ++u) {
        const int64_t t = (int64_t)nodes[k].a + u;
        if (t < 0 || t >= d->n_obs || leaf_of[t] >= 0) return set_err(RVF_EINVAL, "internal: BVH leaves do not partition the primitives");
        leaf_of[t] = k;
      }
    for (int32_t v : leaf_of)
      if (v < 0) return set_err(RVF_EINVAL, "internal: a primitive lies in no BVH leaf");
    if ((rc = upload(s, m->leaf_of, leaf_of.data(), sizeof(int32_t) * leaf_of.size()))) return rc;
    // Start nodes of the pair-list walk: the deepest level of the tree with
    // at most 32 nodes (with the leaves above it), so that one round of 32
    // lanes replaces the walk's first levels.
    {
      std::vector<int32_t> cur{0}, next;
      for (;;) {
        next.clear();
        for (int32_t k : cur) {
          if (nodes[k].b > 0) next.push_back(k);
          else {
            if (nodes[k + 1].miss >= M) return set_err(RVF_EINVAL, "internal: BVH node %d has no right child", k);
            next.push_back(k + 1);
            next.push_back(nodes[k + 1].miss);
          }
        }
        if (next.size() > 32 || next == cur) break;
        cur = next;
      }
      m->n_frontier = (int)cur.size();
      if ((rc = upload(s, m->frontier, cur.data(), sizeof(int32_t) * cur.size()))) return rc;
    }
    // FP32 copy for the certified FP32 traversal (rounding is inside its error allowance)
    std::vector<NodeF> nodesf(M);
    for (int k = 0; k < M; ++k) {
      for (int c = 0; c < 3; ++c) {
        nodesf[k].lo[c] = (float)nodes[k].lo[c];
        nodesf[k].hi[c] = (float)nodes[k].hi[c];
      }
      if (nodes[k].b > 15 || nodes[k].a >= (1 << 26)) return set_err(RVF_EINVAL, "internal: leaf does not fit NodeF");
      nodesf[k].ab = (nodes[k].a << 4) | nodes[k].b;
      nodesf[k].miss = nodes[k].miss;
    }
    if ((rc = upload(s, m->nodesf, nodesf.data(), sizeof(NodeF) * M))) return rc;
    for (double v : m->h_soup) m->extent = std::max(m->extent, 1.0 + std::fabs(v));
    const int64_t T = d->n_obs;
    if (nv == 3) {
      std::vector<TriD> tref(T), tgeo(T);
      for (int64_t k = 0; k < T; ++k) {
        int64_t t = b.tri_idx[k] - 1;
        const double* sp = m->h_soup.data() + 9 * t;
        double rv[3][3], gv[3][3];
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            rv[a][c] = sp[a + 3 * c];  // bvh_tris[a, c, t]: the reference's read (src/GPUBVH.jl:243-245)
            gv[a][c] = sp[c + 3 * a];  // true vertex a
          }
        for (int pass = 0; pass < 2; ++pass) {
          double(*v)[3] = pass == 0 ? rv : gv;
          TriD& o = pass == 0 ? tref[k] : tgeo[k];
          for (int c = 0; c < 3; ++c) {
            o.v0[c] = v[0][c];
            o.e1[c] = v[1][c] - v[0][c];
            o.e2[c] = v[2][c] - v[0][c];
          }
          o.group = m->h_obs_group[t];
          o.pad = 0;
        }
      }
      if ((rc = upload(s, m->tris_ref, tref.data(), sizeof(TriD) * T))) return rc;
      if ((rc = upload(s, m->tris_geo, tgeo.data(), sizeof(TriD) * T))) return rc;
      // Pair-list data per triangle: the corners v0, v0 + e1, v0 + e2 in FP32,
      // the group, and the margin by which rounding can move a hit of the
      // reference's Moller-Trumbore test, 2 (2^-53 / 1e-10) (65 S Lx^2 + 40 Lx^3)
      // with Lx the longest edge and S = 2 sqrt(3) extent >= |o - v0|, t_max, Lx
      // (rounded up).  sat_em: the separating-axis test's FP32 allowance.
      const double S = 2.0 * std::sqrt(3.0) * m->extent;
      m->sat_em = (float)std::ldexp(S, -16);
      for (int pass = 0; pass < 2; ++pass) {
        const std::vector<TriD>& src = pass == 0 ? tref : tgeo;
        std::vector<float> sat((size_t)T * 12);
        for (int64_t k = 0; k < T; ++k) {
          const TriD& t = src[k];
          double l2 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
          for (int c = 0; c < 3; ++c) {
            q1 += t.e1[c] * t.e1[c];
            q2 += t.e2[c] * t.e2[c];
            q3 += (t.e2[c] - t.e1[c]) * (t.e2[c] - t.e1[c]);
          }
          l2 = std::max(q1, std::max(q2, q3)) * (1.0 + 1e-9);
          const double lx = std::min(std::sqrt(l2), S);
          const double mt = 2.0 * 1.111e-6 * (65.0 * S * l2 + 40.0 * l2 * lx);
          float* o = sat.data() + 12 * k;
          for (int c = 0; c < 3; ++c) {
            o[c] = (float)t.v0[c];
            o[4 + c] = (float)(t.v0[c] + t.e1[c]);
            o[8 + c] = (float)(t.v0[c] + t.e2[c]);
          }
          o[3] = std::nextafter((float)mt, INFINITY);
          std::memcpy(&o[7], &t.group, 4);
          o[11] = 0.f;
        }
        if ((rc = upload(s, pass == 0 ? m->sat_ref : m->sat_geo, sat.data(), sizeof(float) * sat.size()))) return rc;
      }
      for (int pass = 0; pass < 2; ++pass) {
        const std::vector<TriD>& src = pass == 0 ? tref : tgeo;
        std::vector<TriF> tf(T);
        for (int64_t k = 0; k < T; ++k) {
          double n1 = 0.0, n2 = 0.0;
          for (int c = 0; c < 3; ++c) {
            tf[k].v0[c] = (float)src[k].v0[c];
            tf[k].e1[c] = (float)src[k].e1[c];
            tf[k].e2[c] = (float)src[k].e2[c];
            n1 += src[k].e1[c] * src[k].e1[c];
            n2 += src[k].e2[c] * src[k].e2[c];
          }
          // |e1|, |e2| rounded up, kept as float bits for the error bounds
          float f1 = std::nextafter((float)std::sqrt(n1), INFINITY), f2 = std::nextafter((float)std::sqrt(n2), INFINITY);
          std::memcpy(&tf[k].pad0, &f1, 4);
          std::memcpy(&tf[k].pad1, &f2, 4);
          tf[k].group = src[k].group;
        }
        if ((rc = upload(s, pass == 0 ? m->trisf_ref : m->trisf_geo, tf.data(), sizeof(TriF) * T))) return rc;
      }
    } else {
      std::vector<SegD> segs(T);
      for (int64_t k = 0; k < T; ++k) {
        int64_t t = b.tri_idx[k] - 1;
        const double* sp = m->h_soup.data() + 6 * t;
        segs[k] = SegD{sp[0], sp[1], sp[3], sp[4], m->h_obs_group[t], 0, 0, 0};
      }
      if ((rc = upload(s, m->segs, segs.data(), sizeof(SegD) * T))) return rc;
    }
    m->n_obs = T;
  }
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_err(e, "mesh upload");
  *out = m.release();
  return RVF_OK;
}

// ---------------------------------------------------------------------------
// quadrature tables for one nquad
// ---------------------------------------------------------------------------
int ensure_tables(Session* s, rvf_mesh* m, int nquad, Tables** out) {
  auto it = m->tables.find(nquad);
  if (it != m->tables.end()) { *out = it->second.get(); return RVF_OK; }
  Rule q = gl2d(nquad), t = tri_rule(nquad), l = line_rule(nquad);
  bool has_q = false, has_t = false, has_l = false;
  for (int8_t f : m->h_fam) {
    if (f == 0 || f == 2) has_q = true;
    else if (f == 1 || f == 3) has_t = true;
    else has_l = true;
  }
  int pmax = std::max({has_q ? q.size() : 0, has_t ? t.size() : 0, has_l ? l.size() : 0, 1});
  if (pmax > kMaxPts)
    return set_err(RVF_EUNSUPPORTED, "nquad=%d gives %d points per element; at most %d are supported", nquad, pmax,
                   kMaxPts);
  auto T = std::make_unique<Tables>();
  T->nquad = nquad;
  T->pmax = pmax;
  const int64_t N = m->N;
  const int64_t nT = (N + kTile - 1) / kTile;
  int rc;
  std::vector<double> rules;
  auto push = [&](const std::vector<double>& v) { rules.insert(rules.end(), v.begin(), v.end()); };
  push(q.xi); push(q.eta); push(q.w); push(t.xi); push(t.eta); push(t.w); push(l.xi); push(l.w);
  if ((rc = upload(s, T->rules, rules.data(), sizeof(double) * rules.size()))) return rc;
  if ((rc = T->tab.alloc(s, sizeof(double) * nT * kComp * pmax * kTile))) return rc;
  if ((rc = T->area.alloc(s, sizeof(double) * std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->area_orig.alloc(s, sizeof(double) * std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->np.alloc(s, std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->flat.alloc(s, std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->nrm.alloc(s, sizeof(double) * 3 * std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->cen.alloc(s, sizeof(double) * 3 * std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->diam.alloc(s, sizeof(double) * std::max<int64_t>(N, 1)))) return rc;
  if ((rc = T->rad.alloc(s, sizeof(double) * std::max<int64_t>(N, 1)))) return rc;
  cudaMemsetAsync(T->tab.ptr, 0, T->tab.bytes, s->stream);
  cudaMemsetAsync(s->err.ptr, 0, sizeof(int), s->stream);
  PrepArgs a{};
  a.N = N;
  a.pmax = pmax;
  a.coords = (const double*)m->coords.ptr;
  a.enodes = (const int32_t*)m->enodes.ptr;
  a.fam = (const int8_t*)m->fam.ptr;
  const double* r = (const double*)T->rules.ptr;
  a.qx = r; r += q.size(); a.qe = r; r += q.size(); a.qw = r; r += q.size();
  a.tx = r; r += t.size(); a.te = r; r += t.size(); a.tw = r; r += t.size();
  a.lx = r; r += l.size(); a.lw = r;
  a.nquadpts = q.size(); a.ntripts = t.size(); a.nline = l.size();
  a.tab = (double*)T->tab.ptr;
  a.area = (double*)T->area.ptr;
  a.orig = m->orig.as<int32_t>();
  a.area_orig = T->area_orig.as<double>();
  a.np = (int8_t*)T->np.ptr;
  a.flat = (uint8_t*)T->flat.ptr;
  a.nrm = (double*)T->nrm.ptr;
  a.cen = (double*)T->cen.ptr;
  a.diam = (double*)T->diam.ptr;
  a.rad = (double*)T->rad.ptr;
  a.err = (int*)s->err.ptr;
  cudaError_t e = launch_prep(a, s->stream);
  if (e != cudaSuccess) return cuda_err(e, "prep kernel launch");
  int herr = 0;
  e = cudaMemcpyAsync(&herr, s->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_err(e, "prep kernel");
  if (herr & kErrBadInput)
    return set_err(RVF_EINVAL, "mesh holds a degenerate element (zero or non-finite area element at a quadrature point)");
  if (N == 1) {  // no pair writes area_out
    cudaMemsetAsync(T->area.ptr, 0, sizeof(double), s->stream);
    cudaMemsetAsync(T->area_orig.ptr, 0, sizeof(double), s->stream);
  }
  *out = T.get();
  m->tables[nquad] = std::move(T);
  return RVF_OK;
}

}  // namespace rvf
