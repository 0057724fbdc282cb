// rules_bvh.cpp -- quadrature rules and the exact BVH build (host side).
//
// Compiled with -ffp-contract=off: the rule constants and the BVH boxes must
// come out bit-for-bit as the reference computes them, because the device's
// ray decisions are required to match the reference ray by ray.
#include <algorithm>
#include <cmath>
#include <exception>
#include <thread>
#include <utility>

#include "rvf_host.h"

namespace rvf {
namespace {

const double kPi = 3.141592653589793;

// Julia Base.min / Base.max / isless for Float64 (NaN-propagating, -0.0 < 0.0).
inline double jmin(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return a - b;
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(a) ? a : b;
}
inline double jmax(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return a - b;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}
inline bool jisless(double a, double b) {
  if (std::isnan(a)) return false;
  if (std::isnan(b)) return true;
  if (a < b) return true;
  if (a == b && a == 0.0) return std::signbit(a) && !std::signbit(b);
  return false;
}

// Nodes and weights for n > 5 (the reference diagonalises the Jacobi matrix,
// src/Quadrature.jl:75-84, pinned to 1e-12 by test/runtests.jl:34-48):
// Newton's method on the Legendre three-term recurrence from the
// Tricomi-style initial guess cos(pi (k + 3/4) / (n + 1/2)).
void legendre(int n, double x, double* pn, double* dpn) {
  double p0 = 1.0, p1 = x;
  for (int m = 2; m <= n; ++m) {
    double p2 = ((2.0 * m - 1.0) * x * p1 - (m - 1.0) * p0) / m;
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *dpn = n * (x * p1 - p0) / (x * x - 1.0);
}
void gl_newton(int n, double* pts, double* wts) {
  for (int k = 0; k < n; ++k) {
    double x = std::cos(kPi * (k + 0.75) / (n + 0.5));
    double p, dp;
    for (int it = 0; it < 100; ++it) {
      legendre(n, x, &p, &dp);
      double dx = p / dp;
      x -= dx;
      if (std::fabs(dx) <= 1e-16 && it > 2) break;
    }
    legendre(n, x, &p, &dp);
    pts[n - 1 - k] = x;
    wts[n - 1 - k] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
}

}  // namespace

void gl1d(int n, std::vector<double>& p, std::vector<double>& w) {
  p.assign(n, 0.0);
  w.assign(n, 0.0);
  switch (n) {  // closed forms of src/Quadrature.jl:35-61, same operation order
    case 1:
      p[0] = 0.0; w[0] = 2.0;
      return;
    case 2:
      p[0] = -1.0 / std::sqrt(3.0); p[1] = 1.0 / std::sqrt(3.0);
      w[0] = 1.0; w[1] = 1.0;
      return;
    case 3: {
      double a = std::sqrt(3.0 / 5.0);
      p[0] = -a; p[1] = 0.0; p[2] = a;
      w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
      return;
    }
    case 4: {
      double a = std::sqrt((3.0 + 2.0 * std::sqrt(6.0 / 5.0)) / 7.0);
      double b = std::sqrt((3.0 - 2.0 * std::sqrt(6.0 / 5.0)) / 7.0);
      double wa = (18.0 - std::sqrt(30.0)) / 36.0, wb = (18.0 + std::sqrt(30.0)) / 36.0;
      p[0] = -a; p[1] = -b; p[2] = b; p[3] = a;
      w[0] = wa; w[1] = wb; w[2] = wb; w[3] = wa;
      return;
    }
    case 5: {
      double a = std::sqrt(5.0 + 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
      double b = std::sqrt(5.0 - 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
      double wa = (322.0 - 13.0 * std::sqrt(70.0)) / 900.0, wb = (322.0 + 13.0 * std::sqrt(70.0)) / 900.0;
      p[0] = -a; p[1] = -b; p[2] = 0.0; p[3] = b; p[4] = a;
      w[0] = wa; w[1] = wb; w[2] = 128.0 / 225.0; w[3] = wb; w[4] = wa;
      return;
    }
    default:
      gl_newton(n, p.data(), w.data());
  }
}

Rule gl2d(int n) {  // src/Quadrature.jl:96-109
  std::vector<double> p, w;
  gl1d(n, p, w);
  Rule r;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      r.xi.push_back(p[i]);
      r.eta.push_back(p[j]);
      r.w.push_back(w[i] * w[j]);
    }
  return r;
}

Rule tri_rule(int nquad) {  // src/GPUKernels.jl:414-439
  Rule r;
  if (nquad <= 1) {
    r.xi = {1.0 / 3.0}; r.eta = {1.0 / 3.0}; r.w = {0.5};
  } else if (nquad == 2) {
    r.xi = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
    r.eta = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
    r.w = {0.5 / 3.0, 0.5 / 3.0, 0.5 / 3.0};
  } else if (nquad == 3) {
    double a1 = 0.101286507323456, b1 = 1.0 - 2.0 * a1;
    double a2 = 0.470142064105115, b2 = 1.0 - 2.0 * a2;
    r.xi = {a1, b1, a1, a2, b2, a2, 1.0 / 3.0};
    r.eta = {a1, a1, b1, a2, a2, b2, 1.0 / 3.0};
    double w1 = 0.125939180544827 / 2.0, w2 = 0.132394440720100 / 2.0, w3 = 0.225 / 2.0;
    r.w = {w1, w1, w1, w2, w2, w2, w3};
  } else {
    double cen = 1.0 / 3.0;
    double a1 = 0.260345966079038, b1 = 1.0 - 2.0 * a1;
    double a2 = 0.065130102902216, b2 = 1.0 - 2.0 * a2;
    double a3 = 0.048690315425316, b3 = 0.312865496004875, c3 = (1.0 - a3) - b3;
    r.xi = {a1, b1, a1, a2, b2, a2, a3, b3, a3, c3, b3, c3, cen};
    r.eta = {a1, a1, b1, a2, a2, b2, b3, a3, c3, a3, c3, b3, cen};
    double wc = -0.149570044467670 / 2.0, wA = 0.175615257433204 / 2.0;
    double wB = 0.053347235608839 / 2.0, wC = 0.077113760890257 / 2.0;
    r.w = {wA, wA, wA, wB, wB, wB, wC, wC, wC, wC, wC, wC, wc};
  }
  return r;
}

Rule line_rule(int n) {
  std::vector<double> p, w;
  gl1d(n, p, w);
  Rule r;
  r.xi = p;
  r.eta.assign(n, 0.0);
  r.w = w;
  return r;
}

// ---------------------------------------------------------------------------
// BVH build: median split on the longest axis, stable sort by centroid,
// LEAF_MAX = 8, parent slot reserved before the children (src/BVH.jl:71-148).
//
// The tree is the reference's bit for bit; two things make it fast.  Each
// primitive's box and centroids are evaluated once, with the reference's
// arithmetic, instead of at every level.  And a subtree's node count depends
// on its primitive count only (the split is mid = (start + stop) / 2), so the
// pre-order slot of every node is known before its subtree is built: the two
// halves of a large node are built on different threads, each into its own
// slots and its own range of the index array.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kLeafMax = 8;
constexpr int64_t kParallelMin = 8192;  // primitives below which a subtree stays on one thread

int64_t subtree_nodes(int64_t n) {
  if (n <= kLeafMax) return 1;
  const int64_t l = (n - 1) / 2 + 1;  // mid - start + 1 for mid = (start + stop) / 2
  return 1 + subtree_nodes(l) + subtree_nodes(n - l);
}

struct Builder {
  const double* soup;
  int nv;
  HostBVH* out;
  std::vector<double> box;   // per primitive: lo x,y,z, hi x,y,z
  std::vector<double> cent;  // per primitive: centroid x,y,z
  double S(int c, int v, int64_t t) const { return soup[c + 3 * (v + (int64_t)nv * t)]; }
  void prepare(int64_t n) {
    box.resize((size_t)n * 6);
    cent.resize((size_t)n * 3);
    for (int64_t t = 0; t < n; ++t) {
      double lox = S(0, 0, t), hix = lox, loy = S(1, 0, t), hiy = loy, loz = S(2, 0, t), hiz = loz;
      for (int v = 1; v < nv; ++v) {
        double x = S(0, v, t); lox = jmin(lox, x); hix = jmax(hix, x);
        double y = S(1, v, t); loy = jmin(loy, y); hiy = jmax(hiy, y);
        double z = S(2, v, t); loz = jmin(loz, z); hiz = jmax(hiz, z);
      }
      double* b = &box[(size_t)t * 6];
      b[0] = lox; b[1] = loy; b[2] = loz; b[3] = hix; b[4] = hiy; b[5] = hiz;
      for (int axis = 0; axis < 3; ++axis) {
        double c = 0.0;
        for (int v = 0; v < nv; ++v) c += S(axis, v, t);
        cent[(size_t)t * 3 + axis] = c / (double)nv;
      }
    }
  }
  // Builds the subtree of tri_idx[start-1 .. stop-1] (1-based inclusive) with
  // its root at node `self` (1-based); `spawn` halves left may go to threads.
  void rec(int64_t start, int64_t stop, int64_t self, int spawn) {
    std::vector<int64_t>& idx = out->tri_idx;
    const double* b0 = &box[(size_t)(idx[start - 1] - 1) * 6];
    double lo[3] = {b0[0], b0[1], b0[2]}, hi[3] = {b0[3], b0[4], b0[5]};
    for (int64_t i = start + 1; i <= stop; ++i) {
      const double* b = &box[(size_t)(idx[i - 1] - 1) * 6];
      for (int c = 0; c < 3; ++c) { lo[c] = jmin(lo[c], b[c]); hi[c] = jmax(hi[c], b[3 + c]); }
    }
    HostBVH::Node& nd = out->nodes[self - 1];
    for (int c = 0; c < 3; ++c) { nd.lo[c] = lo[c]; nd.hi[c] = hi[c]; }
    const int64_t count = stop - start + 1;
    if (count <= kLeafMax) {
      nd.tri_start = start;
      nd.tri_count = count;
      return;
    }
    double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    int axis = 0;
    for (int c = 1; c < 3; ++c)
      if (jisless(ext[axis], ext[c])) axis = c;
    const int64_t mid = (start + stop) / 2;
    std::vector<std::pair<double, int64_t>> keyed;
    keyed.reserve(count);
    for (int64_t i = start; i <= stop; ++i) keyed.push_back({cent[(size_t)(idx[i - 1] - 1) * 3 + axis], idx[i - 1]});
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<double, int64_t>& a, const std::pair<double, int64_t>& b) {
                       return jisless(a.first, b.first);
                     });
    for (int64_t i = start; i <= stop; ++i) idx[i - 1] = keyed[i - start].second;
    std::vector<std::pair<double, int64_t>>().swap(keyed);
    const int64_t l = self + 1;
    const int64_t r = l + subtree_nodes(mid - start + 1);
    nd.left = l;
    nd.right = r;
    if (spawn > 0 && count >= kParallelMin) {
      std::exception_ptr err;  // an exception of the helper thread is rethrown here
      std::thread t([&, start, mid, l, spawn] {
        try {
          rec(start, mid, l, spawn - 1);
        } catch (...) {
          err = std::current_exception();
        }
      });
      try {
        rec(mid + 1, stop, r, spawn - 1);
      } catch (...) {
        t.join();
        throw;
      }
      t.join();
      if (err) std::rethrow_exception(err);
    } else {
      rec(start, mid, l, 0);
      rec(mid + 1, stop, r, 0);
    }
  }
  void miss(int64_t node, int64_t next) {  // src/GPUBVH.jl:69-82
    out->nodes[node - 1].miss = next;
    int64_t l = out->nodes[node - 1].left, r = out->nodes[node - 1].right;
    if (l != 0) {
      miss(l, r);
      miss(r, next);
    }
  }
};

}  // namespace

HostBVH build_bvh(const double* soup, int nv, int64_t n_prims) {
  HostBVH b;
  if (n_prims <= 0) return b;
  b.tri_idx.resize(n_prims);
  for (int64_t i = 0; i < n_prims; ++i) b.tri_idx[i] = i + 1;
  b.nodes.assign((size_t)subtree_nodes(n_prims), HostBVH::Node{});
  Builder bl{soup, nv, &b, {}, {}};
  bl.prepare(n_prims);
  const unsigned hc = std::thread::hardware_concurrency();
  int spawn = 0;  // levels that fork: 2^spawn threads at most
  while (spawn < 4 && (2u << spawn) <= std::max(1u, hc)) ++spawn;
  bl.rec(1, n_prims, 1, spawn);
  bl.miss(1, 0);
  return b;
}

}  // namespace rvf
