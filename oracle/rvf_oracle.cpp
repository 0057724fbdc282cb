// rvf_oracle.cpp -- CPU restatement of RadiativeViewFactor.jl (v0.5.0) for the
// element-pair view-factor assembly path.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker / the timed CPU reference.  The
// product (radiativeviewfactor.jl_b200/) never links or calls it.
//
// Every function cites the reference file:line it restates.  Expressions keep
// the reference's evaluation order (Julia evaluates a+b+c as (a+b)+c and
// a*b*c as (a*b)*c; x^2 and x^3 with literal exponents are x*x and x*x*x);
// the file is compiled with -ffp-contract=off so no multiply-add is fused.
//
// Parity: see rvf_oracle.h.  The Monte Carlo, flat-BVH and Duffy parts are
// "parity unpinned" at the reference level (no vectors in the reference tests).
//
// 2-D Monte Carlo extension (the reference GPU path rejects curve meshes,
// src/Assembly.jl:83-86): per stratum (si outer, sj inner) four draws u1..u4
// are taken as in src/GPUMCKernels.jl:181-190; element i is sampled at
// xi = 2*((si+u1)/s) - 1, element j at xi = 2*((sj+u3)/s) - 1 (u2, u4 drawn
// and discarded); remainder samples use xi = 2*u1-1 and 2*u3-1; the reference
// measure of a line is 2 (src/MCKernel.jl:278-281); the kernel is
// cos*cos/(2r) and occlusion is the 2-D segment test (src/BVH.jl:265-276).
#include "rvf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double PI = 3.141592653589793;  // Float64(pi)

// ---------------------------------------------------------------------------
// Julia semantics helpers
// ---------------------------------------------------------------------------
// Base.min / Base.max for Float64: NaN-propagating, -0.0 < 0.0.
inline double jmin(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return a - b;  // a NaN
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
// Base.isless for Float64 (NaN last, -0.0 < 0.0).
inline bool jisless(double a, double b) {
  if (std::isnan(a)) return false;
  if (std::isnan(b)) return true;
  if (a < b) return true;
  if (a == b && a == 0.0) return std::signbit(a) && !std::signbit(b);
  return false;
}

inline double dot3(const double* a, const double* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

// ---------------------------------------------------------------------------
// Quadrature (src/Quadrature.jl:35-109)
// ---------------------------------------------------------------------------
// Golub-Welsch replacement for n > 5: Newton iteration on the Legendre
// three-term recurrence (nodes agree with the eigen-decomposition of the
// Jacobi matrix to ~1e-16; the reference pins n > 5 only to 1e-12,
// test/runtests.jl:34-48).
void gl_newton(int n, double* pts, double* wts) {
  for (int k = 0; k < n; ++k) {
    double x = std::cos(PI * (k + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int m = 2; m <= n; ++m) {
        double p2 = ((2.0 * m - 1.0) * x * p1 - (m - 1.0) * p0) / m;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (x * p1 - p0) / (x * x - 1.0);
      double dx = p1 / dp;
      x -= dx;
      if (std::fabs(dx) <= 1e-16) {
        if (it > 2) break;
      }
    }
    {
      double p0 = 1.0, p1 = x;
      for (int m = 2; m <= n; ++m) {
        double p2 = ((2.0 * m - 1.0) * x * p1 - (m - 1.0) * p0) / m;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (x * p1 - p0) / (x * x - 1.0);
    }
    pts[n - 1 - k] = x;  // ascending order
    wts[n - 1 - k] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
}

void gl1d(int n, std::vector<double>& p, std::vector<double>& w) {
  p.assign(n, 0.0);
  w.assign(n, 0.0);
  switch (n) {
    case 1:
      p[0] = 0.0; w[0] = 2.0;
      return;
    case 2: {
      double a = 1.0 / std::sqrt(3.0);
      p[0] = -1.0 / std::sqrt(3.0); p[1] = a;
      w[0] = 1.0; w[1] = 1.0;
      return;
    }
    case 3: {
      double a = std::sqrt(3.0 / 5.0);
      p[0] = -a; p[1] = 0.0; p[2] = a;
      w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
      return;
    }
    case 4: {
      double a = std::sqrt((3.0 + 2.0 * std::sqrt(6.0 / 5.0)) / 7.0);
      double b = std::sqrt((3.0 - 2.0 * std::sqrt(6.0 / 5.0)) / 7.0);
      double wa = (18.0 - std::sqrt(30.0)) / 36.0;
      double wb = (18.0 + std::sqrt(30.0)) / 36.0;
      p[0] = -a; p[1] = -b; p[2] = b; p[3] = a;
      w[0] = wa; w[1] = wb; w[2] = wb; w[3] = wa;
      return;
    }
    case 5: {
      double a = std::sqrt(5.0 + 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
      double b = std::sqrt(5.0 - 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
      double wa = (322.0 - 13.0 * std::sqrt(70.0)) / 900.0;
      double wb = (322.0 + 13.0 * std::sqrt(70.0)) / 900.0;
      double wc = 128.0 / 225.0;
      p[0] = -a; p[1] = -b; p[2] = 0.0; p[3] = b; p[4] = a;
      w[0] = wa; w[1] = wb; w[2] = wc; w[3] = wb; w[4] = wa;
      return;
    }
    default:
      gl_newton(n, p.data(), w.data());
  }
}

// tensor rule, xi index fastest (src/Quadrature.jl:96-109)
void gl2d(int n, std::vector<double>& xi, std::vector<double>& eta, std::vector<double>& w) {
  std::vector<double> p, w1;
  gl1d(n, p, w1);
  xi.resize(n * n); eta.resize(n * n); w.resize(n * n);
  int k = 0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      xi[k] = p[i]; eta[k] = p[j]; w[k] = w1[i] * w1[j];
      ++k;
    }
}

// Dunavant rules (src/ViewFactorKernel.jl:42-71 == src/GPUKernels.jl:414-439)
void tri_rule(int nquad, std::vector<double>& xi, std::vector<double>& eta, std::vector<double>& w) {
  if (nquad <= 1) {
    xi = {1.0 / 3.0}; eta = {1.0 / 3.0}; w = {0.5};
  } else if (nquad == 2) {
    xi = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
    eta = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
    w = {0.5 / 3.0, 0.5 / 3.0, 0.5 / 3.0};
  } else if (nquad == 3) {
    double a1 = 0.101286507323456, b1 = 1.0 - 2.0 * a1;
    double a2 = 0.470142064105115, b2 = 1.0 - 2.0 * a2;
    xi = {a1, b1, a1, a2, b2, a2, 1.0 / 3.0};
    eta = {a1, a1, b1, a2, a2, b2, 1.0 / 3.0};
    double w1 = 0.125939180544827 / 2.0, w2 = 0.132394440720100 / 2.0, w3 = 0.225 / 2.0;
    w = {w1, w1, w1, w2, w2, w2, w3};
  } else {
    double cen = 1.0 / 3.0;
    double a1 = 0.260345966079038, b1 = 1.0 - 2.0 * a1;
    double a2 = 0.065130102902216, b2 = 1.0 - 2.0 * a2;
    double a3 = 0.048690315425316, b3 = 0.312865496004875, c3 = (1.0 - a3) - b3;
    xi = {a1, b1, a1, a2, b2, a2, a3, b3, a3, c3, b3, c3, cen};
    eta = {a1, a1, b1, a2, a2, b2, b3, a3, c3, a3, c3, b3, cen};
    double wc = -0.149570044467670 / 2.0, wA = 0.175615257433204 / 2.0;
    double wB = 0.053347235608839 / 2.0, wC = 0.077113760890257 / 2.0;
    w = {wA, wA, wA, wB, wB, wB, wC, wC, wC, wC, wC, wC, wc};
  }
}

// ---------------------------------------------------------------------------
// Shape functions (src/GPUKernels.jl:51-176, src/Geometry.jl)
// ---------------------------------------------------------------------------
void quad8_shape(double x, double e, double* N, double* dx, double* de) {
  N[0] = ((0.25 * (1 - x)) * (1 - e)) * (((-x) - e) - 1);
  N[1] = ((0.25 * (1 + x)) * (1 - e)) * ((x - e) - 1);
  N[2] = ((0.25 * (1 + x)) * (1 + e)) * ((x + e) - 1);
  N[3] = ((0.25 * (1 - x)) * (1 + e)) * (((-x) + e) - 1);
  N[4] = (0.5 * (1 - x * x)) * (1 - e);
  N[5] = (0.5 * (1 + x)) * (1 - e * e);
  N[6] = (0.5 * (1 - x * x)) * (1 + e);
  N[7] = (0.5 * (1 - x)) * (1 - e * e);
  dx[0] = (0.25 * (1 - e)) * (2 * x + e);
  dx[1] = (0.25 * (1 - e)) * (2 * x - e);
  dx[2] = (0.25 * (1 + e)) * (2 * x + e);
  dx[3] = (0.25 * (1 + e)) * (2 * x - e);
  dx[4] = (-x) * (1 - e);
  dx[5] = 0.5 * (1 - e * e);
  dx[6] = (-x) * (1 + e);
  dx[7] = (-0.5) * (1 - e * e);
  de[0] = (0.25 * (1 - x)) * (x + 2 * e);
  de[1] = (0.25 * (1 + x)) * ((-x) + 2 * e);
  de[2] = (0.25 * (1 + x)) * (x + 2 * e);
  de[3] = (0.25 * (1 - x)) * ((-x) + 2 * e);
  de[4] = (-0.5) * (1 - x * x);
  de[5] = (-(1 + x)) * e;
  de[6] = 0.5 * (1 - x * x);
  de[7] = (-(1 - x)) * e;
}
void tri6_shape(double x, double e, double* N, double* dx, double* de) {
  double L1 = (1 - x) - e, L2 = x, L3 = e;
  N[0] = L1 * (2 * L1 - 1); N[1] = L2 * (2 * L2 - 1); N[2] = L3 * (2 * L3 - 1);
  N[3] = (4 * L1) * L2; N[4] = (4 * L2) * L3; N[5] = (4 * L1) * L3;
  dx[0] = (4 * L1 - 1) * (-1.0); dx[1] = 4 * L2 - 1; dx[2] = 0.0;
  dx[3] = 4 * (L2 * (-1.0) + L1); dx[4] = 4 * L3; dx[5] = (4 * L3) * (-1.0);
  de[0] = (4 * L1 - 1) * (-1.0); de[1] = 0.0; de[2] = 4 * L3 - 1;
  de[3] = (4 * L2) * (-1.0); de[4] = 4 * L2; de[5] = 4 * (L3 * (-1.0) + L1);
}
void quad4_shape(double x, double e, double* N, double* dx, double* de) {
  N[0] = (0.25 * (1 - x)) * (1 - e); N[1] = (0.25 * (1 + x)) * (1 - e);
  N[2] = (0.25 * (1 + x)) * (1 + e); N[3] = (0.25 * (1 - x)) * (1 + e);
  dx[0] = (-0.25) * (1 - e); dx[1] = 0.25 * (1 - e); dx[2] = 0.25 * (1 + e); dx[3] = (-0.25) * (1 + e);
  de[0] = (-0.25) * (1 - x); de[1] = (-0.25) * (1 + x); de[2] = 0.25 * (1 + x); de[3] = 0.25 * (1 - x);
}
void tri3_shape(double x, double e, double* N, double* dx, double* de) {
  N[0] = (1 - x) - e; N[1] = x; N[2] = e;
  dx[0] = -1.0; dx[1] = 1.0; dx[2] = 0.0;
  de[0] = -1.0; de[1] = 0.0; de[2] = 1.0;
}
// src/Geometry.jl:247-257
void line3_shape(double x, double* N, double* dN) {
  N[0] = ((-0.5) * x) * (1.0 - x);
  N[1] = (0.5 * x) * (1.0 + x);
  N[2] = 1.0 - x * x;
  dN[0] = -0.5 + x; dN[1] = 0.5 + x; dN[2] = -2.0 * x;
}
// src/Geometry.jl:305-307
void line2_shape(double x, double* N, double* dN) {
  N[0] = 0.5 * (1.0 - x); N[1] = 0.5 * (1.0 + x);
  dN[0] = -0.5; dN[1] = 0.5;
}

int fam_nodes(int f) {
  switch (f) {
    case 0: return 8;
    case 1: return 6;
    case 2: return 4;
    case 3: return 3;
    case 4: return 3;
    case 5: return 2;
  }
  return 0;
}
inline bool is_quad_fam(int f) { return f == 0 || f == 2; }
inline bool is_line_fam(int f) { return f == 4 || f == 5; }

// x, n = c/|c|, dA = |c| (src/GPUKernels.jl:95-176; src/Geometry.jl:83-172)
void eval_surface(const orc_mesh* m, int64_t e, double xi, double eta, double* x, double* n, double* dA) {
  int f = m->family[e];
  double N[8], dX[8], dE[8];
  int nn = fam_nodes(f);
  switch (f) {
    case 0: quad8_shape(xi, eta, N, dX, dE); break;
    case 1: tri6_shape(xi, eta, N, dX, dE); break;
    case 2: quad4_shape(xi, eta, N, dX, dE); break;
    default: tri3_shape(xi, eta, N, dX, dE); break;
  }
  double px[3] = {0.0, 0.0, 0.0}, a[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
  const int32_t* en = m->elem_nodes + 8 * e;
  for (int k = 0; k < nn; ++k) {
    const double* xa = m->coords + 3 * (int64_t)(en[k] - 1);
    for (int c = 0; c < 3; ++c) {
      px[c] = px[c] + N[k] * xa[c];
      a[c] = a[c] + dX[k] * xa[c];
      b[c] = b[c] + dE[k] * xa[c];
    }
  }
  double cx = a[1] * b[2] - a[2] * b[1];
  double cy = a[2] * b[0] - a[0] * b[2];
  double cz = a[0] * b[1] - a[1] * b[0];
  double d = std::sqrt((cx * cx + cy * cy) + cz * cz);
  x[0] = px[0]; x[1] = px[1]; x[2] = px[2];
  n[0] = cx / d; n[1] = cy / d; n[2] = cz / d;
  *dA = d;
}

// src/Geometry.jl:264-278 / 313-334
void eval_line(const orc_mesh* m, int64_t e, double xi, double* x, double* n, double* dL) {
  int f = m->family[e];
  double N[3], dN[3];
  int nn = (f == 4) ? 3 : 2;
  if (f == 4) line3_shape(xi, N, dN); else line2_shape(xi, N, dN);
  double px[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
  const int32_t* en = m->elem_nodes + 8 * e;
  for (int k = 0; k < nn; ++k) {
    const double* xa = m->coords + 3 * (int64_t)(en[k] - 1);
    for (int c = 0; c < 3; ++c) {
      px[c] = px[c] + N[k] * xa[c];
      t[c] = t[c] + dN[k] * xa[c];
    }
  }
  double L = std::sqrt((t[0] * t[0] + t[1] * t[1]) + t[2] * t[2]);
  double tx = t[0] / L, ty = t[1] / L;
  x[0] = px[0]; x[1] = px[1]; x[2] = px[2];
  n[0] = -ty; n[1] = tx; n[2] = 0.0;
  *dL = L;
}

// src/ViewFactorKernel.jl:155-166 == src/GPUKernels.jl:204-215
double vf_kernel(const double* xi, const double* ni, const double* xj, const double* nj) {
  double r[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
  double r2 = dot3(r, r);
  if (r2 < 1e-30) return 0.0;
  double rl = std::sqrt(r2);
  double h[3] = {r[0] / rl, r[1] / rl, r[2] / rl};
  double mh[3] = {-h[0], -h[1], -h[2]};
  double ci = dot3(ni, h);
  double cj = dot3(nj, mh);
  if (ci <= 0.0 || cj <= 0.0) return 0.0;
  return (ci * cj) / (PI * r2);
}
// src/ViewFactorKernel.jl:169-180
double vf_kernel_2d(const double* xi, const double* ni, const double* xj, const double* nj) {
  double r[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
  double r2 = dot3(r, r);
  if (r2 < 1e-30) return 0.0;
  double rl = std::sqrt(r2);
  double h[3] = {r[0] / rl, r[1] / rl, r[2] / rl};
  double mh[3] = {-h[0], -h[1], -h[2]};
  double ci = dot3(ni, h);
  double cj = dot3(nj, mh);
  if (ci <= 0.0 || cj <= 0.0) return 0.0;
  return (ci * cj) / (2.0 * rl);
}

// Per-element quadrature points: x, n, dA, w (what _sample / _quad_points give).
struct Pts {
  int np = 0;
  double x[256][3], n[256][3], dA[256], w[256];  // up to nquad = 16 (256 points)
  const double* X(int p) const { return x[p]; }
  const double* Nn(int p) const { return n[p]; }
  double W(int p) const { return w[p]; }
  double DA(int p) const { return dA[p]; }
};
// The same points of one element inside compact per-mesh arrays
// (x, n: 3 per point; w, dA: 1 per point).
struct PtsView {
  int np = 0;
  const double *x = nullptr, *n = nullptr, *w = nullptr, *dA = nullptr;
  const double* X(int p) const { return x + 3 * p; }
  const double* Nn(int p) const { return n + 3 * p; }
  double W(int p) const { return w[p]; }
  double DA(int p) const { return dA[p]; }
};
struct Rules {
  std::vector<double> qx, qe, qw, tx, te, tw, lx, lw;
};
Rules make_rules(int nquad) {
  Rules r;
  gl2d(nquad, r.qx, r.qe, r.qw);
  tri_rule(nquad, r.tx, r.te, r.tw);
  gl1d(nquad, r.lx, r.lw);
  return r;
}
void element_points(const orc_mesh* m, int64_t e, const Rules& R, Pts& P) {
  int f = m->family[e];
  if (R.qw.size() > 256) { P.np = 0; return; }  // nquad > 16 is outside the oracle's range
  if (is_line_fam(f)) {
    P.np = (int)R.lx.size();
    for (int p = 0; p < P.np; ++p) {
      eval_line(m, e, R.lx[p], P.x[p], P.n[p], &P.dA[p]);
      P.w[p] = R.lw[p];
    }
  } else if (is_quad_fam(f)) {
    P.np = (int)R.qw.size();
    for (int p = 0; p < P.np; ++p) {
      eval_surface(m, e, R.qx[p], R.qe[p], P.x[p], P.n[p], &P.dA[p]);
      P.w[p] = R.qw[p];
    }
  } else {
    P.np = (int)R.tw.size();
    for (int p = 0; p < P.np; ++p) {
      eval_surface(m, e, R.tx[p], R.te[p], P.x[p], P.n[p], &P.dA[p]);
      P.w[p] = R.tw[p];
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// BVH (src/BVH.jl:26-148, src/GPUBVH.jl:69-134)
// ---------------------------------------------------------------------------
struct orc_bvh {
  const double* soup = nullptr;
  int32_t nv = 3;
  int64_t T = 0;
  struct Node {
    double lo[3], hi[3];
    int64_t left, right, tri_start, tri_count, miss;  // 1-based node / tri_idx indices
  };
  std::vector<Node> nodes;      // pre-order (parent slot reserved before children)
  std::vector<int64_t> tri_idx; // 1-based triangle ids
};

namespace {

inline double S(const orc_bvh* b, int c, int v, int64_t t) { return b->soup[c + 3 * (v + (int64_t)b->nv * t)]; }

void prim_aabb(const orc_bvh* b, int64_t t, double* lo, double* hi) {
  double lox = S(b, 0, 0, t), hix = lox;
  double loy = S(b, 1, 0, t), hiy = loy;
  double loz = S(b, 2, 0, t), hiz = loz;
  for (int v = 1; v < b->nv; ++v) {
    double x = S(b, 0, v, t); lox = jmin(lox, x); hix = jmax(hix, x);
    double y = S(b, 1, v, t); loy = jmin(loy, y); hiy = jmax(hiy, y);
    double z = S(b, 2, v, t); loz = jmin(loz, z); hiz = jmax(hiz, z);
  }
  lo[0] = lox; lo[1] = loy; lo[2] = loz;
  hi[0] = hix; hi[1] = hiy; hi[2] = hiz;
}
double centroid(const orc_bvh* b, int64_t t, int axis) {
  double c = 0.0;
  for (int v = 0; v < b->nv; ++v) c += S(b, axis, v, t);
  return c / (double)b->nv;
}

int64_t build_rec(orc_bvh* b, int64_t start, int64_t stop) {  // 1-based inclusive
  double lo[3], hi[3];
  prim_aabb(b, b->tri_idx[start - 1] - 1, lo, hi);
  for (int64_t i = start + 1; i <= stop; ++i) {
    double l2[3], h2[3];
    prim_aabb(b, b->tri_idx[i - 1] - 1, l2, h2);
    for (int c = 0; c < 3; ++c) { lo[c] = jmin(lo[c], l2[c]); hi[c] = jmax(hi[c], h2[c]); }
  }
  int64_t count = stop - start + 1;
  orc_bvh::Node nd;
  for (int c = 0; c < 3; ++c) { nd.lo[c] = lo[c]; nd.hi[c] = hi[c]; }
  nd.miss = 0;
  if (count <= 8) {  // LEAF_MAX, src/BVH.jl:61
    nd.left = 0; nd.right = 0; nd.tri_start = start; nd.tri_count = count;
    b->nodes.push_back(nd);
    return (int64_t)b->nodes.size();
  }
  double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  int axis = 0;  // argmax, first maximum wins
  for (int c = 1; c < 3; ++c)
    if (jisless(ext[axis], ext[c])) axis = c;
  int64_t mid = (start + stop) / 2;
  // stable sort of tri_idx[start:stop] by centroid[axis] (Julia >= 1.9 default sort is stable)
  std::vector<std::pair<double, int64_t>> keyed;
  keyed.reserve(count);
  for (int64_t i = start; i <= stop; ++i) {
    int64_t t = b->tri_idx[i - 1];
    keyed.push_back({centroid(b, t - 1, axis), t});
  }
  std::stable_sort(keyed.begin(), keyed.end(),
                   [](const std::pair<double, int64_t>& A, const std::pair<double, int64_t>& B) {
                     return jisless(A.first, B.first);
                   });
  for (int64_t i = start; i <= stop; ++i) b->tri_idx[i - 1] = keyed[i - start].second;
  nd.left = 0; nd.right = 0; nd.tri_start = 0; nd.tri_count = 0;
  b->nodes.push_back(nd);
  int64_t node_idx = (int64_t)b->nodes.size();
  int64_t lc = build_rec(b, start, mid);
  int64_t rc = build_rec(b, mid + 1, stop);
  b->nodes[node_idx - 1].left = lc;
  b->nodes[node_idx - 1].right = rc;
  return node_idx;
}

void assign_miss(orc_bvh* b, int64_t node, int64_t next) {  // src/GPUBVH.jl:69-82
  b->nodes[node - 1].miss = next;
  const orc_bvh::Node& nd = b->nodes[node - 1];
  if (nd.left != 0) {
    int64_t l = nd.left, r = nd.right;
    assign_miss(b, l, r);
    assign_miss(b, r, next);
  }
}

// slab test, src/GPUBVH.jl:219-229 (== src/BVH.jl:155-169)
inline bool slab(const double* lo, const double* hi, const double* o, const double* inv, double tmax) {
  double t1x = (lo[0] - o[0]) * inv[0], t2x = (hi[0] - o[0]) * inv[0];
  double t1y = (lo[1] - o[1]) * inv[1], t2y = (hi[1] - o[1]) * inv[1];
  double t1z = (lo[2] - o[2]) * inv[2], t2z = (hi[2] - o[2]) * inv[2];
  double tentry = jmax(jmax(jmax(jmin(t1x, t2x), jmin(t1y, t2y)), jmin(t1z, t2z)), 0.0);
  double texit = jmin(jmin(jmin(jmax(t1x, t2x), jmax(t1y, t2y)), jmax(t1z, t2z)), tmax);
  return tentry <= texit;
}

// Moller-Trumbore as in src/GPUBVH.jl:247-269; returns t or +inf on reject.
inline double mt(const double* v0, const double* v1, const double* v2, const double* o, const double* d) {
  double e1x = v1[0] - v0[0], e1y = v1[1] - v0[1], e1z = v1[2] - v0[2];
  double e2x = v2[0] - v0[0], e2y = v2[1] - v0[1], e2z = v2[2] - v0[2];
  double hx = d[1] * e2z - d[2] * e2y;
  double hy = d[2] * e2x - d[0] * e2z;
  double hz = d[0] * e2y - d[1] * e2x;
  double a = (e1x * hx + e1y * hy) + e1z * hz;
  if (std::fabs(a) < 1e-10) return INFINITY;
  double f = 1.0 / a;
  double sx = o[0] - v0[0], sy = o[1] - v0[1], sz = o[2] - v0[2];
  double u = f * ((sx * hx + sy * hy) + sz * hz);
  if (u < 0.0 || u > 1.0) return INFINITY;
  double qx = sy * e1z - sz * e1y;
  double qy = sz * e1x - sx * e1z;
  double qz = sx * e1y - sy * e1x;
  double v = f * ((d[0] * qx + d[1] * qy) + d[2] * qz);
  if (v < 0.0 || u + v > 1.0) return INFINITY;
  return f * ((e2x * qx + e2y * qy) + e2z * qz);
}

void tri_vertices(const orc_bvh* b, int64_t t, int geometric, double* v0, double* v1, double* v2) {
  const double* s = b->soup + 9 * t;
  if (geometric) {
    for (int c = 0; c < 3; ++c) { v0[c] = s[c]; v1[c] = s[3 + c]; v2[c] = s[6 + c]; }
  } else {
    // bvh_tris[a, c, t] with a = vertex slot, c = xyz (src/GPUBVH.jl:243-245):
    // reads element a + 3c of the (3,3,T) soup, i.e. the transposed triangle.
    for (int c = 0; c < 3; ++c) { v0[c] = s[0 + 3 * c]; v1[c] = s[1 + 3 * c]; v2[c] = s[2 + 3 * c]; }
  }
}

// src/BVH.jl:265-276
inline bool seg_blocks_ray(const double* xi, const double* xj, const double* v0, const double* v1) {
  const double tol = 1e-8;
  double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
  double ex = v1[0] - v0[0], ey = v1[1] - v0[1];
  double denom = dx * ey - dy * ex;
  if (std::fabs(denom) < tol) return false;
  double fx = v0[0] - xi[0], fy = v0[1] - xi[1];
  double s = (fx * ey - fy * ex) / denom;
  double t = (fx * dy - fy * dx) / denom;
  return (tol < s && s < 1.0 - tol) && (tol < t && t < 1.0 - tol);
}

}  // namespace

extern "C" {

int orc_gl_1d(int n, double* pts, double* wts) {
  std::vector<double> p, w;
  gl1d(n, p, w);
  for (int i = 0; i < n; ++i) { pts[i] = p[i]; wts[i] = w[i]; }
  return n;
}
int orc_gl_2d(int n, double* pts, double* wts) {
  std::vector<double> x, e, w;
  gl2d(n, x, e, w);
  for (int k = 0; k < n * n; ++k) { pts[2 * k] = x[k]; pts[2 * k + 1] = e[k]; wts[k] = w[k]; }
  return n * n;
}
int orc_tri_rule(int nquad, double* pts, double* wts) {
  std::vector<double> x, e, w;
  tri_rule(nquad, x, e, w);
  for (size_t k = 0; k < w.size(); ++k) { pts[2 * k] = x[k]; pts[2 * k + 1] = e[k]; wts[k] = w[k]; }
  return (int)w.size();
}
void orc_quad8_shape(double xi, double eta, double* N, double* a, double* b) { quad8_shape(xi, eta, N, a, b); }
void orc_quad4_shape(double xi, double eta, double* N, double* a, double* b) { quad4_shape(xi, eta, N, a, b); }
void orc_tri6_shape(double xi, double eta, double* N, double* a, double* b) { tri6_shape(xi, eta, N, a, b); }
void orc_tri3_shape(double xi, double eta, double* N, double* a, double* b) { tri3_shape(xi, eta, N, a, b); }
void orc_line3_shape(double xi, double* N, double* dN) { line3_shape(xi, N, dN); }
void orc_line2_shape(double xi, double* N, double* dN) { line2_shape(xi, N, dN); }

void orc_eval_point(const orc_mesh* m, int64_t e, double xi, double eta, int cpu_norm, double* x, double* n,
                    double* dA) {
  (void)cpu_norm;  // both evaluators form |c| as sqrt(dot(c,c)) for finite normal-range inputs
  if (is_line_fam(m->family[e])) eval_line(m, e, xi, x, n, dA);
  else eval_surface(m, e, xi, eta, x, n, dA);
}

double orc_vf_kernel(const double* xi, const double* ni, const double* xj, const double* nj) {
  return vf_kernel(xi, ni, xj, nj);
}
double orc_vf_kernel_2d(const double* xi, const double* ni, const double* xj, const double* nj) {
  return vf_kernel_2d(xi, ni, xj, nj);
}

orc_bvh* orc_bvh_build(const double* soup, int32_t nv, int64_t n_prims) {
  if (n_prims <= 0) return nullptr;
  orc_bvh* b = new orc_bvh();
  b->soup = soup;
  b->nv = nv;
  b->T = n_prims;
  b->tri_idx.resize(n_prims);
  for (int64_t i = 0; i < n_prims; ++i) b->tri_idx[i] = i + 1;
  build_rec(b, 1, n_prims);
  assign_miss(b, 1, 0);
  return b;
}
void orc_bvh_free(orc_bvh* b) { delete b; }
int64_t orc_bvh_n_nodes(const orc_bvh* b) { return b ? (int64_t)b->nodes.size() : 0; }
void orc_bvh_export(const orc_bvh* b, double* lo, double* hi, int32_t* meta, int32_t* tri_idx) {
  for (size_t k = 0; k < b->nodes.size(); ++k) {
    const orc_bvh::Node& n = b->nodes[k];
    for (int c = 0; c < 3; ++c) { lo[3 * k + c] = n.lo[c]; hi[3 * k + c] = n.hi[c]; }
    meta[5 * k + 0] = (int32_t)n.left;
    meta[5 * k + 1] = (int32_t)n.right;
    meta[5 * k + 2] = (int32_t)n.tri_start;
    meta[5 * k + 3] = (int32_t)n.tri_count;
    meta[5 * k + 4] = (int32_t)n.miss;
  }
  for (int64_t t = 0; t < b->T; ++t) tri_idx[t] = (int32_t)b->tri_idx[t];
}

// src/GPUBVH.jl:202-285
int orc_intersect_flat(const orc_bvh* b, const int32_t* prim_group, const double* o, const double* d,
                       double t_max, int32_t gi, int32_t gj, int geometric, int64_t* counters) {
  double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
  const double t_eps = (double)1e-6f;  // Float32 literal cast to Float64 (src/GPUBVH.jl:200)
  int64_t nidx = 1;
  while (nidx > 0) {
    const orc_bvh::Node& nd = b->nodes[nidx - 1];
    if (counters) counters[2]++;
    if (slab(nd.lo, nd.hi, o, inv, t_max)) {
      if (nd.tri_count > 0) {
        for (int64_t k = nd.tri_start; k <= nd.tri_start + nd.tri_count - 1; ++k) {
          int64_t tidx = b->tri_idx[k - 1];
          int32_t tg = prim_group[tidx - 1];
          if (tg == gi || tg == gj) continue;
          double v0[3], v1[3], v2[3];
          tri_vertices(b, tidx - 1, geometric, v0, v1, v2);
          if (counters) counters[3]++;
          double t = mt(v0, v1, v2, o, d);
          if (t > t_eps && t < t_max) return 1;
        }
        nidx = nd.miss;
      } else {
        nidx = nd.left;
      }
    } else {
      nidx = nd.miss;
    }
  }
  return 0;
}

// src/BVH.jl:213-250 (stack traversal, t_min = 0.0)
int orc_intersect_ray_cpu(const orc_bvh* b, const double* o, const double* d, double t_max) {
  double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
  int64_t stack[64];
  int sp = 0;
  stack[sp++] = 1;
  while (sp > 0) {
    int64_t nidx = stack[--sp];
    const orc_bvh::Node& nd = b->nodes[nidx - 1];
    if (!slab(nd.lo, nd.hi, o, inv, t_max)) continue;
    if (nd.left == 0) {
      for (int64_t k = nd.tri_start; k <= nd.tri_start + nd.tri_count - 1; ++k) {
        int64_t tidx = b->tri_idx[k - 1];
        double v0[3], v1[3], v2[3];
        tri_vertices(b, tidx - 1, 0, v0, v1, v2);
        double t = mt(v0, v1, v2, o, d);
        double tt = (t > 0.0) ? t : INFINITY;
        if (tt < t_max) return 1;
      }
    } else {
      stack[sp++] = nd.left;
      stack[sp++] = nd.right;
    }
  }
  return 0;
}

// src/BVH.jl:285-322 with per-primitive group skip (equivalent to the CPU
// path's per-subset tree for segments: culling never drops a blocking segment).
int orc_intersect_seg(const orc_bvh* b, const int32_t* prim_group, const double* xi, const double* xj,
                      int32_t gi, int32_t gj) {
  double rxlo = jmin(xi[0], xj[0]), rxhi = jmax(xi[0], xj[0]);
  double rylo = jmin(xi[1], xj[1]), ryhi = jmax(xi[1], xj[1]);
  int64_t stack[64];
  int sp = 0;
  stack[sp++] = 1;
  while (sp > 0) {
    int64_t nidx = stack[--sp];
    const orc_bvh::Node& nd = b->nodes[nidx - 1];
    if (nd.lo[0] > rxhi || nd.hi[0] < rxlo || nd.lo[1] > ryhi || nd.hi[1] < rylo) continue;
    if (nd.left == 0) {
      for (int64_t k = nd.tri_start; k <= nd.tri_start + nd.tri_count - 1; ++k) {
        int64_t tidx = b->tri_idx[k - 1];
        if (prim_group && (prim_group[tidx - 1] == gi || prim_group[tidx - 1] == gj)) continue;
        double v0[3] = {S(b, 0, 0, tidx - 1), S(b, 1, 0, tidx - 1), 0.0};
        double v1[3] = {S(b, 0, 1, tidx - 1), S(b, 1, 1, tidx - 1), 0.0};
        if (seg_blocks_ray(xi, xj, v0, v1)) return 1;
      }
    } else {
      stack[sp++] = nd.left;
      stack[sp++] = nd.right;
    }
  }
  return 0;
}

// src/RayCast.jl:20-32
int orc_is_visible_cpu(const orc_bvh* b, const double* xi, const double* xj, int mesh_dim) {
  if (mesh_dim == 1) return !orc_intersect_seg(b, nullptr, xi, xj, 0, 0);
  double d[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
  double L = std::sqrt(dot3(d, d));
  if (L < 2.220446049250313e-16) return 1;
  double u[3] = {d[0] / L, d[1] / L, d[2] / L};
  return !orc_intersect_ray_cpu(b, xi, u, L);
}

uint64_t orc_init_rng(uint64_t seed, uint64_t tid) {  // src/GPUMCKernels.jl:44-50
  uint64_t z = seed + tid * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double orc_xorshift64(uint64_t* state) {  // src/GPUMCKernels.jl:37-42
  uint64_t s = *state;
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  *state = s;
  return (double)(s >> 11) / (double)0x001FFFFFFFFFFFFFULL;
}

}  // extern "C"

namespace {

int threads_for(int n_threads) {
#ifdef _OPENMP
  return n_threads > 0 ? n_threads : omp_get_max_threads();
#else
  (void)n_threads;
  return 1;
#endif
}

// GPU-path ray test for one point pair (src/GPUKernels.jl:289-304).
// Returns 1 if blocked.
inline int ray_blocked_gpu(const orc_bvh* bvh, const int32_t* pg, const double* xi, const double* xj,
                           int32_t gi, int32_t gj, int geometric, int64_t* cnt) {
  double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
  double rlen = std::sqrt((rx * rx + ry * ry) + rz * rz);
  if (!(rlen > 1e-15)) return 0;
  double inv_r = 1.0 / rlen;
  double o[3] = {xi[0], xi[1], xi[2]};
  double d[3] = {rx * inv_r, ry * inv_r, rz * inv_r};
  if (cnt) cnt[1]++;
  return orc_intersect_flat(bvh, pg, o, d, rlen, gi, gj, geometric, cnt);
}

// One pair i < j of src/GPUKernels.jl:276-310 (the double quadrature loop
// with the shadow ray of each point pair with K > 0), or of
// src/ViewFactorKernel.jl:199-241 on curve meshes; c: counters as in
// orc_solve_plain; lg_pair (optional): the pair's ray log, stride pm.
template <class PT>
double pair_plain(const orc_mesh* m, const orc_bvh* bvh, const PT& Pi, const PT& Pj, int32_t gi, int32_t gj,
                  int geometric, int64_t* c, uint8_t* lg_pair, int32_t pm) {
  const bool two_d = (m->mesh_dim == 1);
  double Fij = 0.0;
  for (int p = 0; p < Pi.np; ++p) {
    double inner = 0.0;
    for (int q = 0; q < Pj.np; ++q) {
      c[0]++;
      uint8_t lg = 0;
      double K;
      if (two_d) {
        K = vf_kernel_2d(Pi.X(p), Pi.Nn(p), Pj.X(q), Pj.Nn(q));
        if (K > 0.0 && bvh) {
          c[1]++;
          int blk = orc_intersect_seg(bvh, m->obs_group, Pi.X(p), Pj.X(q), gi, gj);
          lg = blk ? 2 : 1;
          if (blk) K = 0.0;
        }
      } else {
        K = vf_kernel(Pi.X(p), Pi.Nn(p), Pj.X(q), Pj.Nn(q));
        if (bvh && K > 0.0) {
          int64_t before = c[1];
          int blk = ray_blocked_gpu(bvh, m->obs_group, Pi.X(p), Pj.X(q), gi, gj, geometric, c);
          if (c[1] != before) lg = blk ? 2 : 1;
          if (blk) K = 0.0;
        }
      }
      if (lg_pair) lg_pair[p * pm + q] = lg;
      inner += (Pj.W(q) * K) * Pj.DA(q);
    }
    Fij += (Pi.W(p) * inner) * Pi.DA(p);
  }
  return Fij;
}

}  // namespace

extern "C" {

// src/GPUKernels.jl:226-323 (+ the curve-mesh quadrature of
// src/ViewFactorKernel.jl:199-241 for mesh_dim == 1)
int orc_solve_plain(const orc_mesh* m, int nquad, int geometric, int64_t row_begin, int64_t row_end,
                    int64_t row_stride, int n_threads, double* raw, double* area, uint8_t* ray_log, int32_t pm,
                    int64_t* counters) {
  const int64_t N = m->n_elems;
  Rules R = make_rules(nquad);
  std::vector<Pts> P(N);
  for (int64_t e = 0; e < N; ++e) element_points(m, e, R, P[e]);
  for (int64_t e = 0; e < N; ++e) {
    double A = 0.0;
    for (int p = 0; p < P[e].np; ++p) A += P[e].w[p] * P[e].dA[p];
    area[e] = (N >= 2) ? A : 0.0;  // area is only written by pair threads
  }
  orc_bvh* bvh = (m->n_obs > 0) ? orc_bvh_build(m->obs_soup, m->obs_nv, m->n_obs) : nullptr;
  if (row_stride < 1) row_stride = 1;
  if (row_end > N) row_end = N;
  std::vector<int64_t> rows;
  for (int64_t i = row_begin; i < row_end; i += row_stride) rows.push_back(i);
  int nt = threads_for(n_threads);
  int64_t tot[4] = {0, 0, 0, 0};
  std::mutex mu;
#pragma omp parallel num_threads(nt)
  {
    int64_t c[4] = {0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t ri = 0; ri < (int64_t)rows.size(); ++ri) {
      int64_t i = rows[ri];
      const Pts& Pi = P[i];
      int32_t gi = m->elem_group[i];
      for (int64_t j = i + 1; j < N; ++j) {
        const Pts& Pj = P[j];
        int32_t gj = m->elem_group[j];
        uint8_t* lg = ray_log ? ray_log + (i * N + j) * pm * pm : nullptr;
        const double Fij = pair_plain(m, bvh, Pi, Pj, gi, gj, geometric, c, lg, pm);
        raw[i + j * N] = Fij;
        raw[j + i * N] = Fij;
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    for (int k = 0; k < 4; ++k) tot[k] += c[k];
  }
  if (counters) for (int k = 0; k < 4; ++k) counters[k] = tot[k];
  orc_bvh_free(bvh);
  return 0;
}

// Whole rows of raw for the sampled elements rows[0..n_rows): out[r*N + j] =
// raw[rows[r], j] (0 on the diagonal), each pair integrated as
// orc_solve_plain integrates it (lower index first); the points live in
// compact arrays, so large meshes fit.
int orc_solve_rows(const orc_mesh* m, int nquad, int geometric, const int64_t* rows, int64_t n_rows, int n_threads,
                   double* out, double* area, int64_t* counters) {
  const int64_t N = m->n_elems;
  Rules R = make_rules(nquad);
  std::vector<int> npts(N);
  std::vector<int64_t> off(N + 1, 0);
  for (int64_t e = 0; e < N; ++e) {
    const int f = m->family[e];
    npts[e] = is_line_fam(f) ? (int)R.lx.size() : is_quad_fam(f) ? (int)R.qw.size() : (int)R.tw.size();
    off[e + 1] = off[e] + npts[e];
  }
  std::vector<double> X(3 * off[N]), Nv(3 * off[N]), W(off[N]), DA(off[N]);
  const int nt = threads_for(n_threads);
#pragma omp parallel num_threads(nt)
  {
    std::unique_ptr<Pts> tmp(new Pts());
#pragma omp for schedule(static)
    for (int64_t e = 0; e < N; ++e) {
      element_points(m, e, R, *tmp);
      for (int p = 0; p < tmp->np; ++p) {
        for (int k = 0; k < 3; ++k) {
          X[3 * (off[e] + p) + k] = tmp->x[p][k];
          Nv[3 * (off[e] + p) + k] = tmp->n[p][k];
        }
        W[off[e] + p] = tmp->w[p];
        DA[off[e] + p] = tmp->dA[p];
      }
      double A = 0.0;
      for (int p = 0; p < tmp->np; ++p) A += tmp->w[p] * tmp->dA[p];
      area[e] = (N >= 2) ? A : 0.0;
    }
  }
  auto view = [&](int64_t e) {
    PtsView v;
    v.np = npts[e];
    v.x = X.data() + 3 * off[e];
    v.n = Nv.data() + 3 * off[e];
    v.w = W.data() + off[e];
    v.dA = DA.data() + off[e];
    return v;
  };
  orc_bvh* bvh = (m->n_obs > 0) ? orc_bvh_build(m->obs_soup, m->obs_nv, m->n_obs) : nullptr;
  constexpr int64_t kBlock = 256;
  const int64_t nb = (N + kBlock - 1) / kBlock;
  int64_t tot[4] = {0, 0, 0, 0};
  std::mutex mu;
#pragma omp parallel num_threads(nt)
  {
    int64_t c[4] = {0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t w = 0; w < n_rows * nb; ++w) {
      const int64_t r = w / nb, j0 = (w % nb) * kBlock, j1 = std::min<int64_t>(N, j0 + kBlock);
      const int64_t i = rows[r];
      for (int64_t j = j0; j < j1; ++j) {
        if (j == i) {
          out[r * N + j] = 0.0;
          continue;
        }
        const int64_t a = std::min(i, j), b = std::max(i, j);
        out[r * N + j] = pair_plain(m, bvh, view(a), view(b), m->elem_group[a], m->elem_group[b], geometric, c,
                                    (uint8_t*)nullptr, 0);
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    for (int k = 0; k < 4; ++k) tot[k] += c[k];
  }
  if (counters) for (int k = 0; k < 4; ++k) counters[k] = tot[k];
  orc_bvh_free(bvh);
  return 0;
}

// The diagonal of src/GPUKernels.jl:226-323 (i = j), for self_vf
// (src/Assembly.jl:173,193).
int orc_self_gpu(const orc_mesh* m, int nquad, int geometric, double* raw_diag, double* area) {
  const int64_t N = m->n_elems;
  Rules R = make_rules(nquad);
  orc_bvh* bvh = (m->n_obs > 0) ? orc_bvh_build(m->obs_soup, m->obs_nv, m->n_obs) : nullptr;
  const bool two_d = (m->mesh_dim == 1);
  for (int64_t e = 0; e < N; ++e) {
    Pts P;
    element_points(m, e, R, P);
    double A = 0.0;
    for (int p = 0; p < P.np; ++p) A += P.w[p] * P.dA[p];
    area[e] = A;
    const int32_t g = m->elem_group[e];
    double Fii = 0.0;
    for (int p = 0; p < P.np; ++p) {
      double inner = 0.0;
      for (int q = 0; q < P.np; ++q) {
        double K;
        if (two_d) {
          K = vf_kernel_2d(P.x[p], P.n[p], P.x[q], P.n[q]);
          if (K > 0.0 && bvh && orc_intersect_seg(bvh, m->obs_group, P.x[p], P.x[q], g, g)) K = 0.0;
        } else {
          K = vf_kernel(P.x[p], P.n[p], P.x[q], P.n[q]);
          if (bvh && K > 0.0 && ray_blocked_gpu(bvh, m->obs_group, P.x[p], P.x[q], g, g, geometric, nullptr))
            K = 0.0;
        }
        inner += (P.w[q] * K) * P.dA[q];
      }
      Fii += (P.w[p] * inner) * P.dA[p];
    }
    raw_diag[e] = Fii;
  }
  orc_bvh_free(bvh);
  return 0;
}

}  // extern "C"

namespace {

// src/GPUMCKernels.jl:266-281 (surface) / 2-D extension (lines)
inline void mc_sample(const orc_mesh* m, int64_t e, double u1, double u2, double* x, double* n, double* dA) {
  int f = m->family[e];
  if (is_quad_fam(f)) {
    double xi = 2.0 * u1 - 1.0, eta = 2.0 * u2 - 1.0;
    eval_surface(m, e, xi, eta, x, n, dA);
  } else {
    double xi = u1, eta = u2;
    if (xi + eta > 1.0) { xi = 1.0 - xi; eta = 1.0 - eta; }
    eval_surface(m, e, xi, eta, x, n, dA);
  }
}
inline double ref_measure(int f) { return is_quad_fam(f) ? 4.0 : (is_line_fam(f) ? 2.0 : 0.5); }

// One MC pair, i<j (0-based).  Returns raw; writes the two area estimates.
double mc_pair(const orc_mesh* m, const orc_bvh* bvh, int64_t i, int64_t j, int n_samples, uint64_t seed,
               int exclude_groups, int geometric, double* Ai_out, double* Aj_out, uint8_t* log_pair,
               int64_t* c) {
  const int64_t N = m->n_elems;
  const bool two_d = (m->mesh_dim == 1);
  int fi = m->family[i], fj = m->family[j];
  // curves always skip their own groups, as the quadrature path's 2-D test does
  const bool excl = exclude_groups || two_d;
  int32_t gi = excl ? m->elem_group[i] : 0;
  int32_t gj = excl ? m->elem_group[j] : 0;
  uint64_t tid = (uint64_t)(i * N + j + 1);  // (i-1)*N + j with 1-based i, j
  uint64_t st = orc_init_rng(seed, tid);
  double Ai = 0.0, Aj = 0.0, Ks = 0.0;
  int s = (int)std::floor(std::sqrt((double)n_samples));
  int k = 0;
  auto one = [&](double ai1, double ai2, double aj1, double aj2) {
    double xi[3], ni[3], dAi, xj[3], nj[3], dAj, K;
    if (two_d) {
      eval_line(m, i, ai1, xi, ni, &dAi);
      eval_line(m, j, aj1, xj, nj, &dAj);
    } else {
      mc_sample(m, i, ai1, ai2, xi, ni, &dAi);
      mc_sample(m, j, aj1, aj2, xj, nj, &dAj);
    }
    Ai += dAi;
    Aj += dAj;
    uint8_t lg = 0;
    if (c) c[0]++;
    if (two_d) {
      K = vf_kernel_2d(xi, ni, xj, nj);
      if (K > 0.0 && bvh) {
        if (c) c[1]++;
        int blk = orc_intersect_seg(bvh, m->obs_group, xi, xj, gi, gj);
        lg = blk ? 2 : 1;
        if (blk) K = 0.0;
      }
    } else {
      K = vf_kernel(xi, ni, xj, nj);
      if (K > 0.0 && bvh) {
        int64_t before = c ? c[1] : 0;
        int blk = ray_blocked_gpu(bvh, m->obs_group, xi, xj, gi, gj, geometric, c);
        if (!c || c[1] != before) lg = blk ? 2 : 1;
        if (blk) K = 0.0;
      }
    }
    if (log_pair) log_pair[k] = lg;
    Ks += (K * dAi) * dAj;
    ++k;
  };
  for (int si = 0; si < s; ++si)
    for (int sj = 0; sj < s; ++sj) {
      double u1 = orc_xorshift64(&st), u2 = orc_xorshift64(&st);
      double u3 = orc_xorshift64(&st), u4 = orc_xorshift64(&st);
      if (two_d) {
        one(2.0 * ((si + u1) / s) - 1.0, 0.0, 2.0 * ((sj + u3) / s) - 1.0, 0.0);
      } else {
        one((si + u1) / s, (sj + u2) / s, (si + u3) / s, (sj + u4) / s);
      }
    }
  for (int r = s * s; r < n_samples; ++r) {
    double u1 = orc_xorshift64(&st), u2 = orc_xorshift64(&st);
    double u3 = orc_xorshift64(&st), u4 = orc_xorshift64(&st);
    if (two_d) one(2.0 * u1 - 1.0, 0.0, 2.0 * u3 - 1.0, 0.0);
    else one(u1, u2, u3, u4);
  }
  double ri = ref_measure(fi), rj = ref_measure(fj);
  *Ai_out = (Ai * ri) / (double)n_samples;
  *Aj_out = (Aj * rj) / (double)n_samples;
  return ((Ks * ri) * rj) / (double)n_samples;
}

}  // namespace

extern "C" {

int orc_solve_mc(const orc_mesh* m, int n_samples, uint64_t seed, int exclude_groups, int geometric,
                 int64_t row_begin, int64_t row_end, int64_t row_stride, int n_threads, double* raw, double* area,
                 uint8_t* ray_log, int64_t* counters) {
  const int64_t N = m->n_elems;
  orc_bvh* bvh = (m->n_obs > 0) ? orc_bvh_build(m->obs_soup, m->obs_nv, m->n_obs) : nullptr;
  for (int64_t e = 0; e < N; ++e) area[e] = 0.0;
  // deterministic area rule
  for (int64_t e = 0; e < N && N >= 2; ++e) {
    double a, b;
    if (e + 1 < N) { mc_pair(m, bvh, e, e + 1, n_samples, seed, exclude_groups, geometric, &a, &b, nullptr, nullptr); area[e] = a; }
    else { mc_pair(m, bvh, e - 1, e, n_samples, seed, exclude_groups, geometric, &a, &b, nullptr, nullptr); area[e] = b; }
  }
  if (row_stride < 1) row_stride = 1;
  if (row_end > N) row_end = N;
  std::vector<int64_t> rows;
  for (int64_t i = row_begin; i < row_end; i += row_stride) rows.push_back(i);
  int nt = threads_for(n_threads);
  int64_t tot[4] = {0, 0, 0, 0};
  std::mutex mu;
#pragma omp parallel num_threads(nt)
  {
    int64_t c[4] = {0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t ri = 0; ri < (int64_t)rows.size(); ++ri) {
      int64_t i = rows[ri];
      for (int64_t j = i + 1; j < N; ++j) {
        double a, b;
        uint8_t* lp = ray_log ? ray_log + (i * N + j) * (int64_t)n_samples : nullptr;
        double r = mc_pair(m, bvh, i, j, n_samples, seed, exclude_groups, geometric, &a, &b, lp, c);
        raw[i + j * N] = r;
        raw[j + i * N] = r;
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    for (int k = 0; k < 4; ++k) tot[k] += c[k];
  }
  if (counters) for (int k = 0; k < 4; ++k) counters[k] = tot[k];
  orc_bvh_free(bvh);
  return 0;
}

// src/DuffyKernel.jl:95-115
int orc_singularity_type(const orc_mesh* m, int64_t i, int64_t j, int32_t* ci, int32_t* cj) {
  if (m->family[i] != 0 || m->family[j] != 0) return 0;
  int n = 0;
  const int32_t* a = m->elem_nodes + 8 * i;
  const int32_t* b = m->elem_nodes + 8 * j;
  for (int x = 0; x < 4; ++x)
    for (int y = 0; y < 4; ++y)
      if (a[x] == b[y]) {
        if (n < 2) { ci[n] = x + 1; cj[n] = y + 1; }
        ++n;
      }
  if (n == 0) return 0;
  if (n == 1) return 1;
  return 2;
}

}  // extern "C"

namespace {

const double CORNER_UV[4][2] = {{0.0, 0.0}, {1.0, 0.0}, {1.0, 1.0}, {0.0, 1.0}};  // src/DuffyKernel.jl:122-127

// src/DuffyKernel.jl:288-314
inline void vertex_map(int region, double r, double a, double b, double c, double u0i, double v0i, double u0j,
                       double v0j, double* U) {
  double du, dv, ds, dt;
  switch (region) {
    case 1: du = r; dv = r * a; ds = r * b; dt = (r * b) * c; break;
    case 2: du = r; dv = r * a; ds = (r * b) * c; dt = r * b; break;
    case 3: du = r * a; dv = r; ds = r * b; dt = (r * b) * c; break;
    case 4: du = r * a; dv = r; ds = (r * b) * c; dt = r * b; break;
    case 5: du = r * b; dv = (r * b) * c; ds = r; dt = r * a; break;
    case 6: du = (r * b) * c; dv = r * b; ds = r; dt = r * a; break;
    case 7: du = r * b; dv = (r * b) * c; ds = r * a; dt = r; break;
    default: du = (r * b) * c; dv = r * b; ds = r * a; dt = r; break;
  }
  U[0] = u0i + (u0i == 0.0 ? du : -du);
  U[1] = v0i + (v0i == 0.0 ? dv : -dv);
  U[2] = u0j + (u0j == 0.0 ? ds : -ds);
  U[3] = v0j + (v0j == 0.0 ? dt : -dt);
}

// src/DuffyKernel.jl:375-408 (region 4 uses its final, overriding form)
inline void edge_map(int region, double r, double a, double b, double c, double* U) {
  switch (region) {
    case 1: {
      double A = r * (1 - a * (1 - c));
      U[0] = A;
      U[1] = ((r * a) * b) * c;
      U[2] = (A - ((r * a) * (1 - b)) * c) + ((r * a) * b) * c;
      U[3] = ((r * a) * (1 - b)) * c;
      break;
    }
    case 2: {
      double A = r * (1 - (a * b) * c);
      U[0] = A;
      U[1] = ((r * a) * c) * (1 - b);
      U[2] = (A + ((r * a) * b) * c) - (r * a) * c;
      U[3] = ((r * a) * b) * c;
      break;
    }
    case 3: {
      double A = r * (1 - a * b);
      U[0] = A;
      U[1] = ((r * a) * b) * c;
      U[2] = A - ((r * a) * b) * (1 - c);
      U[3] = ((r * a) * b) * (1 - c);
      break;
    }
    case 4: {
      U[0] = r * (b * c + a * (1 - b * c));
      U[1] = ((r * (1 - a)) * b) * c;
      U[2] = (r * b) * c;
      U[3] = ((r * (1 - a)) * b) * c;
      break;
    }
    default: {
      U[0] = (r * a) * c;
      U[1] = ((r * (1 - a)) * b) * c;
      U[2] = (((r * a) * c) * (1 - b)) + (((r * a) * b) * c);
      U[3] = ((r * (1 - a)) * b) * c;
      break;
    }
  }
}
int corners_to_edge(int c1, int c2) {  // src/DuffyKernel.jl:411-419
  int a = std::min(c1, c2), b = std::max(c1, c2);
  if (a == 1 && b == 2) return 1;
  if (a == 2 && b == 3) return 2;
  if (a == 3 && b == 4) return 3;
  if (a == 1 && b == 4) return 4;
  return 1;
}
inline void rotate_to_edge(double u, double v, int e, double* ou, double* ov) {  // :423-429
  switch (e) {
    case 2: *ou = 1.0 - v; *ov = u; return;
    case 3: *ou = 1.0 - u; *ov = 1.0 - v; return;
    case 4: *ou = v; *ov = 1.0 - u; return;
    default: *ou = u; *ov = v; return;
  }
}
// src/DuffyKernel.jl:134-139
inline void eval_quad01(const orc_mesh* m, int64_t e, double u, double v, double* x, double* n, double* dA) {
  double xi = 2 * u - 1.0, eta = 2 * v - 1.0;
  eval_surface(m, e, xi, eta, x, n, dA);
  *dA = *dA * 4.0;
}

}  // namespace

extern "C" {

// src/DuffyKernel.jl:452-487 for one ordered pair (i,j).  bvh == NULL: no
// occlusion.  gpu_semantics == 0: the CPU path's is_visible on `bvh` (the
// per-subset tree of src/Assembly.jl:121-143).  gpu_semantics == 1: the GPU
// path's ray (src/GPUKernels.jl:289-304) on the single tree with group skip.
double orc_pair_duffy(const orc_mesh* m, const orc_bvh* bvh, int gpu_semantics, int geometric, int64_t i,
                      int64_t j, int nquad, double* Ai_out, int* stype_out) {
  Rules R = make_rules(nquad);
  int32_t gi = m->elem_group[i], gj = m->elem_group[j];
  auto visible = [&](const double* xi, const double* xj) -> bool {
    if (!bvh) return true;
    if (gpu_semantics) return !ray_blocked_gpu(bvh, m->obs_group, xi, xj, gi, gj, geometric, nullptr);
    return orc_is_visible_cpu(bvh, xi, xj, m->mesh_dim) != 0;
  };
  auto standard = [&](double* Li) {
    Pts Pi, Pj;
    element_points(m, i, R, Pi);
    element_points(m, j, R, Pj);
    double Fij = 0.0, L = 0.0;
    for (int p = 0; p < Pi.np; ++p) {
      L += Pi.w[p] * Pi.dA[p];
      double inner = 0.0;
      for (int q = 0; q < Pj.np; ++q) {
        double K = (m->mesh_dim == 1) ? vf_kernel_2d(Pi.x[p], Pi.n[p], Pj.x[q], Pj.n[q])
                                      : vf_kernel(Pi.x[p], Pi.n[p], Pj.x[q], Pj.n[q]);
        if (K == 0.0) continue;
        if (!visible(Pi.x[p], Pj.x[q])) continue;
        inner += (Pj.w[q] * K) * Pj.dA[q];
      }
      Fij += (Pi.w[p] * inner) * Pi.dA[p];
    }
    if (Li) *Li = L;
    return Fij;
  };
  if (m->family[i] != 0 || m->family[j] != 0 || m->mesh_dim == 1) {
    *stype_out = -1;
    return standard(Ai_out);
  }
  double Ai = 0.0;
  for (size_t p = 0; p < R.qw.size(); ++p) {
    double x[3], n[3], dA;
    eval_surface(m, i, R.qx[p], R.qe[p], x, n, &dA);
    Ai += R.qw[p] * dA;
  }
  *Ai_out = Ai;
  int32_t ci[2] = {0, 0}, cj[2] = {0, 0};
  int st = orc_singularity_type(m, i, j, ci, cj);
  *stype_out = st;
  if (st == 0) return standard(nullptr);  // _standard_integral, src/DuffyKernel.jl:157-177
  std::vector<double> p1, w1;
  gl1d(nquad, p1, w1);
  const int nq = nquad;
  std::vector<double> p01(nq), w01(nq);
  for (int k = 0; k < nq; ++k) { p01[k] = (p1[k] + 1.0) / 2.0; w01[k] = w1[k] / 2.0; }
  int nreg = (st == 1) ? 8 : 5;
  double u0i = CORNER_UV[ci[0] - 1][0], v0i = CORNER_UV[ci[0] - 1][1];
  double u0j = CORNER_UV[cj[0] - 1][0], v0j = CORNER_UV[cj[0] - 1][1];
  int edge_i = corners_to_edge(ci[0], ci[1]), edge_j = corners_to_edge(cj[0], cj[1]);
  double Fij = 0.0;
  for (int region = 1; region <= nreg; ++region)
    for (int ir = 0; ir < nq; ++ir)
      for (int i1 = 0; i1 < nq; ++i1)
        for (int i2 = 0; i2 < nq; ++i2)
          for (int i3 = 0; i3 < nq; ++i3) {
            double r = p01[ir], wr = w01[ir];
            double a = p01[i1], wa = w01[i1];
            double b = p01[i2], wb = w01[i2];
            double c = p01[i3], wc = w01[i3];
            double U[4];
            if (st == 1) {
              vertex_map(region, r, a, b, c, u0i, v0i, u0j, v0j, U);
            } else {
              double E[4];
              edge_map(region, r, a, b, c, E);
              rotate_to_edge(E[0], E[1], edge_i, &U[0], &U[1]);
              rotate_to_edge(E[2], E[3], edge_j, &U[2], &U[3]);
            }
            if (U[0] < 0 || U[0] > 1 || U[1] < 0 || U[1] > 1 || U[2] < 0 || U[2] > 1 || U[3] < 0 || U[3] > 1)
              continue;
            double xi[3], ni[3], dAi, xj[3], nj[3], dAj;
            eval_quad01(m, i, U[0], U[1], xi, ni, &dAi);
            eval_quad01(m, j, U[2], U[3], xj, nj, &dAj);
            double K = vf_kernel(xi, ni, xj, nj);
            if (K == 0.0) continue;
            if (!visible(xi, xj)) continue;
            double jac = (r * r) * r;
            Fij += ((((((wr * wa) * wb) * wc) * jac) * K) * dAi) * dAj;
          }
  return Fij;
}

// src/Assembly.jl:102-225, quadrature branch (CPU path; the timed CPU reference)
int orc_solve_cpu(const orc_mesh* m, int nquad, int use_duffy, int self_vf, const int32_t* og, int32_t n_og,
                  int64_t row_begin, int64_t row_end, int64_t row_stride, int n_threads, double* raw,
                  double* area, int64_t* counters) {
  const int64_t N = m->n_elems;
  // Areas: serial loop, element_pair_view_factor(e_i, e_i) (src/Assembly.jl:186-190).
  {
    Rules R = make_rules(nquad);
    for (int64_t e = 0; e < N; ++e) {
      Pts P;
      element_points(m, e, R, P);
      double L = 0.0, F = 0.0;
      for (int p = 0; p < P.np; ++p) {
        L += P.w[p] * P.dA[p];
        double inner = 0.0;
        for (int q = 0; q < P.np; ++q) {
          double K = (m->mesh_dim == 1) ? vf_kernel_2d(P.x[p], P.n[p], P.x[q], P.n[q])
                                        : vf_kernel(P.x[p], P.n[p], P.x[q], P.n[q]);
          if (K == 0.0) continue;
          inner += (P.w[q] * K) * P.dA[q];
        }
        F += (P.w[p] * inner) * P.dA[p];
      }
      (void)F;
      area[e] = L;
    }
  }
  // One BVH per active obstruction subset (src/Assembly.jl:121-143): soups of
  // the sorted active groups, merged in that order.
  std::map<std::vector<int32_t>, orc_bvh*> cache;
  std::vector<std::vector<double>> soups_keep;
  std::vector<int32_t> sorted_og(og, og + n_og);
  std::sort(sorted_og.begin(), sorted_og.end());
  auto subset_for = [&](int32_t gi, int32_t gj) {
    std::vector<int32_t> act;
    for (int32_t g : sorted_og)
      if (g != gi && g != gj) act.push_back(g);
    return act;
  };
  std::vector<int32_t> egroups(m->elem_group, m->elem_group + N);
  std::sort(egroups.begin(), egroups.end());
  egroups.erase(std::unique(egroups.begin(), egroups.end()), egroups.end());
  if (n_og > 0 && m->n_obs > 0) {
    for (int32_t gi : egroups)
      for (int32_t gj : egroups) {
        std::vector<int32_t> act = subset_for(gi, gj);
        if (act.empty() || cache.count(act)) continue;
        std::vector<double> merged;
        for (int32_t g : act)
          for (int64_t t = 0; t < m->n_obs; ++t)
            if (m->obs_group[t] == g)
              merged.insert(merged.end(), m->obs_soup + 3 * m->obs_nv * t, m->obs_soup + 3 * m->obs_nv * (t + 1));
        if (merged.empty()) { cache[act] = nullptr; continue; }
        soups_keep.push_back(std::move(merged));  // inner buffers survive outer reallocation
        const std::vector<double>& sk = soups_keep.back();
        cache[act] = orc_bvh_build(sk.data(), m->obs_nv, (int64_t)(sk.size() / (3 * m->obs_nv)));
      }
  }
  if (row_stride < 1) row_stride = 1;
  if (row_end > N) row_end = N;
  std::vector<int64_t> rows;
  for (int64_t i = row_begin; i < row_end; i += row_stride) rows.push_back(i);
  int nt = threads_for(n_threads);
  int64_t tot[4] = {0, 0, 0, 0};
  std::mutex mu;
#pragma omp parallel num_threads(nt)
  {
    int64_t c[4] = {0, 0, 0, 0};
    Rules R = make_rules(nquad);
#pragma omp for schedule(dynamic, 1)
    for (int64_t ri = 0; ri < (int64_t)rows.size(); ++ri) {
      int64_t i = rows[ri];
      int32_t gi = m->elem_group[i];
      for (int64_t j = self_vf ? i : i + 1; j < N; ++j) {
        int32_t gj = m->elem_group[j];
        const orc_bvh* bvh = nullptr;
        if (n_og > 0) {
          auto it = cache.find(subset_for(gi, gj));
          if (it != cache.end()) bvh = it->second;
        }
        double integ;
        if (use_duffy) {
          double Ai;
          int st;
          integ = orc_pair_duffy(m, bvh, 0, 0, i, j, nquad, &Ai, &st);
        } else {
          // element_pair_view_factor, src/ViewFactorKernel.jl:199-241 (points
          // re-evaluated per pair as _quad_points does)
          Rules Rl = make_rules(nquad);
          Pts Pi, Pj;
          element_points(m, i, Rl, Pi);
          element_points(m, j, Rl, Pj);
          double Fij = 0.0;
          for (int p = 0; p < Pi.np; ++p) {
            double inner = 0.0;
            for (int q = 0; q < Pj.np; ++q) {
              c[0]++;
              double K = (m->mesh_dim == 1) ? vf_kernel_2d(Pi.x[p], Pi.n[p], Pj.x[q], Pj.n[q])
                                            : vf_kernel(Pi.x[p], Pi.n[p], Pj.x[q], Pj.n[q]);
              if (K == 0.0) continue;
              if (bvh) {
                c[1]++;
                if (!orc_is_visible_cpu(bvh, Pi.x[p], Pj.x[q], m->mesh_dim)) continue;
              }
              inner += (Pj.w[q] * K) * Pj.dA[q];
            }
            Fij += (Pi.w[p] * inner) * Pi.dA[p];
          }
          integ = Fij;
        }
        raw[i + j * N] = integ;
        raw[j + i * N] = integ;
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    for (int k = 0; k < 4; ++k) tot[k] += c[k];
  }
  if (counters) for (int k = 0; k < 4; ++k) counters[k] = tot[k];
  for (auto& kv : cache) orc_bvh_free(kv.second);
  return 0;
}

// src/Results.jl:56-82
void orc_aggregate(int64_t N, const double* F, const double* A, const int32_t* eg, int32_t G,
                   const int32_t* tags, double* Fg, double* Ag) {
  std::vector<std::vector<int64_t>> members(G);
  for (int64_t e = 0; e < N; ++e)
    for (int32_t k = 0; k < G; ++k)
      if (eg[e] == tags[k]) members[k].push_back(e);
  for (int32_t k = 0; k < G; ++k) {
    Ag[k] = 0.0;
    for (int64_t e : members[k]) Ag[k] += A[e];
  }
  for (int64_t k = 0; k < (int64_t)G * G; ++k) Fg[k] = 0.0;
  for (int32_t gi = 0; gi < G; ++gi) {
    for (int64_t ei : members[gi])
      for (int32_t gj = 0; gj < G; ++gj) {
        double sum = 0.0;
        bool first = true;
        for (int64_t ej : members[gj]) {
          double v = F[ei + ej * N];
          sum = first ? v : sum + v;
          first = false;
        }
        Fg[gi + (int64_t)gj * G] += A[ei] * sum;
      }
    for (int32_t gj = 0; gj < G; ++gj) Fg[gi + (int64_t)gj * G] /= Ag[gi];
  }
}

// src/Results.jl:105-114
double orc_reciprocity_error(int64_t N, const double* F, const double* A) {
  double mx = 0.0;
  for (int64_t i = 0; i < N; ++i)
    for (int64_t j = i + 1; j < N; ++j) {
      double e = std::fabs(A[i] * F[i + j * N] - A[j] * F[j + i * N]) / jmax(A[i] * F[i + j * N], 1e-30);
      mx = jmax(mx, e);
    }
  return mx;
}

// sum(F, dims=2) (src/Results.jl:123)
void orc_row_sums(int64_t N, const double* F, double* out) {
  for (int64_t i = 0; i < N; ++i) out[i] = 0.0;
  for (int64_t j = 0; j < N; ++j)
    for (int64_t i = 0; i < N; ++i) out[i] += F[i + j * N];
}

}  // extern "C"
