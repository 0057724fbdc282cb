// rvf_host.h -- host-side building blocks of librvf_b200: quadrature rules,
// the exact BVH build and the device data layouts shared with the kernels.
#pragma once

#include <cstdint>
#include <vector>

namespace rvf {

// ---------------------------------------------------------------------------
// quadrature rules (src/Quadrature.jl:35-109, src/GPUKernels.jl:414-439)
// ---------------------------------------------------------------------------
struct Rule {
  std::vector<double> xi, eta, w;
  int size() const { return (int)w.size(); }
};
void gl1d(int n, std::vector<double>& p, std::vector<double>& w);
Rule gl2d(int n);        // tensor rule, xi index fastest
Rule tri_rule(int nquad);  // Dunavant 1/3/7/13 points by nquad
Rule line_rule(int n);   // 1-D Gauss-Legendre on [-1,1] (eta = 0)

// ---------------------------------------------------------------------------
// BVH (src/BVH.jl:71-148 build, src/GPUBVH.jl:69-134 miss links)
// ---------------------------------------------------------------------------
struct HostBVH {
  struct Node {
    double lo[3], hi[3];
    int64_t left, right, tri_start, tri_count, miss;  // 1-based, 0 = none (reference convention)
  };
  std::vector<Node> nodes;       // pre-order: the left child of node k is k+1
  std::vector<int64_t> tri_idx;  // 1-based primitive ids in leaf order
};
// soup layout: soup[c + 3*(v + nv*t)]
HostBVH build_bvh(const double* soup, int nv, int64_t n_prims);

// ---------------------------------------------------------------------------
// device layouts
// ---------------------------------------------------------------------------
// error flags raised by kernels (bit mask, read by the host after a launch)
constexpr int kErrWaitTimeout = 1;
constexpr int kErrBadInput = 2;
constexpr int kErrClaimGaveUp = 4;  // a tile claim ran out of retries (not an error unless nothing progressed)

constexpr int kTile = 32;      // elements per tile side
constexpr int kComp = 7;       // x, y, z, nx, ny, nz, w*dA per quadrature point
constexpr int kMaxPts = 64;    // quadrature points per element (nquad <= 8 for surfaces)
constexpr int kMaxLinePts = 32;

// FP64 BVH node, 64 B.  a = first primitive (0-based, leaf order) for leaves;
// b = primitive count (0 for interior nodes, whose left child is node+1);
// miss = pre-order successor of the subtree (n_nodes = end).
struct alignas(16) NodeD {
  double lo[3];
  double hi[3];
  int32_t a, b, miss, pad;
};
static_assert(sizeof(NodeD) == 64, "NodeD layout");

// FP64 triangle in leaf order, 80 B: vertex slot 0 and the two edge vectors
// (v1 - v0, v2 - v0) exactly as the reference forms them per test.
struct alignas(16) TriD {
  double v0[3];
  double e1[3];
  double e2[3];
  int32_t group, pad;
};
static_assert(sizeof(TriD) == 80, "TriD layout");

// 2-D segment in leaf order, 48 B: endpoints (x0,y0), (x1,y1).
struct alignas(16) SegD {
  double x0, y0, x1, y1;
  int32_t group, pad0, pad1, pad2;
};
static_assert(sizeof(SegD) == 48, "SegD layout");

// FP32 node (32 B) and triangle (48 B) for the mixed-precision traversal.
struct alignas(16) NodeF {
  float lo[3];
  float hi[3];
  int32_t ab;   // leaf: (first << 4) | count ; interior: 0
  int32_t miss;
};
static_assert(sizeof(NodeF) == 32, "NodeF layout");
struct alignas(16) TriF {
  float v0[3], e1[3], e2[3];
  int32_t group, pad0, pad1;
};
static_assert(sizeof(TriF) == 48, "TriF layout");

}  // namespace rvf
