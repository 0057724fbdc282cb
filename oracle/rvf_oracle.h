/*
 * rvf_oracle.h -- CPU restatement of RadiativeViewFactor.jl's element-pair
 * view-factor assembly.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this library: only tests/, __graft_entry__.smoke() and the CPU-baseline leg
 * of bench.py use it, and only as the checker / the timed CPU reference.
 *
 * Parity status (per part):
 *   - quadrature rules, shape functions, Quad8 geometry, vf kernel, CPU BVH ray
 *     casting / visibility, parallel-plate view factors: PINNED against the
 *     reference's own known-answer tests (test/runtests.jl:16-436), restated in
 *     tests/test_oracle_golden.py.
 *   - flat-BVH stackless traversal (src/GPUBVH.jl), GPU Monte Carlo streams
 *     (src/GPUMCKernels.jl) and the Duffy integrals (src/DuffyKernel.jl): the
 *     reference's tests hold no vectors for them -> "parity unpinned" at the
 *     reference level; they are checked against independent properties
 *     (brute-force any-hit over reachable leaves, splitmix64/xorshift64
 *     published constants, analytic view factors).
 *
 * Floating point: compiled with -O2 -ffp-contract=off (SSE2 doubles, no FMA
 * contraction), every expression written in the reference's evaluation order,
 * Julia's NaN-propagating min/max for the slab tests.
 *
 * Element family codes follow src/GPUKernels.jl:344 (0=Quad8, 1=Tri6,
 * 2=Quad4, 3=Tri3), extended with 4=Line3 and 5=Line2 for curve meshes.
 */
#ifndef RVF_ORACLE_H
#define RVF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t mesh_dim;          /* 2 = surface mesh (3-D kernel), 1 = curve mesh (2-D) */
  int64_t n_nodes;
  const double* coords;      /* 3 x n_nodes, column-major (x,y,z of node k at 3k) */
  int64_t n_elems;
  const int8_t* family;      /* per element family code */
  const int32_t* elem_nodes; /* n_elems x 8, 1-based node ids, element-major, zero padded */
  const int32_t* elem_group; /* physical group tag per element */
  int64_t n_obs;             /* obstruction primitives (merged in obstruction_groups order) */
  int32_t obs_nv;            /* 3 = triangle soup, 2 = segment soup */
  const double* obs_soup;    /* reference layout soup[c + 3*(v + nv*t)], c=xyz, v=vertex */
  const int32_t* obs_group;  /* group tag per primitive (pre-permutation) */
} orc_mesh;

/* ---- quadrature (src/Quadrature.jl, src/ViewFactorKernel.jl:42-71) ---- */
int orc_gl_1d(int n, double* pts, double* wts);
int orc_gl_2d(int n, double* pts /*2*n*n*/, double* wts);
int orc_tri_rule(int nquad, double* pts /*2*np*/, double* wts);

/* ---- shape functions (src/Geometry.jl, src/ViewFactorKernel.jl) ---- */
void orc_quad8_shape(double xi, double eta, double* N, double* dNdxi, double* dNdeta);
void orc_quad4_shape(double xi, double eta, double* N, double* dNdxi, double* dNdeta);
void orc_tri6_shape(double xi, double eta, double* N, double* dNdxi, double* dNdeta);
void orc_tri3_shape(double xi, double eta, double* N, double* dNdxi, double* dNdeta);
void orc_line3_shape(double xi, double* N, double* dN);
void orc_line2_shape(double xi, double* N, double* dN);

/* Point, unit normal and area (length) element of element e at (xi,eta).
 * cpu_norm=0: GPU evaluator semantics (src/GPUKernels.jl:95-176, sqrt(dot)).
 * cpu_norm=1: CPU evaluator semantics (src/Geometry.jl, LinearAlgebra.norm). */
void orc_eval_point(const orc_mesh* m, int64_t e, double xi, double eta, int cpu_norm,
                    double* x, double* n, double* dA);

double orc_vf_kernel(const double* xi, const double* ni, const double* xj, const double* nj);
double orc_vf_kernel_2d(const double* xi, const double* ni, const double* xj, const double* nj);

/* ---- BVH (src/BVH.jl:71-148, src/GPUBVH.jl:69-174) ---- */
typedef struct orc_bvh orc_bvh;
orc_bvh* orc_bvh_build(const double* soup, int32_t nv, int64_t n_prims);
void orc_bvh_free(orc_bvh* b);
int64_t orc_bvh_n_nodes(const orc_bvh* b);
/* lo/hi: 3*M; meta: 5*M [left,right,tri_start,tri_count,miss] (1-based as in
 * src/GPUBVH.jl:48-55); tri_idx: n_prims (1-based permutation). */
void orc_bvh_export(const orc_bvh* b, double* lo, double* hi, int32_t* meta, int32_t* tri_idx);

/* Stackless traversal, src/GPUBVH.jl:202-285 (transposed-vertex read when
 * geometric==0, exactly as the reference; true vertices when geometric==1). */
int orc_intersect_flat(const orc_bvh* b, const int32_t* prim_group,
                       const double* o, const double* d, double t_max,
                       int32_t gi, int32_t gj, int geometric, int64_t* counters);
/* CPU stack traversal, src/BVH.jl:213-250 (t_min = 0). */
int orc_intersect_ray_cpu(const orc_bvh* b, const double* o, const double* d, double t_max);
/* 2-D segment traversal, src/BVH.jl:285-322, with per-primitive group skip. */
int orc_intersect_seg(const orc_bvh* b, const int32_t* prim_group,
                      const double* xi, const double* xj, int32_t gi, int32_t gj);
/* src/RayCast.jl:20-32 */
int orc_is_visible_cpu(const orc_bvh* b, const double* xi, const double* xj, int mesh_dim);

/* ---- assembly ----
 * raw/area follow src/GPUKernels.jl:226-323: raw is N x N column-major with
 * raw[i,j] = raw[j,i] for i<j, area[i] from the same quadrature rule.
 * rows are processed for i = row_begin, row_begin+row_stride, ... < row_end.
 * ray_log (optional): byte per (i,j,p,q) at ((i*N+j)*pm + p)*pm + q,
 *   0 = no ray cast, 1 = ray cast and unobstructed, 2 = ray cast and blocked.
 * counters (optional, 4 int64): point pairs, rays, slab tests, triangle tests.
 * geometric: 0 = reference (transposed) triangle read, 1 = true vertices. */
int orc_solve_plain(const orc_mesh* m, int nquad, int geometric,
                    int64_t row_begin, int64_t row_end, int64_t row_stride, int n_threads,
                    double* raw, double* area, uint8_t* ray_log, int32_t pm, int64_t* counters);

/* Whole rows of raw (both i < j and j < i pairs, each integrated as
 * orc_solve_plain integrates it) for the sampled elements rows[0..n_rows):
 * out[r*N + j] = raw[rows[r], j], 0 on the diagonal; area as orc_solve_plain.
 * Points live in compact arrays (large meshes fit). */
int orc_solve_rows(const orc_mesh* m, int nquad, int geometric, const int64_t* rows, int64_t n_rows,
                   int n_threads, double* out, double* area, int64_t* counters);

/* Self pairs (i, i), which the reference integrates on its CPU path only
 * (self_vf, src/Assembly.jl:173,193), with the GPU path's arithmetic of
 * orc_solve_plain: the same points, kernel, summation order and shadow rays
 * (one tree, the element's own group skipped, t_eps; geometric as there).
 * raw_diag[i] = raw[i,i]; area[i] = sum_p w_p dA_p for every element. */
int orc_self_gpu(const orc_mesh* m, int nquad, int geometric, double* raw_diag, double* area);

/* GPU Monte Carlo, src/GPUMCKernels.jl:146-281.  area rule: A_i from the
 * stream of pair (i,i+1) in the i-role, A_N from pair (N-1,N) in the j-role.
 * Curve meshes (mesh_dim=1) use the 2-D extension documented in the header of
 * this library's implementation file. exclude_groups=0 passes group tags 0/0
 * to the traversal as the reference does (src/GPUMCKernels.jl:164). */
int orc_solve_mc(const orc_mesh* m, int n_samples, uint64_t seed, int exclude_groups,
                 int geometric, int64_t row_begin, int64_t row_end, int64_t row_stride,
                 int n_threads, double* raw, double* area, uint8_t* ray_log, int64_t* counters);

/* Duffy (src/DuffyKernel.jl:95-487) for one ordered pair.  bvh == NULL: no
 * occlusion; gpu_semantics 0: CPU is_visible on bvh; 1: GPU-path ray with group
 * skip on the single tree.  stype: -1 not Quad8/Quad8, 0 none, 1 vertex, 2 edge. */
int orc_singularity_type(const orc_mesh* m, int64_t i, int64_t j, int32_t* ci, int32_t* cj);
double orc_pair_duffy(const orc_mesh* m, const orc_bvh* bvh, int gpu_semantics, int geometric, int64_t i,
                      int64_t j, int nquad, double* Ai, int* stype);

/* src/Assembly.jl:102-225 (_compute_cpu), quadrature (use_duffy 0/1).  The
 * CPU path builds one BVH per active obstruction subset (src/Assembly.jl:121-143)
 * and uses is_visible / intersect_ray_bvh (t_min = 0).  Areas come from the
 * serial loop at src/Assembly.jl:186-190. */
int orc_solve_cpu(const orc_mesh* m, int nquad, int use_duffy, int self_vf,
                  const int32_t* obstruction_groups, int32_t n_obstruction_groups,
                  int64_t row_begin, int64_t row_end, int64_t row_stride, int n_threads,
                  double* raw, double* area, int64_t* counters);

/* src/Results.jl:56-82: groups given as sorted tags; F_group G x G col-major. */
void orc_aggregate(int64_t N, const double* F, const double* A, const int32_t* elem_group,
                   int32_t G, const int32_t* group_tags, double* F_group, double* A_group);
double orc_reciprocity_error(int64_t N, const double* F, const double* A);
void orc_row_sums(int64_t N, const double* F, double* out);

/* splitmix64 / xorshift64 stream helpers (src/GPUMCKernels.jl:37-50) */
uint64_t orc_init_rng(uint64_t seed, uint64_t thread_id);
double orc_xorshift64(uint64_t* state);

#ifdef __cplusplus
}
#endif
#endif
