/*
 * rvf_b200.h -- C ABI of librvf_b200.so, the B200 backend for
 * RadiativeViewFactor.jl's element-pair view-factor assembly.
 *
 * The library replaces the GPU path behind compute_view_factors(mesh; ...)
 * (src/Assembly.jl:64-96): everything below the GPU hook _GPU_HOOK_REF
 * (src/Assembly.jl:241-252) -- compute_view_factors_gpu (src/GPUAssembly.jl:32-105),
 * the pair kernel (src/GPUKernels.jl:226-323), the flat BVH and its traversal
 * (src/GPUBVH.jl:99-285), the Monte Carlo kernel (src/GPUMCKernels.jl:146-328)
 * and, as a device path the reference lacks, the Duffy integrals
 * (src/DuffyKernel.jl:452-487).
 *
 * Conventions
 *   - Every entry point returns an int status (RVF_OK == 0, negative on error)
 *     and never aborts or throws; rvf_last_error() gives the message of the
 *     last failure on the calling thread.
 *   - Matrices are column-major like Julia's (element (i,j) of an N x N matrix
 *     at i + j*N, 0-based); F[i,j] is the view factor from element i to j.
 *   - Node ids inside the node tables are 1-based, exactly as
 *     build_gpu_arrays (src/GPUKernels.jl:336-412) produces them.
 *   - One session drives one GPU.  Calls on one session are serialised by an
 *     internal mutex; results are written before rvf_solve returns
 *     (synchronous, like KernelAbstractions.synchronize at src/GPUKernels.jl:498).
 */
#ifndef RVF_B200_H
#define RVF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RVF_ABI_VERSION 2

/* status codes */
#define RVF_OK 0
#define RVF_EINVAL (-1)       /* malformed argument / mesh (bad node id, zero-area element, ...) */
#define RVF_ENOMEM (-2)       /* device or pinned host allocation failed */
#define RVF_EBUDGET (-3)      /* request exceeds the session's HBM budget */
#define RVF_ECUDA (-4)        /* CUDA runtime error */
#define RVF_ETIMEDOUT (-5)    /* a bounded device wait gave up, or rvf_wait timed out */
#define RVF_ECANCELED (-6)    /* request cancelled */
#define RVF_EUNSUPPORTED (-7) /* option combination not implemented */
#define RVF_ENODEV (-8)       /* no usable sm_100 device */
#define RVF_EBUSY (-9)        /* result not ready yet (rvf_poll) */
#define RVF_ECLOSED (-10)     /* serving queue closed */
#define RVF_EINTERNAL (-11)   /* unexpected internal error (no C++ exception crosses this interface) */

/* element family codes: src/GPUKernels.jl:344 (0..3), extended with curves */
#define RVF_QUAD8 0
#define RVF_TRI6 1
#define RVF_QUAD4 2
#define RVF_TRI3 3
#define RVF_LINE3 4
#define RVF_LINE2 5

#define RVF_METHOD_QUADRATURE 0
#define RVF_METHOD_MONTE_CARLO 1

#define RVF_PREC_FP64 0  /* everything in FP64 (the plain path) */
#define RVF_PREC_MIXED 1 /* FP32 far field and traversal, FP64 where stability needs it */

typedef struct rvf_session rvf_session;
typedef struct rvf_mesh rvf_mesh;
typedef struct rvf_request rvf_request;

typedef struct {
  int32_t device;             /* CUDA ordinal (default 0) */
  uint64_t hbm_budget_bytes;  /* 0 = 90% of the device's free memory at creation */
  int32_t n_host_threads;     /* host staging threads (0 = hardware concurrency) */
  int32_t reserved[8];
} rvf_session_opts;

/* Mesh, laid out as build_gpu_arrays (src/GPUKernels.jl:336-412) flattens
 * MeshData, plus the merged obstruction soup of build_flat_bvh_from_mesh
 * (src/GPUBVH.jl:146-174) and the sorted group tags of _aggregate
 * (src/Results.jl:59).  The library copies everything it needs; the caller
 * keeps ownership of these buffers. */
typedef struct {
  int32_t mesh_dim;             /* 2 = surface mesh (3-D view factors), 1 = curve mesh (2-D, per unit depth) */
  int64_t n_nodes;
  const double* coords;         /* 3 x n_nodes, column-major */
  int64_t n_elems;
  const int8_t* elem_family;    /* RVF_QUAD8 ... RVF_LINE2 */
  const int32_t* elem_node_idx; /* 1-based column of the element in its family's node table */
  const int32_t* elem_group;    /* physical group tag */
  const int32_t* nodes[6];      /* per family: k x n_family[f] column-major, 1-based node ids (k = 8,6,4,3,3,2) */
  int64_t n_family[6];
  int64_t n_obs;                /* obstruction primitives (0 = no obstruction) */
  int32_t obs_nv;               /* 3 = triangle soup, 2 = segment soup */
  const double* obs_soup;       /* soup[c + 3*(v + obs_nv*t)], the layout of src/MeshIO.jl:648-685 */
  const int32_t* obs_group;     /* group tag per primitive, pre-permutation */
  int32_t n_groups;             /* number of sorted group tags (F_group is n_groups^2) */
  const int32_t* group_tags;    /* sorted ascending */
} rvf_mesh_desc;

typedef struct {
  int32_t nquad;              /* Gauss points per direction / Dunavant selector (src/GPUKernels.jl:388-393) */
  int32_t method;             /* RVF_METHOD_* */
  int32_t use_duffy;          /* Sauter-Schwab integrals for Quad8 pairs sharing corners */
  int32_t n_samples;          /* Monte Carlo samples per pair */
  uint64_t seed;              /* Monte Carlo seed (the reference draws rand(UInt64), src/GPUAssembly.jl:72) */
  int32_t precision;          /* RVF_PREC_* */
  int32_t occlusion;          /* 1: cast shadow rays against the mesh's obstruction soup */
  int32_t geometric_soup;     /* 0: read soup triangles as the reference does (parity); 1: true vertices */
  int32_t mc_exclude_groups;  /* MC: 0 passes group tags 0/0 like src/GPUMCKernels.jl:164; 1 skips src/dst groups */
  double near_field_factor;   /* mixed: centroid distance < factor * max diameter runs in FP64 (default 2) */
  uint8_t* ray_log;           /* debug: host buffer of n_elems^2 * ray_log_pm^2 bytes, or NULL */
  int32_t ray_log_pm;         /* stride of the ray log (>= points per element) */
  int32_t disable_pair_lists; /* 3-D occlusion: 1 = every ray walks the tree (same results; for testing) */
  int32_t self_vf;            /* 1: also integrate the pairs (i, i) -- concave elements see themselves
                                 (src/Assembly.jl:173,193, j_start = self_vf ? i : i + 1); quadrature only */
  int32_t disable_tile_cull;  /* 1: no tile classification -- every shadow ray goes through the ray pipeline
                                 and every tile through its generation loop (same view factors; for testing) */
  int32_t fault_inject;       /* test hooks, 0 in production: RVF_FAULT_* bits */
  int32_t fast_points;        /* quadrature-only tiles: destination points per lane block -- 0 = by the
                                 rule's size; FP64 2..4, mixed 2, 3, 4, 5, 7 or 8 (same view factors) */
  int32_t fast_row_groups;    /* quadrature-only tiles: warp tasks per tile, 1 (whole tile), 2, 4, 8 or 32
                                 (one row each); 0 = enough tasks for four per resident warp */
  int32_t reserved[2];
} rvf_options;

/* fault_inject bits (failure-path tests; each injects one host-visible failure
 * and leaves the session usable for the next call) */
#define RVF_FAULT_CLAIM 1 /* the pair pipeline's tile claims get no retries: every claim gives up -> RVF_ETIMEDOUT */
#define RVF_FAULT_ALLOC 2 /* the first device allocation of this call fails -> RVF_ENOMEM */

typedef struct {
  double ms_upload;       /* host->device of the mesh description */
  double ms_prep;         /* quadrature tables, areas, BVH upload */
  double ms_pairs;        /* pair integration (+ occlusion) */
  double ms_duffy;        /* singular pairs */
  double ms_reduce;       /* group aggregation and row sums */
  double ms_download;     /* device->host of the results */
  double ms_total;
  int64_t n_pairs;        /* unordered element pairs integrated */
  int64_t n_point_pairs;  /* quadrature / sample point pairs evaluated */
  int64_t n_rays;         /* shadow rays cast */
  int64_t n_rays_fp64;    /* rays traced in FP64 (all of them in FP64 mode; re-tests in mixed mode) */
  int64_t n_pairs_fp64;   /* mixed mode: pairs integrated in FP64 (near field / grazing) */
  int64_t n_duffy_pairs;  /* vertex- or edge-sharing Quad8 pairs */
  double max_row_sum_dev; /* max_i |sum_j F_ij - 1| */
  int64_t n_node_visits;  /* BVH box tests, as executed */
  int64_t n_prim_tests;   /* ray-primitive tests, as executed */
  int64_t n_kernels;      /* kernels of this library launched by the call */
  int64_t n_graze_fp64;   /* mixed: grazing point pairs evaluated in FP64 */
  int64_t n_unsure_rays;  /* mixed: FP32 rays with an uncertain decision (traced again in FP64) */
  int64_t n_unsure_slab;  /* ... uncertain at a box test */
  int64_t n_unsure_prim;  /* ... uncertain at a triangle test */
  int64_t n_unsure_dir;   /* mixed: rays with a direction component below 1e-4 (FP64 from the start) */
  int64_t n_rays_traced;  /* rays that passed the root box and went through the traversal queues */
  int64_t n_chunks;       /* queue refills of the pair pipeline */
  double ms_gen;          /* pair pipeline phases (CUDA events on the solve stream, summed over chunks): */
  double ms_trace;        /*   traversal (FP32 in mixed mode) */
  double ms_trace_fp64;   /*   mixed mode: FP64 traversal of the uncertain and FP64 rays */
  double ms_resolve;      /*   visible terms of the traced rays */
  int64_t n_list_pairs;   /* 3-D occlusion: pending pairs whose rays test a per-pair triangle list */
  int64_t n_walk_pairs;   /*   ... whose list overflowed (their rays walk the tree) */
  double ms_lists;        /*   building the per-pair lists (part of ms_trace) */
  int64_t n_tiles_culled; /* 3-D occlusion: tiles none of whose shadow rays can be blocked (no ray work) */
  int64_t n_pairs_masked; /*   pairs whose rays may be blocked (the only ones through the ray pipeline) */
  double ms_cull;         /* tile classification before the pair pipeline */
  int64_t n_tiles_unclassified; /* tiles whose walk overflowed its frontier or lists (every pair keeps its rays) */
  int64_t reserved[1];
} rvf_stats;

const char* rvf_version(void);
int rvf_abi_version(void);
int rvf_last_error(char* buf, size_t n);
void rvf_default_options(rvf_options* o);

/* session: replaces the CUDABackend / CuArray registration of
 * ext/RadiativeViewFactorCUDAExt.jl:11-12 (device selection, Float64). */
int rvf_session_create(const rvf_session_opts* opts, rvf_session** out);
int rvf_session_destroy(rvf_session* s);
int rvf_device_info(rvf_session* s, int* sm_count, uint64_t* hbm_total, uint64_t* hbm_free);

/* mesh upload: build_gpu_arrays (src/GPUKernels.jl:336-412) +
 * build_flat_bvh_from_mesh (src/GPUBVH.jl:146-174). */
int rvf_mesh_upload(rvf_session* s, const rvf_mesh_desc* d, rvf_mesh** out);
int rvf_mesh_release(rvf_session* s, rvf_mesh* m);
int rvf_mesh_n_elems(const rvf_mesh* m, int64_t* n);

/* Solve: compute_view_factors_gpu (src/GPUAssembly.jl:32-105).
 * F_elem (N*N), A_elem (N), F_group (G*G), A_group (G), row_sums (N) are
 * caller-owned host buffers or NULL.  The element matrix also stays on the
 * device until the next solve on this mesh (rvf_result_copy). */
int rvf_solve(rvf_session* s, rvf_mesh* m, const rvf_options* o, double* F_elem, double* A_elem,
              double* F_group, double* A_group, double* row_sums, rvf_stats* st);
int rvf_result_copy(rvf_session* s, rvf_mesh* m, double* F_elem, double* A_elem);
/* Device address of the element matrix of the last solve (column-major N*N). */
int rvf_result_device(rvf_mesh* m, const double** F_dev, const double** A_dev);

/* pinned host memory for result buffers (faster device->host copies) */
int rvf_host_alloc(size_t bytes, void** p);
int rvf_host_free(void* p);

/* quadrature rule tables used by the device (for cross-checks) */
int rvf_quadrature_rule(int32_t family, int32_t nquad, double* pts, double* wts, int32_t* n_pts);

/* Measured FMA throughput of the device (fp64 = 1: FP64, 0: FP32) in TFLOP/s:
 * the denominator of the pair kernels' roofline (they are FMA-pipe bound). */
int rvf_fma_peak(int32_t device, int32_t fp64, double* tflops);

/* max |a - b| over n device doubles (for example two results of
 * rvf_result_device: the mixed-precision F against the FP64 F). */
int rvf_max_abs_diff(const double* a_dev, const double* b_dev, int64_t n, double* out);

/* ---------------------------------------------------------------------------
 * Serving: continuous batching of solves (the request loop a Julia service
 * would run around _gpu_compute_hook, src/Assembly.jl:241-260; the
 * reference itself solves one mesh per call, synchronously).
 *
 * rvf_submit copies the mesh and options and returns at once.  A worker
 * thread admits requests in arrival order while their device footprint
 * (F matrix, quadrature tables, BVH) fits the admission budget, keeps each
 * admitted mesh's geometry, BVH and F on the device, and feeds every
 * admitted quadrature request of one launch class (precision, surface or
 * curve, occlusion) to the same batched launches: each chunk's generation
 * kernel drains one device-side queue of tiles drawn from all of them, so
 * requests that arrive while others run join at the next chunk and their work
 * overlaps on the device.  Launches of a class replay a CUDA graph captured
 * for its shape; the grid sizes are chosen by a short autotuning sweep on the
 * first chunks of the class.  Monte Carlo requests run one at a time between
 * chunks.  Results stay on the device until rvf_request_result copies them;
 * rvf_release frees them and the admission budget.  Every request's result
 * is bit-identical to rvf_solve of the same mesh and options.
 * The server drives the session's stream: do not call rvf_solve on the same
 * session while a server exists on it.
 * ------------------------------------------------------------------------- */
typedef struct rvf_server rvf_server;

#define RVF_REQ_QUEUED 0
#define RVF_REQ_RUNNING 1
#define RVF_REQ_DONE 2
#define RVF_REQ_FAILED 3
#define RVF_REQ_CANCELED 4

typedef struct {
  uint64_t admit_bytes;  /* admission budget for the admitted requests' footprints (0 = 70% of the session budget) */
  int32_t max_batch;     /* requests per batched launch, 1..64 (0 = 64) */
  int32_t use_graphs;    /* 0 or 1: replay a CUDA graph per launch shape; -1: eager launches */
  int32_t autotune;      /* >= 0: sweep launch shapes -- the chunk grids on the first chunks of each launch
                            class, the quadrature-only kernel's shape on the first admissions of each launch
                            class and size class -- and keep the fastest; -1: default shapes */
  int32_t reserved[8];
} rvf_server_opts;

typedef struct {
  int32_t state;             /* RVF_REQ_* */
  int32_t status;            /* RVF_OK, or the error of a failed request */
  int64_t n_elems;
  uint64_t footprint_bytes;  /* device memory charged to the admission budget */
  double t_submit_ms;        /* since the server was created */
  double t_admit_ms;
  double t_done_ms;
  int64_t n_chunks;          /* batched chunks the request took part in */
  int32_t reserved[8];
} rvf_request_info;

/* A launch shape the server's autotuner chose for one launch class (precision,
 * occlusion, surface or curve mesh, points per element) and size class of
 * requests.  The quadrature-only kernel's candidates all run on the class's
 * first request (each forms the same F), and the fastest is kept. */
typedef struct {
  int32_t mixed, occlusion, dim3;
  int32_t size_class;              /* requests with 4^k <= quadrature-only tiles < 4^(k+1) */
  int32_t gen_blocks_per_sm;       /* chunked generation grid (0: occupancy default; chunk sweep) */
  int32_t trace_blocks_per_sm;     /* traversal grid (0: occupancy default; chunk sweep) */
  int32_t fast_points;             /* quadrature-only kernel: destination points per lane block */
  int32_t fast_row_groups;         /*   and warp tasks per tile */
  int32_t rule_points;             /* quadrature points per element of the class's rule */
  int32_t reserved;
  double fast_ms_per_gpp;          /* its measured time per 1e9 point pairs */
  double fast_ms_per_gpp_default;  /*   and the default shape's (points by the rule, 1 task per tile) */
} rvf_tuned_shape;

typedef struct {
  int64_t submitted, completed, failed, canceled, in_flight;
  double p50_ms, p99_ms, mean_ms;  /* latency submit -> done of the completed requests */
  double wall_ms;                  /* first submit -> last completion */
  int64_t pairs_done;              /* element pairs of the completed requests */
  int64_t chunks;                  /* batched launches */
  int64_t graph_replays;
  int64_t batched_requests;        /* sum over chunks of the requests in the chunk */
  uint64_t admitted_bytes_peak;
  int32_t n_tuned;                 /* entries of tuned[] in use */
  int32_t reserved;
  double ms_admit;                 /* worker time: admissions (upload, tables, classes, quadrature-only tiles) */
  double ms_quad_chunks;           /*   batched quadrature chunks (with the tail of the requests they finish) */
  double ms_mc_chunks;             /*   Monte Carlo chunks */
  double ms_free;                  /*   freeing released requests' device memory */
  double ms_idle;                  /*   waiting for work (nothing admissible, nothing running) */
  rvf_tuned_shape tuned[8];        /* the autotuner's choices, kept by the session for all its servers (the
                                      last 8 classes it finished) */
} rvf_server_stats;

int rvf_server_create(rvf_session* s, const rvf_server_opts* o, rvf_server** out);
/* Cancels the queued requests, finishes the running chunk, frees everything. */
int rvf_server_destroy(rvf_server* sv);
/* ray_log is not supported here (RVF_EINVAL). */
int rvf_submit(rvf_server* sv, const rvf_mesh_desc* d, const rvf_options* o, int64_t* id);
/* RVF_OK when done, RVF_EBUSY while queued or running, the request's error
 * when it failed, RVF_ECANCELED when cancelled; info may be NULL. */
int rvf_poll(rvf_server* sv, int64_t id, rvf_request_info* info);
/* As rvf_poll, waiting up to timeout_ms (< 0: no limit); RVF_ETIMEDOUT when
 * the request is still queued or running at the limit. */
int rvf_wait(rvf_server* sv, int64_t id, int64_t timeout_ms, rvf_request_info* info);
/* Waits up to timeout_ms (< 0: no limit) for any request to finish (done,
 * failed or cancelled) that no earlier rvf_wait_any returned, in the order
 * they finished, and stores its id; RVF_ETIMEDOUT when none did.  A client
 * collecting results as they complete needs no polling loop. */
int rvf_wait_any(rvf_server* sv, int64_t timeout_ms, int64_t* id);
int rvf_cancel(rvf_server* sv, int64_t id);
/* Host copies of a done request's result (any pointer may be NULL). */
int rvf_request_result(rvf_server* sv, int64_t id, double* F_elem, double* A_elem, double* F_group,
                       double* A_group, double* row_sums);
/* Device addresses of a done request's F (n_elems^2, column-major) and A,
 * valid until rvf_release: for callers that read the result on the GPU. */
int rvf_request_result_device(rvf_server* sv, int64_t id, const double** F_dev, const double** A_dev);
/* Drops a finished request: its admission charge at once, its device memory
 * when the server's worker next looks for work (the caller does not wait
 * for a running chunk). */
int rvf_release(rvf_server* sv, int64_t id);
int rvf_server_stats_get(rvf_server* sv, rvf_server_stats* st);

/* Plain FP64 assembly that allocates no memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- code under an
 * allocator that owns all device memory, memory-capped services, hosts that
 * hand the library pre-placed buffers only.  Inputs and outputs are the
 * caller's device pointers, all on the current device (each is checked with
 * cudaPointerGetAttributes; host memory or another device's buffer is
 * RVF_EINVAL): coords (3 x n_nodes column-major), elem_family
 * (RVF_QUAD8..RVF_LINE2), elem_nodes (n_elems x 8 element-major, 1-based node
 * ids, zero padded), elem_group; outputs F (n_elems^2 column-major, F[i,j] =
 * raw/A_i as rvf_solve) and A (n_elems).  No obstruction, no group sums.
 * Scratch lives in one fixed 16 MiB __device__ array inside the library
 * (held by every GPU that loads the library until exit); a mesh whose tables
 * need more (about 90 B per element + 1792 B per 32 elements per quadrature
 * point; at most 114,900 elements) is rejected with RVF_EINVAL, and nquad
 * above 8 (surfaces) or 64 (curves) with RVF_EUNSUPPORTED.  The first call on
 * a device (and again after the device's context changes, e.g. after
 * cudaDeviceReset) looks up that array's device address, so make it before
 * any stream capture.  Calls
 * share the array; they take a process-wide lock and synchronise `stream`
 * (a cudaStream_t, NULL = legacy default stream) before returning, because
 * calls that overlapped on the GPU would race on it. */
int rvf_solve_fp64_noalloc(const double* coords, int64_t n_nodes, const int8_t* elem_family,
                           const int32_t* elem_nodes, const int32_t* elem_group, int64_t n_elems, int32_t mesh_dim,
                           int32_t nquad, double* F, double* A, void* stream);

/* Host-side BVH build of rvf_mesh_upload (build_bvh, src/BVH.jl:71-148, plus
 * the miss links of src/GPUBVH.jl:69-82), exported for cross-checks; needs no
 * GPU.  Call with lo == NULL to get the node count in *n_nodes; then lo/hi
 * (3*M), meta (5*M: left,right,tri_start,tri_count,miss, 1-based as
 * src/GPUBVH.jl:48-55) and tri_idx (n_prims, 1-based) are filled. */
int rvf_bvh_build_host(const double* soup, int32_t nv, int64_t n_prims, double* lo, double* hi, int32_t* meta,
                       int32_t* tri_idx, int64_t* n_nodes);

#ifdef __cplusplus
}
#endif
#endif
