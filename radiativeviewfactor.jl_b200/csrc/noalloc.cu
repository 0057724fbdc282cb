// noalloc.cu -- plain FP64 assembly for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: code running under an allocator that
// owns all device memory (a framework's caching pool, a memory-capped
// service), code that must not create allocations while other work is being
// captured or timed, or embedded hosts that hand this library pre-placed
// buffers only.  rvf_solve_fp64_noalloc serves them: the caller passes its
// inputs and outputs as device pointers, and the scratch the kernels need
// (quadrature tables, per-element data, counters) lives in one fixed
// file-scope __device__ array of kNoAllocScratchBytes (16 MiB).  Every GPU
// that loads this library holds that array until the process exits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/rvf_b200.h"
#include "kernels.h"
#include "rvf_internal.h"

namespace rvf {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device addresses of the scratch array, one per (device, context): a device
// reset or a new primary context can load the array at a new address, so the
// address is looked up again whenever the current context changes.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct ScratchAddr {
  void* ctx = nullptr;
  unsigned char* addr = nullptr;
};
ScratchAddr g_noalloc_addr[kMaxDevices];

// cuCtxGetCurrent through the runtime's driver entry-point table (no libcuda
// link); returns the current context handle, or null when it is unavailable.
void* current_context() {
  using Fn = int (*)(void**);
  static Fn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<Fn>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// True when p is device (or managed) memory that device `dev` owns.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free error of an unknown pointer
    return false;
  }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == dev;
}

// Largest mesh the array can hold: about 90 bytes of per-element data plus
// at least 1 quadrature point's table (56 bytes) per element.
constexpr int64_t kNoAllocMaxElems = (int64_t)(kNoAllocScratchBytes / 146);

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

// 1-based padded node table -> 0-based, with the range and family checks the
// host cannot do on device-resident input; bad input raises kErrBadInput and
// leaves a safe (0) node id behind.
__global__ void k_noalloc_nodes(const int32_t* __restrict__ en1, const int8_t* __restrict__ fam, int64_t N,
                                int64_t n_nodes, int mesh_dim, int32_t* __restrict__ en0, int* err) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N) return;
  const int f = fam[e];
  bool ok = f >= 0 && f <= 5 && ((mesh_dim == 2) == (f <= 3));
  const int nn = !ok ? 0 : f == 0 ? 8 : f == 1 ? 6 : f == 2 ? 4 : f == 3 ? 3 : f == 4 ? 3 : 2;
  for (int k = 0; k < 8; ++k) {
    int32_t v = 0;
    if (k < nn) {
      const int32_t id = en1[8 * e + k];
      if (id >= 1 && id <= n_nodes) v = id - 1;
      else ok = false;
    }
    en0[8 * e + k] = v;
  }
  if (!ok) atomicOr(err, kErrBadInput);
}

}  // namespace
}  // namespace rvf

using namespace rvf;

extern "C" int rvf_solve_fp64_noalloc(const double* coords, int64_t n_nodes, const int8_t* elem_family,
                                      const int32_t* elem_nodes, const int32_t* elem_group, int64_t n_elems,
                                      int32_t mesh_dim, int32_t nquad, double* F, double* A, void* stream) try {
  if (n_elems < 0 || n_nodes < 0) return set_err(RVF_EINVAL, "negative sizes");
  if (mesh_dim != 1 && mesh_dim != 2) return set_err(RVF_EINVAL, "mesh_dim must be 1 or 2, got %d", mesh_dim);
  if (nquad < 1) return set_err(RVF_EINVAL, "nquad must be >= 1, got %d", nquad);
  // surfaces: nquad^2 Gauss-Legendre points (at most kMaxPts = 64); curves: nquad points
  const int nq_max = mesh_dim == 2 ? 8 : kMaxPts;
  if (nquad > nq_max)
    return set_err(RVF_EUNSUPPORTED, "nquad=%d: at most %d is supported for mesh_dim %d", nquad, nq_max, mesh_dim);
  if (n_elems == 0) return RVF_OK;
  if (n_elems > kNoAllocMaxElems)
    return set_err(RVF_EINVAL,
                   "rvf_solve_fp64_noalloc: %lld elements exceed the fixed scratch array (%zu bytes, at most %lld "
                   "elements)",
                   (long long)n_elems, kNoAllocScratchBytes, (long long)kNoAllocMaxElems);
  if (!coords || !elem_family || !elem_nodes || !elem_group || !F || !A)
    return set_err(RVF_EINVAL, "null device pointer");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return set_err(RVF_ENODEV, "device ordinal %d out of range", dev);
  {
    const void* ptrs[6] = {coords, elem_family, elem_nodes, elem_group, F, A};
    const char* names[6] = {"coords", "elem_family", "elem_nodes", "elem_group", "F", "A"};
    for (int k = 0; k < 6; ++k)
      if (!on_device(ptrs[k], dev))
        return set_err(RVF_EINVAL, "rvf_solve_fp64_noalloc: %s is not device memory of the current device %d",
                       names[k], dev);
  }
  // once per device and context, with that device current
  void* ctx = current_context();
  ScratchAddr& sa = g_noalloc_addr[dev];
  if (!sa.addr || !ctx || sa.ctx != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetSymbolAddress(scratch)");
    sa.addr = static_cast<unsigned char*>(p);
    sa.ctx = ctx;
  }
  unsigned char* base = sa.addr;
  int sm_count = 0;
  if ((e = cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return cuda_err(e, "cudaDeviceGetAttribute");

  const int64_t N = n_elems;
  const Rule q = gl2d(nquad), t = tri_rule(nquad), l = line_rule(nquad);
  const int pmax = mesh_dim == 1 ? l.size() : std::max(q.size(), t.size());
  if (pmax > kMaxPts)
    return set_err(RVF_EUNSUPPORTED, "nquad=%d gives %d points per element; at most %d are supported", nquad, pmax,
                   kMaxPts);
  const int64_t nT = (N + kTile - 1) / kTile;
  std::vector<double> rules;
  for (const auto* v : {&q.xi, &q.eta, &q.w, &t.xi, &t.eta, &t.w, &l.xi, &l.w}) rules.insert(rules.end(), v->begin(), v->end());

  // scratch layout
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align256(bytes); return o; };
  const size_t o_ctl = take(256);  // err (int) | tile counter (u64) | counters (u64 x 4)
  const size_t o_rules = take(sizeof(double) * rules.size());
  const size_t o_en = take(sizeof(int32_t) * 8 * N);
  const size_t o_tab = take(sizeof(double) * nT * kComp * pmax * kTile);
  const size_t o_np = take(N);
  const size_t o_flat = take(N);
  const size_t o_nrm = take(sizeof(double) * 3 * N);
  const size_t o_cen = take(sizeof(double) * 3 * N);
  const size_t o_diam = take(sizeof(double) * N);
  if (off > kNoAllocScratchBytes)
    return set_err(RVF_EINVAL,
                   "rvf_solve_fp64_noalloc: %lld elements with %d points each need %zu bytes of scratch; the fixed "
                   "array holds %zu bytes",
                   (long long)N, pmax, off, kNoAllocScratchBytes);
  int* err = reinterpret_cast<int*>(base + o_ctl);
  unsigned long long* tile_counter = reinterpret_cast<unsigned long long*>(base + o_ctl + 64);
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(base + o_ctl + 128);
  int32_t* en0 = reinterpret_cast<int32_t*>(base + o_en);

  // the array keeps the previous call's contents: clear what must start at zero
  if ((e = cudaMemsetAsync(base + o_ctl, 0, 256, st)) != cudaSuccess) return cuda_err(e, "cudaMemsetAsync");
  if ((e = cudaMemsetAsync(base + o_tab, 0, sizeof(double) * nT * kComp * pmax * kTile, st)) != cudaSuccess)
    return cuda_err(e, "cudaMemsetAsync");
  if ((e = cudaMemcpyAsync(base + o_rules, rules.data(), sizeof(double) * rules.size(), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return cuda_err(e, "cudaMemcpyAsync(rules)");
  k_noalloc_nodes<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(elem_nodes, elem_family, N, n_nodes, mesh_dim, en0,
                                                                err);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "node table kernel");
  int herr = 0;
  if ((e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_err(e, "node table check");
  if (herr) return set_err(RVF_EINVAL, "rvf_solve_fp64_noalloc: a node id is outside 1..n_nodes or a family code is invalid");

  PrepArgs pa{};
  pa.N = N;
  pa.pmax = pmax;
  pa.coords = coords;
  pa.enodes = en0;
  pa.fam = elem_family;
  const double* r = reinterpret_cast<const double*>(base + o_rules);
  pa.qx = r; r += q.size(); pa.qe = r; r += q.size(); pa.qw = r; r += q.size();
  pa.tx = r; r += t.size(); pa.te = r; r += t.size(); pa.tw = r; r += t.size();
  pa.lx = r; r += l.size(); pa.lw = r;
  pa.nquadpts = q.size();
  pa.ntripts = t.size();
  pa.nline = l.size();
  pa.tab = reinterpret_cast<double*>(base + o_tab);
  pa.area = A;
  pa.np = reinterpret_cast<int8_t*>(base + o_np);
  pa.flat = reinterpret_cast<uint8_t*>(base + o_flat);
  pa.nrm = reinterpret_cast<double*>(base + o_nrm);
  pa.cen = reinterpret_cast<double*>(base + o_cen);
  pa.diam = reinterpret_cast<double*>(base + o_diam);
  pa.err = err;
  if ((e = launch_prep(pa, st)) != cudaSuccess) return cuda_err(e, "prep kernel launch");
  if (N == 1 && (e = cudaMemsetAsync(A, 0, sizeof(double), st)) != cudaSuccess) return cuda_err(e, "cudaMemsetAsync");

  PairArgs a{};
  a.N = N;
  a.nT = nT;
  a.n_tiles = nT * (nT + 1) / 2;
  a.pmax = pmax;
  a.dim3 = (mesh_dim == 2);
  a.tab = pa.tab;
  a.np = pa.np;
  a.area = A;
  a.flat = pa.flat;
  a.nrm = pa.nrm;
  a.group = elem_group;
  a.F = F;
  a.tile_counter = tile_counter;
  a.counters = counters;
  a.err = err;
  if ((e = launch_pairs_fp64(a, sm_count, st)) != cudaSuccess) return cuda_err(e, "pair kernel launch");
  if ((e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_err(e, "rvf_solve_fp64_noalloc kernels");
  if (herr & kErrWaitTimeout) return set_err(RVF_ETIMEDOUT, "a bounded device wait gave up");
  if (herr & kErrBadInput) return set_err(RVF_EINVAL, "mesh holds a degenerate element");
  return RVF_OK;
} catch (...) {
  return exception_status();
}
