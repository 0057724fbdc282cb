// kernels_mixed.cu -- mixed-precision pair integration (surface meshes).
//
// Far-field pairs (centroid distance >= near_field_factor x the larger element
// diameter) integrate in FP32 with FP32 per-pair accumulation; positions are
// FP32 offsets from an FP64 per-element anchor, so r = (anchor_j - anchor_i)
// + (off_q - off_p) keeps ~1e-7 relative accuracy.  FP64 is kept where
// stability needs it:
//   * near-field pairs: the whole pair runs the FP64 path of k_pairs_fp64;
//   * grazing point pairs (|cos| < 1e-5 in FP32): the reference's K in FP64;
//   * every shadow ray whose FP32 traversal met an uncertain decision (or
//     whose direction has a component below 1e-4): traced again in FP64 with
//     the reference's arithmetic, so every visibility decision is the
//     reference's (device_mixed.cuh);
//   * F = raw/A and the group / row reductions stay FP64.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_mixed.cuh"
#include "kernels.h"

namespace rvf {

// FP32 table: per point the offset from the element centroid, the normal and
// w*dA, tile-blocked like the FP64 table ([tile][7][pmax][32] floats).
__global__ void k_prep_f32(PrepF32Args a) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.N) return;
  const int64_t tile = e / kTile;
  const int lane = (int)(e % kTile);
  const double* src = a.tab + tile * kComp * a.pmax * kTile + lane;
  float* dst = a.tabf + tile * kComp * a.pmax * kTile + lane;
  const int np = a.np[e];
  const double c0 = a.cen[3 * e], c1 = a.cen[3 * e + 1], c2 = a.cen[3 * e + 2];
  for (int p = 0; p < np; ++p) {
    dst[(0 * a.pmax + p) * kTile] = (float)(src[(0 * a.pmax + p) * kTile] - c0);
    dst[(1 * a.pmax + p) * kTile] = (float)(src[(1 * a.pmax + p) * kTile] - c1);
    dst[(2 * a.pmax + p) * kTile] = (float)(src[(2 * a.pmax + p) * kTile] - c2);
    for (int c = 3; c < kComp; ++c) dst[(c * a.pmax + p) * kTile] = (float)src[(c * a.pmax + p) * kTile];
  }
}

cudaError_t launch_prep_f32(const PrepF32Args& a, cudaStream_t st) {
  if (a.N == 0) return cudaSuccess;
  k_prep_f32<<<(unsigned)((a.N + 127) / 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace rvf
