// kernels_util.cu -- device microbenchmark of the FMA pipes (the roofline
// denominator of the pair kernels, which are FP64 / FP32 FMA bound).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/rvf_b200.h"
#include "rvf_internal.h"

namespace rvf {

// 8 independent dependent-chains of fma per thread: enough ILP to fill the
// pipe at full occupancy.  The result is written so nothing is dead code.
template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters, T b, T c) {
  T a0 = (T)threadIdx.x, a1 = a0 + (T)1, a2 = a0 + (T)2, a3 = a0 + (T)3;
  T a4 = a0 + (T)4, a5 = a0 + (T)5, a6 = a0 + (T)6, a7 = a0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
      a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
  }
  T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == (T)-1.2345) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// max |a - b| over n doubles (NaN in exactly one of them counts as +inf);
// non-negative doubles order like their bit patterns, so atomicMax on the
// bits is a max on the values.
__global__ void k_max_abs_diff(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                               unsigned long long* out) {
  double m = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const double x = a[k], y = b[k];
    const bool nx = x != x, ny = y != y;
    double d = (nx && ny) ? 0.0 : (nx || ny) ? INFINITY : fabs(x - y);
    m = fmax(m, d);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

}  // namespace rvf

using namespace rvf;

extern "C" int rvf_max_abs_diff(const double* a, const double* b, int64_t n, double* out) {
  if (!out || n < 0 || (n > 0 && (!a || !b))) return set_err(RVF_EINVAL, "bad argument");
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_err(e, "cudaMalloc");
  cudaMemset(d, 0, sizeof(unsigned long long));
  if (n > 0) k_max_abs_diff<<<1184, 256>>>(a, b, n, d);
  unsigned long long h = 0;
  e = cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_err(e, "max_abs_diff");
  double v;
  std::memcpy(&v, &h, sizeof v);
  *out = v;
  return RVF_OK;
}

extern "C" int rvf_fma_peak(int32_t device, int32_t fp64, double* tflops) {
  if (!tflops) return set_err(RVF_EINVAL, "null out");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_err(e, "cudaSetDevice");
  cudaDeviceProp p;
  if ((e = cudaGetDeviceProperties(&p, device)) != cudaSuccess) return cuda_err(e, "cudaGetDeviceProperties");
  const int blocks = p.multiProcessorCount * 8, threads = 256;
  const int iters = fp64 ? 2048 : 8192;
  void* out = nullptr;
  if ((e = cudaMalloc(&out, sizeof(double) * blocks * threads)) != cudaSuccess) return cuda_err(e, "cudaMalloc");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(a);
    if (fp64) k_fma_peak<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
    else k_fma_peak<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0 && ms < best) best = ms;
  }
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_err(e, "fma peak kernel");
  const double flops = 2.0 * 64.0 * iters * (double)blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return RVF_OK;
}
