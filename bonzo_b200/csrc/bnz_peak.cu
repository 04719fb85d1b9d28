// bnz_peak.cu -- the FP64 FMA throughput of the device, measured: the
// denominator of the kernels' FP64-pipe fraction (the HBM roofline's
// denominator is a measured copy bandwidth).  Eight independent FMA chains per
// thread keep the pipe busy; the result is written so nothing is elided.
// Also the check entry of the fast build's reciprocal (bnz_fastmath.cuh).
#include <cuda_runtime.h>

#include "bnz_fastmath.cuh"
#include "bnz_gpu.h"

namespace {

constexpr int PEAK_ITERS = 4096;
constexpr int PEAK_CHAINS = 8;

__global__ void k_fp64_fma(double* __restrict__ out, double a, double b) {
  double x[PEAK_CHAINS];
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; ++c) x[c] = 1e-3 * (threadIdx.x + c);
  for (int i = 0; i < PEAK_ITERS; ++i) {
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.;
#pragma unroll
  for (int c = 0; c < PEAK_CHAINS; ++c) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_nr_rcp(const double* __restrict__ x, double* __restrict__ y, int n) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) y[q] = bnz_nr_rcp(x[q]);
}

}  // namespace

extern "C" int bnz_fast_rcp(const double* x, double* y, int n, void* stream) {
  if (n < 0 || (n > 0 && (!x || !y))) return BNZ_ERR_ARG;
  if (n == 0) return BNZ_OK;
  const int threads = 256, blocks = (n + threads - 1) / threads < 4096 ? (n + threads - 1) / threads : 4096;
  k_nr_rcp<<<blocks, threads, 0, (cudaStream_t)stream>>>(x, y, n);
  return cudaGetLastError() == cudaSuccess ? BNZ_OK : BNZ_ERR_CUDA;
}

extern "C" int bnz_fp64_fma_peak(double* tflops) {
  if (!tflops) return BNZ_ERR_ARG;
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess)
    return BNZ_ERR_CUDA;
  const int threads = 256, blocks = nsm * 8;
  double* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = BNZ_OK;
  if (cudaMalloc((void**)&out, (size_t)threads * blocks * sizeof(double)) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = BNZ_ERR_CUDA;
  } else {
    float best = 0.f;
    for (int r = 0; r < 4 && rc == BNZ_OK; ++r) {  // the first run warms up
      cudaEventRecord(e0, 0);
      k_fp64_fma<<<blocks, threads>>>(out, 0.999999, 1e-7);
      cudaEventRecord(e1, 0);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        rc = BNZ_ERR_CUDA;
      else if (r > 0 && (best == 0.f || ms < best))
        best = ms;
    }
    if (rc == BNZ_OK) {
      const double flops = 2.0 * PEAK_CHAINS * PEAK_ITERS * (double)threads * blocks;
      *tflops = best > 0.f ? flops / (best * 1e-3) / 1e12 : 0.;
    }
  }
  if (out) cudaFree(out);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return rc;
}
