// peaks.cu -- FP64 FMA throughput microbenchmark (the denominator for the
// FP64-bound R builder's roofline; the measured peaks file has none).
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/pofd_b200.h"
#include "common.cuh"

namespace {
// 8 independent FMA chains per thread; 2 flops per FMA.
__global__ void k_dfma(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
  double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
    x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 1.2345) out[0] = s;  // keep the chains alive
}
// Relative difference between the table exp2 and the library exp2 over
// n arguments spread over [lo, hi) (a stratified grid with a per-point
// offset), reduced to the maximum per block.
__global__ void k_exp2_check(int n, double lo, double hi, double* __restrict__ out) {
  __shared__ pofd::dev::Exp2Table e2;
  __shared__ double sh[32];
  e2.load();
  __syncthreads();
  double worst = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double u = (static_cast<double>(i) + 0.5 + 0.37 * sin(static_cast<double>(i))) /
                     static_cast<double>(n);
    const double x = lo + (hi - lo) * u;
    const double a = pofd::dev::exp2_tab(x, e2.t);
    const double b = exp2(x);
    const double d = (x < -1022.0) ? fabs(a) : fabs(a - b) / b;
    worst = fmax(worst, d);
  }
  worst = pofd::dev::block_max<256>(worst, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = worst;
}
}  // namespace

extern "C" int pofd_exp2_check(int device, int n, double lo, double hi, double* max_rel) {
  if (!max_rel || n <= 0 || !(lo < hi) || !(hi < 1023.0)) return POFD_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return POFD_E_CUDA;
  const int blocks = 592;
  double* d = nullptr;
  if (cudaMalloc(&d, blocks * sizeof(double)) != cudaSuccess) return POFD_E_NOMEM;
  k_exp2_check<<<blocks, 256>>>(n, lo, hi, d);
  double h[blocks];
  const cudaError_t e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return POFD_E_CUDA;
  double w = 0.0;
  for (double v : h) w = std::fmax(w, v);
  *max_rel = w;
  return POFD_OK;
}

extern "C" int pofd_fp64_peak(int device, double* tflops) {
  if (!tflops) return POFD_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return POFD_E_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return POFD_E_CUDA;
  double* d = nullptr;
  if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return POFD_E_NOMEM;
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 20000;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_dfma<<<blocks, threads>>>(d, 1000, 0.999999, 1e-7);  // warm
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    k_dfma<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (err != cudaSuccess) return POFD_E_CUDA;
  const double flops = 2.0 * 8.0 * iters * static_cast<double>(threads) * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return POFD_OK;
}
