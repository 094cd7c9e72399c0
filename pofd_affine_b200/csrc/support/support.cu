// support.cu -- libpofd_b200_support.so: measurement and test helpers that
// are not part of the likelihood's C ABI (include/pofd_b200_support.h):
//   * pofd_fp64_peak   FP64 FMA throughput of a device, the denominator of
//                      the FP64-bound kernels' roofline (the measured peaks
//                      file carries HBM and BF16 figures only);
//   * pofd_exp2_check  the table-driven exp2 of the R builders against the
//                      CUDA library exp2;
//   * pofd_wait_check  the tensor-core kernels' bounded mbarrier wait running
//                      out and reporting it;
//   * pofd_gauss_*     a multivariate Gaussian target with the batched
//                      likelihood signature, for checking the sampler and
//                      the surrogate on a known posterior.
// None has a counterpart in the reference.
#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <new>

#include "../../../include/pofd_b200_support.h"
#include "../common.cuh"
#include "../umma.cuh"

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

// The tensor-core kernels' failure path without a fault: an mbarrier
// (arrival count 1) waited on with the kernels' bounded wait (limit
// try_wait rounds).  With arrive = 0 nothing ever arrives on it, and the
// timeout must come back as a status the host reads, with the kernel
// returning normally; with arrive = 1 thread 0 arrives first and the wait
// must succeed.  No tensor memory is allocated here.
__global__ void k_wait_check(unsigned limit, int arrive, int* __restrict__ out) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    pofd::umma::mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (arrive)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(pofd::umma::smem_u32(&bar))
                   : "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !pofd::umma::mbar_wait(&bar, 0u, limit)) atomicExch(&abort_flag, 1);
  __syncthreads();
  if (threadIdx.x == 0) out[0] = abort_flag;
}

constexpr unsigned kMaxDim = 64;

// log N(theta; mean, cov) up to a constant: -(1/2) d^T icov d, one thread per
// proposal; a NaN parameter gives POFD_E_INVALID_MODEL.
__global__ void k_gauss(unsigned nprop, unsigned npar, unsigned k,
                        const double* __restrict__ mean,
                        const double* __restrict__ icov,
                        const float* __restrict__ theta,
                        double* __restrict__ logl, int* __restrict__ status) {
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nprop) return;
  const float* x = theta + static_cast<size_t>(t) * npar;
  double d[kMaxDim];
  int st = POFD_OK;
  for (unsigned p = 0; p < k; ++p) {
    d[p] = static_cast<double>(x[p]) - mean[p];
    if (isnan(d[p])) st = POFD_E_INVALID_MODEL;
  }
  double q = 0.0;
  for (unsigned a = 0; a < k; ++a) {
    double r = 0.0;
    for (unsigned b = 0; b < k; ++b) r += icov[a * k + b] * d[b];
    q += d[a] * r;
  }
  logl[t] = (st == POFD_OK) ? -0.5 * q : __longlong_as_double(0x7ff8000000000000LL);
  status[t] = st;
}

}  // namespace

struct pofd_gauss {
  int device = 0;
  unsigned k = 0;
  double* mean = nullptr;
  double* icov = nullptr;
};

extern "C" {

int pofd_fp64_peak(int device, double* tflops) {
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

int pofd_exp2_check(int device, int n, double lo, double hi, double* max_rel) {
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

int pofd_wait_check(int device, unsigned limit, int arrive, int* timed_out) {
  if (!timed_out || limit == 0 || limit > (1u << 20) || (arrive != 0 && arrive != 1))
    return POFD_E_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return POFD_E_CUDA;
  int* d = nullptr;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return POFD_E_NOMEM;
  k_wait_check<<<1, 32>>>(limit, arrive, d);
  const cudaError_t e = cudaMemcpy(timed_out, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? POFD_OK : POFD_E_CUDA;
}

int pofd_gauss_create(int device, unsigned k, const double* mean, const double* icov,
                      pofd_gauss** out) {
  if (!mean || !icov || !out || k == 0 || k > kMaxDim) return POFD_E_ARG;
  if (device < 0 || cudaSetDevice(device) != cudaSuccess) return POFD_E_CUDA;
  std::unique_ptr<pofd_gauss> g(new (std::nothrow) pofd_gauss());
  if (!g) return POFD_E_NOMEM;
  g->device = device;
  g->k = k;
  if (cudaMalloc(&g->mean, k * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&g->icov, static_cast<size_t>(k) * k * sizeof(double)) != cudaSuccess) {
    cudaFree(g->mean);
    cudaFree(g->icov);
    return POFD_E_NOMEM;
  }
  if (cudaMemcpy(g->mean, mean, k * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(g->icov, icov, static_cast<size_t>(k) * k * sizeof(double),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(g->mean);
    cudaFree(g->icov);
    return POFD_E_CUDA;
  }
  *out = g.release();
  return POFD_OK;
}

int pofd_gauss_destroy(pofd_gauss* g) {
  if (!g) return POFD_OK;
  cudaSetDevice(g->device);
  cudaFree(g->mean);
  cudaFree(g->icov);
  delete g;
  return POFD_OK;
}

int pofd_gauss_eval_batch_device(void* gv, unsigned nprop, const float* theta, unsigned npar,
                                 double* logl, int* status, void* stream) {
  pofd_gauss* g = static_cast<pofd_gauss*>(gv);
  if (!g || !theta || !logl || !status) return POFD_E_ARG;
  if (npar < g->k) return POFD_E_ARG;
  if (nprop == 0) return POFD_OK;
  k_gauss<<<(nprop + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      nprop, npar, g->k, g->mean, g->icov, theta, logl, status);
  return cudaGetLastError() == cudaSuccess ? POFD_OK : POFD_E_CUDA;
}

}  // extern "C"
