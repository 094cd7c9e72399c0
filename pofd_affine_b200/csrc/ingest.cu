// ingest.cu -- data-map ingestion on the GPU: mean subtraction and binning
// of 1D and two-band maps already in device memory (fitsData::meanSubtract
// and applyBinning, fitsData.cc:393-437; fitsDataDouble.cc:557-608).
//
// The results equal the host set-up's (setup.cc) bit for bit:
//   * the mean is the reference's sequential sum in pixel order (one block
//     stages the data through shared memory and one thread adds it in
//     order), divided by the pixel count; each pixel is then v - mean;
//   * the minimum and maximum are exact (order free);
//   * bin indices are (unsigned)((v - bincent0) * (1/bindelta) + 0.5) with
//     every operation rounded separately, as the host evaluates them (no
//     fused multiply-add), and the counts are integers (atomic adds).
// The sequential mean dominates (a dependent chain of one add per pixel);
// the rest is a few passes over the map.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <sstream>
#include <vector>

#include "../../include/pofd_b200.h"
#include "common.cuh"
#include "setup.hh"

namespace pofd {

namespace {

constexpr int INT = 256;       // threads per block
constexpr int STAGE = 2048;    // values staged per round of the sequential sum

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << what << ": " << cudaGetErrorString(e);
    throw Error(e == cudaErrorMemoryAllocation ? POFD_E_NOMEM : POFD_E_CUDA, s.str());
  }
}

// out[b] = (x_b[0] + x_b[1] + ... + x_b[n-1]) / n, added in index order
// (the rounding of the host set-up's sequential sum); block b takes array b
// (xa, or xb for a second band).  The adds form one dependent chain, so one
// thread does them, from registers eight values at a time, while warps
// 1 .. 7 stage the next STAGE values into the other half of a double buffer.
__global__ void __launch_bounds__(INT) k_seqmean(const double* __restrict__ xa,
                                                 const double* __restrict__ xb, size_t n,
                                                 double* __restrict__ out) {
  __shared__ double buf[2][STAGE];
  const double* __restrict__ x = blockIdx.x ? xb : xa;
  const size_t nst = (n + STAGE - 1) / STAGE;
  for (int i = threadIdx.x; i < static_cast<int>(min(static_cast<size_t>(STAGE), n)); i += INT)
    buf[0][i] = x[i];
  __syncthreads();
  double s = 0.0;
  for (size_t k = 0; k < nst; ++k) {
    const size_t base = k * STAGE;
    if (threadIdx.x >= 32) {
      const size_t nb = base + STAGE;
      if (nb < n) {
        const int m2 = static_cast<int>(min(static_cast<size_t>(STAGE), n - nb));
        double* d = buf[(k + 1) & 1];
        for (int i = threadIdx.x - 32; i < m2; i += INT - 32) d[i] = x[nb + i];
      }
    } else if (threadIdx.x == 0) {
      const int m = static_cast<int>(min(static_cast<size_t>(STAGE), n - base));
      const double* b = buf[k & 1];
      int i = 0;
      if (k == 0) s = b[i++];
      for (; i + 8 <= m; i += 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = b[i + q];
#pragma unroll
        for (int q = 0; q < 8; ++q) s = __dadd_rn(s, v[q]);
      }
      for (; i < m; ++i) s = __dadd_rn(s, b[i]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = __ddiv_rn(s, static_cast<double>(n));
}

__global__ void k_subtract(double* __restrict__ x, size_t n, const double* __restrict__ m) {
  const double mv = *m;
  for (size_t i = blockIdx.x * static_cast<size_t>(INT) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * INT)
    x[i] = __dsub_rn(x[i], mv);
}

// Per-block minimum and maximum.
__global__ void __launch_bounds__(INT) k_minmax(const double* __restrict__ x, size_t n,
                                                double* __restrict__ part) {
  __shared__ double slo[INT], shi[INT];
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (size_t i = blockIdx.x * static_cast<size_t>(INT) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * INT) {
    const double v = x[i];
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  slo[threadIdx.x] = lo;
  shi[threadIdx.x] = hi;
  __syncthreads();
  for (int o = INT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      slo[threadIdx.x] = fmin(slo[threadIdx.x], slo[threadIdx.x + o]);
      shi[threadIdx.x] = fmax(shi[threadIdx.x], shi[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = slo[0];
    part[2 * blockIdx.x + 1] = shi[0];
  }
}

__device__ __forceinline__ unsigned bin_index(double v, double bc0, double ib) {
  return static_cast<unsigned>(__dadd_rn(__dmul_rn(__dsub_rn(v, bc0), ib), 0.5));
}

// 1D counts, privatised per block in shared memory (nb <= kMaxSharedBins).
constexpr unsigned kMaxSharedBins = 8192;
__global__ void __launch_bounds__(INT) k_bin1(const double* __restrict__ x, size_t n, double bc0,
                                              double ib, unsigned nb, unsigned* __restrict__ bins) {
  extern __shared__ unsigned sb[];
  for (unsigned i = threadIdx.x; i < nb; i += INT) sb[i] = 0u;
  __syncthreads();
  for (size_t i = blockIdx.x * static_cast<size_t>(INT) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * INT) {
    const unsigned b = bin_index(x[i], bc0, ib);
    if (b < nb) atomicAdd(&sb[b], 1u);
  }
  __syncthreads();
  for (unsigned i = threadIdx.x; i < nb; i += INT)
    if (sb[i]) atomicAdd(&bins[i], sb[i]);
}

// 1D counts straight into global memory (nb > kMaxSharedBins).
__global__ void k_bin1g(const double* __restrict__ x, size_t n, double bc0, double ib, unsigned nb,
                        unsigned* __restrict__ bins) {
  for (size_t i = blockIdx.x * static_cast<size_t>(INT) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * INT) {
    const unsigned b = bin_index(x[i], bc0, ib);
    if (b < nb) atomicAdd(&bins[b], 1u);
  }
}

// Two-band counts [nb1][nb2] in global memory.
__global__ void k_bin2(const double* __restrict__ x1, const double* __restrict__ x2, size_t n,
                       double bc1, double ib1, unsigned nb1, double bc2, double ib2, unsigned nb2,
                       unsigned* __restrict__ bins) {
  for (size_t i = blockIdx.x * static_cast<size_t>(INT) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * INT) {
    const unsigned a = bin_index(x1[i], bc1, ib1), b = bin_index(x2[i], bc2, ib2);
    if (a < nb1 && b < nb2) atomicAdd(&bins[static_cast<size_t>(a) * nb2 + b], 1u);
  }
}

int grid_for(size_t n, int sms) {
  const size_t g = (n + INT - 1) / INT;
  return static_cast<int>(std::min<size_t>(g, static_cast<size_t>(sms) * 8));
}

// min and max of x[0..n) (device) to the host
void minmax(const double* x, size_t n, int sms, double* part, double* lo, double* hi,
            cudaStream_t st) {
  const int g = grid_for(n, sms);
  k_minmax<<<g, INT, 0, st>>>(x, n, part);
  ck(cudaGetLastError(), "k_minmax");
  std::vector<double> h(2 * static_cast<size_t>(g));
  ck(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
  ck(cudaStreamSynchronize(st), "synchronize");
  *lo = h[0];
  *hi = h[1];
  for (int b = 1; b < g; ++b) {
    *lo = std::fmin(*lo, h[2 * b]);
    *hi = std::fmax(*hi, h[2 * b + 1]);
  }
}

// bincent0 and bindelta as Data1::applyBinning forms them
void bin_axis(double lo, double hi, unsigned nb, double* bc, double* bd) {
  *bc = lo;
  *bd = (nb == 1) ? 2 * (hi - lo) : (hi - lo) / static_cast<double>(nb - 1);
}

}  // namespace

// Mean subtraction (optional) and binning of n values in device memory x
// (modified in place when meansub); bins (device, nb) receive the counts;
// info3 = {mean (0 without meansub), bincent0, bindelta}.
void ingest_bin1(double* x, size_t n, bool meansub, unsigned nb, unsigned* bins, double* info3,
                 void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) throw Error(POFD_E_ARG, "No pixels in data");
  if (nb == 0) throw Error(POFD_E_ARG, "Trying to bin with no bins");
  int dev = 0, sms = 148;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
  double* scratch = nullptr;
  ck(cudaMallocAsync(&scratch, (2 * static_cast<size_t>(sms) * 8 + 1) * sizeof(double), st),
     "cudaMallocAsync");
  double mean = 0.0;
  if (meansub) {
    k_seqmean<<<1, INT, 0, st>>>(x, x, n, scratch);
    k_subtract<<<grid_for(n, sms), INT, 0, st>>>(x, n, scratch);
    ck(cudaGetLastError(), "mean subtraction");
    ck(cudaMemcpyAsync(&mean, scratch, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
  }
  double lo, hi;
  minmax(x, n, sms, scratch + 1, &lo, &hi, st);
  double bc, bd;
  bin_axis(lo, hi, nb, &bc, &bd);
  const double ib = 1.0 / bd;
  ck(cudaMemsetAsync(bins, 0, nb * sizeof(unsigned), st), "memset");
  if (nb <= kMaxSharedBins)
    k_bin1<<<grid_for(n, sms), INT, nb * sizeof(unsigned), st>>>(x, n, bc, ib, nb, bins);
  else
    k_bin1g<<<grid_for(n, sms), INT, 0, st>>>(x, n, bc, ib, nb, bins);
  ck(cudaGetLastError(), "binning");
  ck(cudaFreeAsync(scratch, st), "cudaFreeAsync");
  ck(cudaStreamSynchronize(st), "synchronize");
  info3[0] = mean;
  info3[1] = bc;
  info3[2] = bd;
}

// The two-band form (Data2::meanSubtract / applyBinning): counts [nb1][nb2];
// info6 = {mean1, mean2, bincent01, bindelta1, bincent02, bindelta2}.
void ingest_bin2(double* x1, double* x2, size_t n, bool meansub, unsigned nb1, unsigned nb2,
                 unsigned* bins, double* info6, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) throw Error(POFD_E_ARG, "No pixels in data");
  if (nb1 == 0 || nb2 == 0) throw Error(POFD_E_ARG, "Trying to bin with no bins");
  int dev = 0, sms = 148;
  ck(cudaGetDevice(&dev), "cudaGetDevice");
  ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
  double* scratch = nullptr;
  ck(cudaMallocAsync(&scratch, (2 * static_cast<size_t>(sms) * 8 + 2) * sizeof(double), st),
     "cudaMallocAsync");
  double means[2] = {0.0, 0.0};
  if (meansub) {
    k_seqmean<<<2, INT, 0, st>>>(x1, x2, n, scratch);
    k_subtract<<<grid_for(n, sms), INT, 0, st>>>(x1, n, scratch);
    k_subtract<<<grid_for(n, sms), INT, 0, st>>>(x2, n, scratch + 1);
    ck(cudaGetLastError(), "mean subtraction");
    ck(cudaMemcpyAsync(means, scratch, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
  }
  double lo1, hi1, lo2, hi2;
  minmax(x1, n, sms, scratch + 2, &lo1, &hi1, st);
  minmax(x2, n, sms, scratch + 2, &lo2, &hi2, st);
  for (double v : {lo1, hi1, lo2, hi2})
    if (!std::isfinite(v)) throw Error(POFD_E_ARG, "Non-valid min or max");
  double bc1, bd1, bc2, bd2;
  bin_axis(lo1, hi1, nb1, &bc1, &bd1);
  bin_axis(lo2, hi2, nb2, &bc2, &bd2);
  ck(cudaMemsetAsync(bins, 0, static_cast<size_t>(nb1) * nb2 * sizeof(unsigned), st), "memset");
  k_bin2<<<grid_for(n, sms), INT, 0, st>>>(x1, x2, n, bc1, 1.0 / bd1, nb1, bc2, 1.0 / bd2, nb2,
                                           bins);
  ck(cudaGetLastError(), "binning");
  ck(cudaFreeAsync(scratch, st), "cudaFreeAsync");
  ck(cudaStreamSynchronize(st), "synchronize");
  info6[0] = means[0];
  info6[1] = means[1];
  info6[2] = bc1;
  info6[3] = bd1;
  info6[4] = bc2;
  info6[5] = bd2;
}

}  // namespace pofd
