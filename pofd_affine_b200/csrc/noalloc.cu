// noalloc.cu -- the allocation-free variant of the 1D P(D) reduction and
// log-likelihood step (pofd_pd1_loglike_noalloc in pofd_b200.h).
//
// Some callers cannot allocate GPU memory when they evaluate a likelihood:
// a host program whose device memory is already reserved by another
// allocator (a framework's caching pool that owns the GPU), or a
// latency-sensitive caller that cannot take the device-wide
// synchronisation cudaMalloc/cudaFree imply.  For them this entry point runs
// the split-point search, unwrap, normalisation and binned log-likelihood of
// one wrapped P(D) (the array the inverse FFT produces) on caller-owned
// inputs and outputs, keeping its only scratch -- the per-chunk partial
// reductions -- in a fixed-size file-scope device array.
//
// Limits and sharing:
//   * n <= kMaxN (64 chunks of 4096 values, 262144); larger n is rejected.
//   * The scratch array exists once per GPU that loads the library and is
//     held until the process exits.  Every call shares it and it keeps the
//     last call's contents; each call overwrites every slot it reads, so
//     nothing has to start at zero.  Calls whose kernels overlap on the GPU
//     (different streams, or different host threads on one device) race on
//     the array: serialise them.
//   * The first call on each device looks up the array's device address
//     with cudaGetSymbolAddress (with that device current); make that first
//     call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/pofd_b200.h"
#include "common.cuh"

namespace {

constexpr int kNT = 256;
constexpr int kChunk = kNT * 16;
constexpr int kMaxChunks = 64;
constexpr unsigned kMaxN = kMaxChunks * kChunk;  // 262144
constexpr int kSlot = 5;  // max, sum, index-weighted sum, min value, min index

// The scratch: partial reductions of every chunk of the P(D).
static __device__ __align__(256) double g_noalloc_scratch[kMaxChunks * kSlot];

constexpr int kMaxDevices = 64;
std::mutex g_mtx;
double* g_scratch_addr[kMaxDevices] = {nullptr};

struct NaSplit {
  double sgpos, sgneg, n1sigpos, n1signeg;
  long long botidx, topidx;
};

__device__ __forceinline__ long long na_index(double v) {
  if (!(v < 9.0e15)) return 0x7fffffffffffLL;
  if (!(v > -9.0e15)) return -0x7fffffffffffLL;
  return static_cast<long long>(v);
}

// Split-search window (PDFactory.cc:756-815) from the variance without noise
// and the dataset's noise level (PDFactory.cc:1225-1233).
__device__ __forceinline__ NaSplit na_split(double dflux, double minflux_R,
                                            int wrap, double var,
                                            double sigma) {
  NaSplit sp;
  sp.sgpos = sqrt(var + sigma * sigma);
  sp.sgneg = (9 * sigma * sigma > var) ? sigma : sp.sgpos;
  sp.n1sigpos = 2.5 * sp.sgpos;
  sp.n1signeg = 2.5 * sp.sgneg;
  sp.botidx = na_index(sp.n1sigpos / dflux);
  if (sp.n1sigpos > fabs(minflux_R)) sp.topidx = wrap;
  else sp.topidx = na_index(-(sp.n1signeg + minflux_R) / dflux + wrap + 1);
  return sp;
}

__device__ __forceinline__ double na_clip(double v) { return (v < 0) ? 0.0 : v; }

__global__ void __launch_bounds__(kNT)
k_na_pscan(const double* __restrict__ p, int n, double dflux,
           double minflux_R, int wrap, double var, double sigma,
           double* __restrict__ scratch) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  const NaSplit sp = na_split(dflux, minflux_R, wrap, var, sigma);
  const int base = blockIdx.x * kChunk;
  double mx = -1.0e308, sum = 0.0, wsum = 0.0, mnv = 1.0e308;
  int mni = 0x7fffffff;
  for (int k = 0; k < kChunk / kNT; ++k) {
    const int li = k * kNT + threadIdx.x;
    const int i = base + li;
    if (i >= n) break;
    const double v = na_clip(p[i]);
    if (v > mx) mx = v;
    sum += v;
    wsum += static_cast<double>(li) * v;
    if (i >= sp.botidx && i <= sp.topidx) pofd::dev::argmin_merge(mnv, mni, v, i);
  }
  mx = pofd::dev::block_max<kNT>(mx, shd);
  sum = pofd::dev::block_sum<kNT>(sum, shd);
  wsum = pofd::dev::block_sum<kNT>(wsum, shd);
  pofd::dev::block_argmin<kNT>(mnv, mni, shd, shi);
  if (threadIdx.x == 0) {
    double* o = scratch + blockIdx.x * kSlot;
    o[0] = mx;
    o[1] = sum;
    o[2] = wsum;
    o[3] = mnv;
    o[4] = static_cast<double>(mni);
  }
}

__device__ __forceinline__ double na_logp(const double* __restrict__ p, int n,
                                          int split, double itot, int j) {
  int s = j + split;
  if (s >= n) s -= n;
  const double v = na_clip(p[s]) * itot;
  return (v > 0.0) ? log2(v) : pofd::dev::kSmallLogVal;
}

// Split point, unwrap, normalisation, mean and binned log-likelihood
// (PDFactory.cc:691-1009, PD.cc:146-274, 557-619, calcLike.cc:419-425).
// out = {(logL - like_offset)/like_norm, split index, flux of element 0}.
__global__ void __launch_bounds__(kNT)
k_na_pfinish(const double* __restrict__ p, int n, double dflux,
             double minflux_R, int wrap, double var, double sigma,
             const int* __restrict__ nzidx, const double* __restrict__ nzcnt,
             int nnz, double bincent0, double bindelta, double like_offset,
             double like_norm, double log2toe, int nchunk,
             const double* __restrict__ scratch, double* __restrict__ out,
             int* __restrict__ status) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  __shared__ int s_state, s_split;
  __shared__ double s_jitter;
  const NaSplit sp = na_split(dflux, minflux_R, wrap, var, sigma);
  if (threadIdx.x == 0) {
    int st = 0;
    double peak = -1.0e308, minval = 1.0e308;
    int minidx = 0x7fffffff;
    for (int c = 0; c < nchunk; ++c) {
      const double* o = scratch + c * kSlot;
      if (o[0] > peak) peak = o[0];
      pofd::dev::argmin_merge(minval, minidx, o[3], static_cast<int>(o[4]));
    }
    const long long bot = sp.botidx, top = sp.topidx;
    double jitter = 0.0;
    int split = -1;
    if (sp.sgpos <= 0 || sp.sgneg <= 0) st = POFD_E_SPLIT_RANGE;
    else if (n * dflux < (sp.n1sigpos + sp.n1signeg)) st = POFD_E_SPLIT_RANGE;
    else if (!(peak > 0.0)) st = POFD_E_SPLIT_PEAK;
    else if (bot >= n || top >= n || bot < 0 || top < 0) st = POFD_E_SPLIT_LOGIC;
    if (st == 0) {
      if (bot > top) { minidx = static_cast<int>(bot); minval = na_clip(p[minidx]); }
      if (minidx < 0 || minidx >= n) st = POFD_E_SPLIT_MIN;
      else if (minval > 1e-5 * peak) st = POFD_E_SPLIT_MIN;
    }
    bool found = false;
    if (st == 0) {
      const int pre = 17;
      if (minidx > pre) {
        bool mono = true;
        double prev = na_clip(p[minidx - pre]);
        jitter = prev;
        for (int i = minidx - pre + 1; i < minidx; ++i) {
          const double cv = na_clip(p[i]);
          if (cv >= prev) mono = false;
          jitter += cv;
          prev = cv;
        }
        if (mono) { split = minidx; found = true; }
        else jitter = 1.1 * (jitter + minval) / static_cast<double>(pre + 1);
      } else {
        jitter = 5e-14 * peak;
        if (minval > jitter) { split = minidx; found = true; }
      }
      if (!found) {
        if (minval <= 0.0) {
          long long bi = (minidx < bot) ? bot : minidx - 3;
          const long long ti = (minidx > top - 3) ? top - 3 : minidx + 3;
          if (bi < 0) bi = 0;
          for (long long i = bi; i < ti; ++i) {
            const double cv = na_clip(p[i]);
            if (cv > minval) minval = cv;
          }
        }
        if (minval > 0) jitter = (5.0 * minval) < jitter ? (5.0 * minval) : jitter;
        if (bot >= top) st = POFD_E_SPLIT_LOGIC;
        else if (na_clip(p[top]) < jitter) st = POFD_E_SPLIT_TOP;
      }
    }
    s_state = (st != 0) ? st : (found ? 1 : 0);
    s_split = split;
    s_jitter = jitter;
  }
  __syncthreads();
  int state = s_state;
  if (state == 0) {
    const double jitter = s_jitter;
    int hitidx = -1;
    for (long long t = sp.topidx - 1; t >= sp.botidx; t -= kNT) {
      const long long i = t - threadIdx.x;
      int hit = -1;
      if (i >= sp.botidx && na_clip(p[i]) < jitter) hit = static_cast<int>(i);
      const int m = pofd::dev::block_max_int<kNT>(hit, shi);
      if (m >= 0) { hitidx = m; break; }
    }
    if (hitidx >= 0) { state = 1; if (threadIdx.x == 0) s_split = hitidx + 1; }
    else state = POFD_E_SPLIT_NONE;
    __syncthreads();
  }
  if (state < 0) {
    if (threadIdx.x == 0) {
      *status = state;
      out[0] = 0.0; out[1] = -1.0; out[2] = 0.0;
    }
    return;
  }
  const int split = s_split;
  const int cfull = split / kChunk;
  double part = 0.0;
  for (int i = cfull * kChunk + threadIdx.x; i < split; i += kNT) part += na_clip(p[i]);
  part = pofd::dev::block_sum<kNT>(part, shd);
  double S = 0.0, W = 0.0, T = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    const double* o = scratch + c * kSlot;
    S += o[1];
    W += static_cast<double>(c) * kChunk * o[1] + o[2];
    if (c < cfull) T += o[1];
  }
  T += part;
  const double q0 = na_clip(p[split]);
  const double qlast = na_clip(p[split == 0 ? n - 1 : split - 1]);
  const double itot = 1.0 / ((S - 0.5 * q0 - 0.5 * qlast) * dflux);
  const double srot = W - static_cast<double>(split) * S + static_cast<double>(n) * T;
  const double tmn = itot * (srot - 0.5 * static_cast<double>(n - 1) * qlast) * dflux * dflux;
  if (isinf(tmn) || isnan(tmn)) {
    if (threadIdx.x == 0) { *status = POFD_E_UNSHIFT; out[0] = 0.0; out[1] = split; out[2] = 0.0; }
    return;
  }
  const double minflux = -tmn;
  const double maxfluxval = minflux + static_cast<double>(n - 1) * dflux - dflux;
  const double idflux = 1.0 / dflux;
  double ll = 0.0;
  for (int e = threadIdx.x; e < nnz; e += kNT) {
    const double cnt = nzcnt[e];
    const double cflux = bincent0 + static_cast<double>(nzidx[e]) * bindelta;
    double v;
    if (cflux < minflux) v = cnt * na_logp(p, n, split, itot, 0);
    else if (cflux > maxfluxval) v = cnt * na_logp(p, n, split, itot, n - 1);
    else {
      const double delt = (cflux - minflux) * idflux;
      const int idx = static_cast<int>(delt);
      const double t = delt - static_cast<double>(idx);
      v = ((1.0 - t) * na_logp(p, n, split, itot, idx) +
           t * na_logp(p, n, split, itot, idx + 1)) * cnt;
    }
    ll += v;
  }
  ll = pofd::dev::block_sum<kNT>(ll, shd);
  if (threadIdx.x == 0) {
    *status = 0;
    out[0] = (log2toe * ll - like_offset) / like_norm;
    out[1] = static_cast<double>(split);
    out[2] = minflux;
  }
}

}  // namespace

namespace pofd {
void set_last_error(const char* msg);  // capi.cu
}

extern "C" int pofd_pd1_loglike_noalloc(
    const double* pofd_dev, unsigned n, double dflux, double minflux_R,
    unsigned wrapRidx, double var_noi, double sigma, const int* nzidx_dev,
    const double* nzcnt_dev, unsigned nnz, double bincent0, double bindelta,
    double like_offset, double like_norm, double* out_dev, int* status_dev,
    void* stream) {
  if (!pofd_dev || !out_dev || !status_dev || (nnz > 0 && (!nzidx_dev || !nzcnt_dev))) {
    pofd::set_last_error("pofd_pd1_loglike_noalloc: null device pointer");
    return POFD_E_ARG;
  }
  if (n < 2 || n > kMaxN) {
    // n beyond the fixed scratch (64 chunks of 4096 values)
    pofd::set_last_error("pofd_pd1_loglike_noalloc: n must be in [2, 262144]");
    return POFD_E_ARG;
  }
  if (!(dflux > 0) || wrapRidx < 1 || wrapRidx >= n) {
    pofd::set_last_error("pofd_pd1_loglike_noalloc: need dflux > 0 and 1 <= wrapRidx < n");
    return POFD_E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    pofd::set_last_error("pofd_pd1_loglike_noalloc: no usable current device");
    return POFD_E_CUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    pofd::set_last_error("pofd_pd1_loglike_noalloc: stream query failed");
    return POFD_E_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    // Outside stream capture the address is looked up on every call (with
    // the device current): a device reset reloads the module and moves the
    // array, and a stored address would then be stale.  Inside a capture
    // the address from the last uncaptured call on this device is used.
    if (cs == cudaStreamCaptureStatusNone || !g_scratch_addr[dev]) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
        pofd::set_last_error("pofd_pd1_loglike_noalloc: scratch address lookup failed");
        return POFD_E_CUDA;
      }
      g_scratch_addr[dev] = static_cast<double*>(ptr);
    }
    scratch = g_scratch_addr[dev];
  }
  const int nchunk = static_cast<int>((n + kChunk - 1) / kChunk);
  k_na_pscan<<<nchunk, kNT, 0, st>>>(pofd_dev, static_cast<int>(n), dflux,
                                     minflux_R, static_cast<int>(wrapRidx),
                                     var_noi, sigma, scratch);
  k_na_pfinish<<<1, kNT, 0, st>>>(pofd_dev, static_cast<int>(n), dflux,
                                  minflux_R, static_cast<int>(wrapRidx),
                                  var_noi, sigma, nzidx_dev, nzcnt_dev,
                                  static_cast<int>(nnz), bincent0, bindelta,
                                  like_offset, like_norm, std::log(2.0),
                                  nchunk, scratch, out_dev, status_dev);
  return (cudaGetLastError() == cudaSuccess) ? POFD_OK : POFD_E_CUDA;
}
