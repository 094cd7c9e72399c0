// common.cuh -- device helpers shared by the P(D) kernels.
#ifndef POFD_COMMON_CUH
#define POFD_COMMON_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

namespace pofd {

// A named NVTX range for the life of the object: host entry points show up
// as ranges in a timeline profiler (NVTX v3 is header-only; without a tool
// attached the calls return at once).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace dev {

constexpr double kTwoPi = 6.283185307179586476925286766559005768394;
constexpr double kSmallLogVal = -30.0;

// ------------------------------------------------------------------ exp2
// Table-driven 2^x after Tang ("Table-driven implementation of the
// exponential function in IEEE floating-point arithmetic", ACM TOMS 15,
// 1989): x = k + j/256 + r with j in [0, 256), |r| <= 1/512;
// 2^x = 2^k * T[j] * 2^r, T[j] = 2^(j/256) from a 256-entry table built at
// block start, 2^r from its Taylor series sum_{m<=4} (r ln 2)^m / m!
// (truncation < 4e-17 relative: (ln 2 / 512)^5 / 5!), 2^k by adding k to
// the exponent field.  Arguments below -1022 give exactly 0 (results under
// 2^-1022 never change the sums they enter); arguments must be below 1023.
struct Exp2Table {
  double t[256];
  __device__ __forceinline__ void load() {
    for (int j = threadIdx.x; j < 256; j += blockDim.x) t[j] = exp2(static_cast<double>(j) / 256.0);
  }
};

__device__ __forceinline__ double exp2_tab(double x, const double* __restrict__ tab) {
  // n = round(256 x) via the 1.5 * 2^52 shifter; its low word holds n
  const double sh = 6755399441055744.0;
  const double t = fma(x, 256.0, sh);
  const double nd = t - sh;
  const int n = __double2loint(t);
  const double r = fma(nd, -0.00390625, x);
  // (ln 2)^m / m!, m = 4 .. 1
  double p = 9.6181291076284772e-03;
  p = fma(p, r, 5.5504108664821580e-02);
  p = fma(p, r, 2.4022650695910071e-01);
  p = fma(p, r, 6.9314718055994531e-01);
  p = fma(p, r, 1.0);
  const double v = p * tab[n & 255];
  const int k = n >> 8;
  const double s = __hiloint2double(__double2hiint(v) + (k << 20), __double2loint(v));
  return (x < -1022.0) ? 0.0 : s;
}


// -------------------------------------------------------------- reductions
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < NT / 32) ? sh[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

// max that ignores nothing special: plain (a > b ? a : b) semantics
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

template <int NT>
__device__ __forceinline__ double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < NT / 32) ? sh[l] : -1.0e308;
    for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

// (value, index) minimum; ties go to the smaller index, matching a forward
// scan that replaces the minimum only on strictly smaller values.
__device__ __forceinline__ void argmin_merge(double& v, int& i, double v2, int i2) {
  if (v2 < v || (v2 == v && i2 < i)) { v = v2; i = i2; }
}

template <int NT>
__device__ __forceinline__ void block_argmin(double& v, int& i, double* shv,
                                             int* shi) {
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
    argmin_merge(v, i, v2, i2);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) { shv[w] = v; shi[w] = i; }
  __syncthreads();
  if (w == 0) {
    v = (l < NT / 32) ? shv[l] : 1.0e308;
    i = (l < NT / 32) ? shi[l] : 0x7fffffff;
    for (int o = 16; o > 0; o >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
      argmin_merge(v, i, v2, i2);
    }
    if (l == 0) { shv[0] = v; shi[0] = i; }
  }
  __syncthreads();
  v = shv[0];
  i = shi[0];
  __syncthreads();
}

template <int NT>
__device__ __forceinline__ int block_max_int(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < NT / 32) ? sh[l] : -0x7fffffff;
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) sh[0] = v;
  }
  __syncthreads();
  const int r = sh[0];
  __syncthreads();
  return r;
}

// ------------------------------------------------------ affine-map scans
// Inclusive scan over threads of affine maps z -> a z + b, composed in
// thread order (thread t's result = map_t o ... o map_0).  NT threads,
// shared scratch of 2*NT doubles.  Returns the composed (a, b).
template <int NT>
__device__ __forceinline__ void block_affine_scan(double& a, double& b,
                                                  double* sh) {
  double* sa = sh;
  double* sb = sh + NT;
  const int t = threadIdx.x;
  sa[t] = a;
  sb[t] = b;
  __syncthreads();
  for (int off = 1; off < NT; off <<= 1) {
    double pa = 1.0, pb = 0.0;
    const bool has = t >= off;
    if (has) { pa = sa[t - off]; pb = sb[t - off]; }
    __syncthreads();
    if (has) {
      // (a,b) o (pa,pb): z -> a (pa z + pb) + b
      b = a * pb + b;
      a = a * pa;
      sa[t] = a;
      sb[t] = b;
    }
    __syncthreads();
  }
}

// Same, composed in reverse thread order (thread t's result =
// map_t o map_{t+1} o ... o map_{NT-1}).
template <int NT>
__device__ __forceinline__ void block_affine_rscan(double& a, double& b,
                                                   double* sh) {
  double* sa = sh;
  double* sb = sh + NT;
  const int t = threadIdx.x;
  sa[t] = a;
  sb[t] = b;
  __syncthreads();
  for (int off = 1; off < NT; off <<= 1) {
    double pa = 1.0, pb = 0.0;
    const bool has = t + off < NT;
    if (has) { pa = sa[t + off]; pb = sb[t + off]; }
    __syncthreads();
    if (has) {
      b = a * pb + b;
      a = a * pa;
      sa[t] = a;
      sb[t] = b;
    }
    __syncthreads();
  }
}

// Warp-shuffle forms of the two scans for NT threads (a multiple of 32,
// at most 1024): a register scan inside each warp, one warp scanning the
// warp totals, and each warp composed with the total of the warps before it
// (after it, for the reverse scan).  Shared scratch of 2 * 32 doubles, two
// barriers.  Besides the inclusive map of the thread, returns the b of the
// neighbour's inclusive map (the previous thread's, 0 for thread 0; the
// next thread's, 0 for the last), i.e. the value the neighbour's composed
// map takes at z = 0.
template <int NT>
__device__ __forceinline__ double block_affine_scan_w(double& a, double& b, double* sh) {
  const int t = threadIdx.x, l = t & 31, w = t >> 5;
  constexpr int NW = NT / 32;
  for (int off = 1; off < 32; off <<= 1) {
    const double pa = __shfl_up_sync(0xffffffffu, a, off);
    const double pb = __shfl_up_sync(0xffffffffu, b, off);
    if (l >= off) {
      b = a * pb + b;
      a = a * pa;
    }
  }
  if (l == 31) {
    sh[w] = a;
    sh[32 + w] = b;
  }
  __syncthreads();
  if (w == 0) {
    double wa = (l < NW) ? sh[l] : 1.0, wb = (l < NW) ? sh[32 + l] : 0.0;
    for (int off = 1; off < 32; off <<= 1) {
      const double pa = __shfl_up_sync(0xffffffffu, wa, off);
      const double pb = __shfl_up_sync(0xffffffffu, wb, off);
      if (l >= off) {
        wb = wa * pb + wb;
        wa = wa * pa;
      }
    }
    if (l < NW) {
      sh[l] = wa;
      sh[32 + l] = wb;
    }
  }
  __syncthreads();
  const double pb0 = (w > 0) ? sh[32 + w - 1] : 0.0;
  if (w > 0) {
    b = a * pb0 + b;
    a = a * sh[w - 1];
  }
  const double nb = __shfl_up_sync(0xffffffffu, b, 1);
  return (l > 0) ? nb : pb0;
}

template <int NT>
__device__ __forceinline__ double block_affine_rscan_w(double& a, double& b, double* sh) {
  const int t = threadIdx.x, l = t & 31, w = t >> 5;
  constexpr int NW = NT / 32;
  for (int off = 1; off < 32; off <<= 1) {
    const double pa = __shfl_down_sync(0xffffffffu, a, off);
    const double pb = __shfl_down_sync(0xffffffffu, b, off);
    if (l + off < 32) {
      b = a * pb + b;
      a = a * pa;
    }
  }
  if (l == 0) {
    sh[w] = a;
    sh[32 + w] = b;
  }
  __syncthreads();
  if (w == 0) {
    double wa = (l < NW) ? sh[l] : 1.0, wb = (l < NW) ? sh[32 + l] : 0.0;
    for (int off = 1; off < 32; off <<= 1) {
      const double pa = __shfl_down_sync(0xffffffffu, wa, off);
      const double pb = __shfl_down_sync(0xffffffffu, wb, off);
      if (l + off < NW) {
        wb = wa * pb + wb;
        wa = wa * pa;
      }
    }
    if (l < NW) {
      sh[l] = wa;
      sh[32 + l] = wb;
    }
  }
  __syncthreads();
  const double nb0 = (w + 1 < NW) ? sh[32 + w + 1] : 0.0;
  if (w + 1 < NW) {
    b = a * nb0 + b;
    a = a * sh[w + 1];
  }
  const double nb = __shfl_down_sync(0xffffffffu, b, 1);
  return (l < 31) ? nb : nb0;
}

// Largest i in [lo, hi-1] with x[i] <= v (x increasing): the bisection of
// the interpolation library the reference uses, clamped to [lo, hi-1].
__device__ __forceinline__ int bsearch_lo(const double* __restrict__ x,
                                          double v, int lo, int hi) {
  int ilo = lo, ihi = hi;
  while (ihi > ilo + 1) {
    const int i = (ihi + ilo) >> 1;
    if (x[i] > v) ihi = i; else ilo = i;
  }
  return ilo;
}

}  // namespace dev
}  // namespace pofd
#endif
