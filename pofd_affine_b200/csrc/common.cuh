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

// e^x by the same table: x log2(e) is formed as y + e with y = RN(x L_hi)
// and e = (x L_hi - y) + x L_lo (one FMA recovers the product's rounding
// error; L_hi + L_lo = log2(e) to ~1e-33), so that the reduction
// 2^(y + e) = 2^k T[j] 2^(r + e) loses nothing to the scaling by log2(e)
// even at |x| ~ 700.  Arguments below -708 give exactly 0 (the true values
// are below 2^-1021 and never change the sums they enter); above 708 the
// library exp is used.
__device__ __forceinline__ double exp_tab(double x, const double* __restrict__ tab) {
  if (x > 708.0) return exp(x);
  const double lhi = 1.4426950408889634, llo = 2.0355273740931033e-17;
  const double y = x * lhi;
  const double e = fma(x, lhi, -y) + x * llo;
  const double sh = 6755399441055744.0;
  const double t = fma(y, 256.0, sh);
  const double nd = t - sh;
  const int n = __double2loint(t);
  const double r = fma(nd, -0.00390625, y) + e;
  double p = 9.6181291076284772e-03;
  p = fma(p, r, 5.5504108664821580e-02);
  p = fma(p, r, 2.4022650695910071e-01);
  p = fma(p, r, 6.9314718055994531e-01);
  p = fma(p, r, 1.0);
  const double v = p * tab[n & 255];
  const int k = n >> 8;
  const double s = __hiloint2double(__double2hiint(v) + (k << 20), __double2loint(v));
  return (x < -708.0) ? 0.0 : s;
}

// ------------------------------------------------------------- sin / cos
// Table-driven sin and cos (the reduction-and-table scheme of Tang's exp
// applied to the circle): x = k (2 pi / 256) + r, |r| <= pi / 256, with the
// reduction done in three FMA steps on 2 pi / 256 = C1 + C2 + C3 (Cody and
// Waite, "Software Manual for the Elementary Functions", 1980; C1 and C2
// carry 31 significant bits, so k C1 and k C2 are exact for |k| < 2^22);
// (cos, sin)(2 pi j / 256) for j = k mod 256 from a table built at block
// start; sin r and cos r - 1 by their Taylor series to r^7 and r^6
// (truncation < 2e-20); then the angle-sum formulas.  Absolute error a few
// units of 2^-53.  For |x| > 65536 the library sincos is used.
struct SinCosTable {
  double2 t[256];  // (cos, sin)(2 pi j / 256)
  __device__ __forceinline__ void load() {
    for (int j = threadIdx.x; j < 256; j += blockDim.x) {
      double sn, cs;
      sincospi(static_cast<double>(j) / 128.0, &sn, &cs);
      t[j] = make_double2(cs, sn);
    }
  }
};

__device__ __forceinline__ void sincos_tab(double x, const double2* __restrict__ tab, double* sn,
                                           double* cs) {
  if (!(fabs(x) <= 65536.0)) {
    sincos(x, sn, cs);
    return;
  }
  const double c1 = 0.024543692605220713, c2 = 9.495469545335112e-13,
               c3 = -3.9191856348971346e-22, inv = 40.74366543152521;
  const double sh = 6755399441055744.0;
  const double t = fma(x, inv, sh);
  const double kd = t - sh;
  const int k = __double2loint(t);
  double r = fma(-kd, c1, x);
  r = fma(-kd, c2, r);
  r = fma(-kd, c3, r);
  const double r2 = r * r;
  const double sr = fma(r * r2, fma(r2, fma(r2, -1.984126984126984e-04, 8.333333333333333e-03),
                                    -1.6666666666666666e-01), r);
  const double cm = r2 * fma(r2, fma(r2, -1.388888888888889e-03, 4.1666666666666664e-02), -0.5);
  const double2 e = tab[k & 255];
  *sn = fma(e.y, cm, fma(e.x, sr, e.y));
  *cs = fma(e.x, cm, fma(-e.y, sr, e.x));
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
