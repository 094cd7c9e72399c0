// fft1d.cuh -- FP64 building blocks of the 1D four-step FFT.
//
// A real transform of length n = 2m runs as a complex transform of length
// m = m1 * 256 on z_j = x_{2j} + i x_{2j+1} (Cooley-Tukey with the
// "four-step" factorisation, Bailey 1990):
//
//   pass A   m1-point DFTs down the columns b of the m1 x 256 view
//            (z[a * 256 + b]), times the twiddle W_m^{c b}, stored as rows
//            Y[c][b];
//   pass B   256-point DFTs along each row c, stored transposed to natural
//            order Z[c + m1 d].
//
// Inside a pass each DFT is split again (L = L1 * L2, L1 <= 16): one thread
// does an L1-point DFT in registers, multiplies by W_L^{n2 k1}, and the
// partial results meet in shared memory for the L2-point register DFTs.
// The register DFTs are radix-2 decimation in time on at most 16 points with
// exact constant twiddles; all other twiddles come from tables built on the
// host in long double and are read from shared memory (fft::tw2).
#ifndef POFD_FFT1D_CUH
#define POFD_FFT1D_CUH

#include <cuda_runtime.h>

namespace pofd {
namespace fft {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }

// e^{S 2 pi i t / 16}, t in [0, 8): cos and sin of multiples of pi/8.
template <int S>
__device__ __forceinline__ double2 w16(int t) {
  constexpr double c1 = 0.92387953251128675613;  // cos(pi/8)
  constexpr double c2 = 0.70710678118654752440;  // cos(pi/4)
  constexpr double c3 = 0.38268343236508977173;  // cos(3 pi/8)
  double c = 1.0, s = 0.0;
  switch (t) {
    case 0: c = 1.0; s = 0.0; break;
    case 1: c = c1; s = c3; break;
    case 2: c = c2; s = c2; break;
    case 3: c = c3; s = c1; break;
    case 4: c = 0.0; s = 1.0; break;
    case 5: c = -c3; s = c1; break;
    case 6: c = -c2; s = c2; break;
    case 7: c = -c1; s = c3; break;
  }
  return make_double2(c, S * s);
}

// In-register DFT of N <= 16 points: v[k] <- sum_j v[j] e^{S 2 pi i j k / N},
// radix-2 decimation in time written as a template recursion so that every
// register index is a compile-time constant.
template <int N, int S>
__device__ __forceinline__ void dft(double2* v) {
  if constexpr (N > 1) {
    double2 e[N / 2], o[N / 2];
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    dft<N / 2, S>(e);
    dft<N / 2, S>(o);
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const int t = k * (16 / N);  // e^{S 2 pi i k / N} = w16(k * 16 / N)
      double2 b = o[k];
      if (t == 4) {
        b = make_double2(-S * b.y, S * b.x);  // times S i
      } else if (t != 0) {
        b = cmul(b, w16<S>(t));
      }
      v[k] = cadd(e[k], b);
      v[k + N / 2] = csub(e[k], b);
    }
  }
}

// Twiddle e^{S 2 pi i t / m}, t < m, from two shared-memory tables:
// H[j] = e^{-2 pi i 128 j / m} (m / 128 entries) and L[i] = e^{-2 pi i i / m}
// (128 entries), W^t = H[t >> 7] L[t & 127] -- exact (one table entry) when
// t is a multiple of 128, else one complex product of two correctly rounded
// values.
template <int S>
__device__ __forceinline__ double2 tw2(const double2* H, const double2* L, int t) {
  const double2 h = H[t >> 7];
  const int lo = t & 127;
  const double2 w = lo ? cmul(h, L[lo]) : h;
  return (S < 0) ? w : make_double2(w.x, -w.y);
}

// Loads the two twiddle tables (nh = m / 128 entries of H, then 128 of L)
// into shared memory; the caller synchronises before use.
__device__ __forceinline__ void load_tw2(double2* Hs, const double2* __restrict__ WH,
                                         const double2* __restrict__ WL, int nh, int t,
                                         int nthreads) {
  for (int i = t; i < nh + 128; i += nthreads) {
    if (i < nh) Hs[i] = __ldg(WH + i);
    else Hs[i] = __ldg(WL + (i - nh));
  }
}

}  // namespace fft
}  // namespace pofd
#endif
