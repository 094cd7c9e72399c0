// fastfft.hh -- fast real DFTs for the timed CPU baseline of the oracle.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY (see pofd_oracle.h).  The reference
// transforms with FFTW plans made with FFTW_MEASURE (PDFactory.cc:86,
// 293-338; PDFactoryDouble.cc:121, 727-768), single threaded.  The
// oracle's own radix-2 transform (numerics.cc) is kept for parity checks;
// this one exists so that the CPU baseline the GPU is measured against
// transforms at a speed comparable to such plans:
//   * complex transforms by the radix-4 Stockham autosort algorithm (a
//     radix-2 last stage for odd powers of two) on split real/imaginary
//     arrays, the innermost loop running over contiguous elements so that
//     it vectorises; twiddles per stage from a table built once per size;
//   * a real transform of n points as the complex transform of the n/2
//     points x[2j] + i x[2j+1] followed by the even/odd split (and its
//     inverse before the inverse complex transform);
//   * 2D real transforms by rows, then the columns in blocks of adjacent
//     columns, the block index innermost;
//   * an AVX2/FMA build of the inner loops chosen at run time when the CPU
//     has them, a plain build otherwise.
// Sign and scale conventions are FFTW's (forward e^{-i}, inverse e^{+i},
// unnormalised); the c2r forms take the Hermitian part of the
// self-conjugate bins, as the oracle's irfft/irfft2 do.  Powers of two
// >= 8 only.
#ifndef POFD_ORACLE_FASTFFT_HH
#define POFD_ORACLE_FASTFFT_HH

#include <complex>
#include <cstddef>

namespace orc {

bool fastfft_supported(size_t n);
void rfft_fast(size_t n, const double* in, std::complex<double>* out);
void irfft_fast(size_t n, const std::complex<double>* in, double* out);
void rfft2_fast(size_t n, const double* in, std::complex<double>* out);
void irfft2_fast(size_t n, const std::complex<double>* in, double* out);

}  // namespace orc
#endif
