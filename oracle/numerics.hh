// numerics.hh -- numerical building blocks of the P(D) oracle.
//
// TEST INFRASTRUCTURE ONLY (see pofd_oracle.h).  The reference calls GSL and
// FFTW for these; neither is available, so each is restated here from the
// published algorithm:
//   * natural cubic spline: the tridiagonal "natural" spline equations with a
//     symmetric LDL^T (Cholesky-style) tridiagonal solve, evaluated by the
//     per-interval cubic b,c,d form -- the formulation GSL's
//     gsl_interp_cspline uses (call sites e.g. numberCountsKnotsSpline.cc:271,
//     PDFactory.cc:482).  Interval lookup is the bisection that returns the
//     largest i with x[i] <= v, clamped to [0, n-2].
//   * linear interpolation (gsl_interp_linear, numberCountsDoubleLogNormal.cc:117)
//   * unnormalised real DFTs with FFTW's sign convention (forward e^{-i},
//     inverse e^{+i}); radix-2 for powers of two, direct DFT otherwise.
//   * Brent's root finder (Brent 1973, "Algorithms for Minimization without
//     Derivatives", ch. 4), iterated like GSL's brent solver
//     (numberCountsDoubleLogNormal.cc:1448-1461).
//   * Gauss-Legendre quadrature (nodes by Newton iteration on P_n).
#ifndef POFD_ORACLE_NUMERICS_HH
#define POFD_ORACLE_NUMERICS_HH

#include <cmath>
#include <complex>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

struct OrcError : public std::runtime_error {
  int code;
  OrcError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

using cplx = std::complex<double>;

// ---------------------------------------------------------------- bisection
// Largest i in [lo, hi-1] with x[i] <= v (x strictly increasing).
inline size_t bsearch_lo(const double* x, double v, size_t lo, size_t hi) {
  size_t ilo = lo, ihi = hi;
  while (ihi > ilo + 1) {
    size_t i = (ihi + ilo) / 2;
    if (x[i] > v) ihi = i; else ilo = i;
  }
  return ilo;
}

// ------------------------------------------------------ natural cubic spline
struct NatSpline {
  std::vector<double> x, y, c;  // c = half second derivatives

  void init(const double* xa, const double* ya, size_t n) {
    if (n < 3) throw OrcError(-20, "cspline needs at least 3 points");
    for (size_t i = 1; i < n; ++i)
      if (!(xa[i] > xa[i - 1]))
        throw OrcError(-21, "cspline x values must be strictly increasing");
    x.assign(xa, xa + n);
    y.assign(ya, ya + n);
    c.assign(n, 0.0);
    const size_t sys = n - 2;
    std::vector<double> g(sys), diag(sys), offdiag(sys);
    for (size_t i = 0; i < sys; ++i) {
      const double h_i = xa[i + 1] - xa[i];
      const double h_ip1 = xa[i + 2] - xa[i + 1];
      const double ydiff_i = ya[i + 1] - ya[i];
      const double ydiff_ip1 = ya[i + 2] - ya[i + 1];
      const double g_i = (h_i != 0.0) ? 1.0 / h_i : 0.0;
      const double g_ip1 = (h_ip1 != 0.0) ? 1.0 / h_ip1 : 0.0;
      offdiag[i] = h_ip1;
      diag[i] = 2.0 * (h_ip1 + h_i);
      g[i] = 3.0 * (ydiff_ip1 * g_ip1 - ydiff_i * g_i);
    }
    if (sys == 1) {
      c[1] = g[0] / diag[0];
      return;
    }
    // Symmetric tridiagonal LDL^T solve.
    const size_t N = sys;
    std::vector<double> gamma(N), alpha(N), cc(N), z(N);
    alpha[0] = diag[0];
    gamma[0] = offdiag[0] / alpha[0];
    for (size_t i = 1; i + 1 < N; ++i) {
      alpha[i] = diag[i] - offdiag[i - 1] * gamma[i - 1];
      gamma[i] = offdiag[i] / alpha[i];
    }
    alpha[N - 1] = diag[N - 1] - offdiag[N - 2] * gamma[N - 2];
    z[0] = g[0];
    for (size_t i = 1; i < N; ++i) z[i] = g[i] - gamma[i - 1] * z[i - 1];
    for (size_t i = 0; i < N; ++i) cc[i] = z[i] / alpha[i];
    c[1 + N - 1] = cc[N - 1];
    for (size_t k = N - 1; k-- > 0;) c[1 + k] = cc[k] - gamma[k] * c[1 + k + 1];
  }

  size_t find(double v) const { return bsearch_lo(x.data(), v, 0, x.size() - 1); }

  double eval(double v) const {
    const size_t n = x.size();
    if (v < x[0] || v > x[n - 1])
      throw OrcError(-22, "interpolation error: argument outside spline range");
    const size_t i = find(v);
    return eval_at(i, v);
  }

  double eval_at(size_t i, double v) const {
    const double x_lo = x[i], x_hi = x[i + 1];
    const double dx = x_hi - x_lo;
    const double y_lo = y[i], y_hi = y[i + 1];
    const double dy = y_hi - y_lo;
    const double delx = v - x_lo;
    const double c_i = c[i], c_ip1 = c[i + 1];
    const double b = (dy / dx) - dx * (c_ip1 + 2.0 * c_i) / 3.0;
    const double d = (c_ip1 - c_i) / (3.0 * dx);
    return y_lo + delx * (b + delx * (c_i + delx * d));
  }
};

// ------------------------------------------------------- linear interpolation
inline double linear_interp(const std::vector<double>& x,
                            const std::vector<double>& y, double v) {
  const size_t i = bsearch_lo(x.data(), v, 0, x.size() - 1);
  const double x_lo = x[i], x_hi = x[i + 1];
  const double y_lo = y[i], y_hi = y[i + 1];
  const double dx = x_hi - x_lo;
  return y_lo + (v - x_lo) / dx * (y_hi - y_lo);
}

// ------------------------------------------------------------------- DFTs
// Complex DFT in place, sign = -1 forward, +1 inverse, unnormalised.
void cfft(std::vector<cplx>& a, int sign);
void cfft_strided(cplx* a, size_t n, size_t stride, int sign,
                  std::vector<cplx>& work);
// Real forward: out has n/2+1 entries.
// Process-wide switch (default off): route the real transforms below to
// the fast radix-4 ones of fastfft.hh for powers of two >= 8.  For the
// timed CPU baseline; the parity checks keep the radix-2 transforms.
void set_fast_fft(bool on);
bool fast_fft();
void rfft(size_t n, const double* in, cplx* out);
// Real inverse (c2r), unnormalised.  The DC and (even n) Nyquist bins are
// taken by their real parts, which is how an FFTW-style c2r treats them.
void irfft(size_t n, const cplx* in, double* out);
// 2D (n x n, row-major, last dimension halved): out is n x (n/2+1).
void rfft2(size_t n, const double* in, cplx* out);
// 2D inverse.  Columns 0 and n/2 (the self-conjugate ones of the half
// spectrum) are projected onto their Hermitian part, (X_i + conj X_{n-i})/2,
// before the column transforms; the row c2r then takes real parts as above.
void irfft2(size_t n, const cplx* in, double* out);

// ------------------------------------------------------------ Brent roots
struct BrentState {
  double a, b, c, d, e, fa, fb, fc;
};
template <class F>
void brent_init(BrentState& s, F& f, double xl, double xu) {
  const double fl = f(xl), fu = f(xu);
  s.a = xl; s.fa = fl;
  s.b = xu; s.fb = fu;
  s.c = xu; s.fc = fu;
  s.d = xu - xl; s.e = xu - xl;
  if ((fl < 0.0 && fu < 0.0) || (fl > 0.0 && fu > 0.0))
    throw OrcError(-30, "endpoints do not straddle y=0");
}
// One iteration; returns root estimate and updates bracket [xl, xu].
template <class F>
double brent_iterate(BrentState& s, F& f, double& xl, double& xu) {
  const double DBL_EPS = 2.2204460492503131e-16;
  double a = s.a, b = s.b, c = s.c, d = s.d, e = s.e;
  double fa = s.fa, fb = s.fb, fc = s.fc;
  bool ac_equal = false;
  if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) {
    ac_equal = true;
    c = a; fc = fa;
    d = b - a; e = b - a;
  }
  if (std::fabs(fc) < std::fabs(fb)) {
    ac_equal = true;
    a = b; b = c; c = a;
    fa = fb; fb = fc; fc = fa;
  }
  const double tol = 0.5 * DBL_EPS * std::fabs(b);
  const double m = 0.5 * (c - b);
  if (fb == 0) {
    xl = b; xu = b;
    s = {a, b, c, d, e, fa, fb, fc};
    return b;
  }
  if (std::fabs(m) <= tol) {
    if (b < c) { xl = b; xu = c; } else { xl = c; xu = b; }
    s = {a, b, c, d, e, fa, fb, fc};
    return b;
  }
  if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
    d = m; e = m;  // bisection
  } else {
    double p, q, r;
    const double sr = fb / fa;
    if (ac_equal) {
      p = 2 * m * sr;
      q = 1 - sr;
    } else {
      q = fa / fc;
      r = fb / fc;
      p = sr * (2 * m * q * (q - r) - (b - a) * (r - 1));
      q = (q - 1) * (r - 1) * (sr - 1);
    }
    if (p > 0) q = -q; else p = -p;
    const double lim1 = 3 * m * q - std::fabs(tol * q);
    const double lim2 = std::fabs(e * q);
    if (2 * p < (lim1 < lim2 ? lim1 : lim2)) {
      e = d;
      d = p / q;
    } else {
      d = m; e = m;
    }
  }
  a = b; fa = fb;
  if (std::fabs(d) > tol) b += d;
  else b += (m > 0 ? +tol : -tol);
  fb = f(b);
  s = {a, b, c, d, e, fa, fb, fc};
  if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) c = a;
  if (b < c) { xl = b; xu = c; } else { xl = c; xu = b; }
  return b;
}
// Relative interval test (|xu - xl| < epsabs + epsrel * min|x| when the
// bracket does not straddle 0).
inline bool root_interval_ok(double xl, double xu, double epsabs,
                             double epsrel) {
  const double al = std::fabs(xl), au = std::fabs(xu);
  double min_abs;
  if ((xl > 0.0 && xu > 0.0) || (xl < 0.0 && xu < 0.0))
    min_abs = (al < au) ? al : au;
  else
    min_abs = 0;
  const double tol = epsabs + epsrel * min_abs;
  return std::fabs(xu - xl) < tol;
}

// ------------------------------------------------- Gauss-Legendre quadrature
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

}  // namespace orc
#endif
