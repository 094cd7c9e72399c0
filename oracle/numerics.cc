// numerics.cc -- DFTs and quadrature nodes of the P(D) oracle.
// TEST INFRASTRUCTURE ONLY (see pofd_oracle.h and numerics.hh).
#include "numerics.hh"

#include <atomic>
#include <map>
#include <mutex>

#include "fastfft.hh"

namespace orc {

namespace {

const double kTwoPi = 2.0 * 3.141592653589793238462643383279502884197;

bool is_pow2(size_t n) { return n && !(n & (n - 1)); }

// Twiddle table w[k] = exp(-2 pi i k / n), k < n, from exact angles
// (sin/cos of 2 pi k / n reduced to the first octant by symmetry would be
// marginally better; direct evaluation is accurate to ~1 ulp here).
const std::vector<cplx>& twiddles(size_t n) {
  static std::mutex mtx;
  static std::map<size_t, std::vector<cplx>> cache;
  std::lock_guard<std::mutex> lk(mtx);
  auto it = cache.find(n);
  if (it != cache.end()) return it->second;
  std::vector<cplx> w(n);
  for (size_t k = 0; k < n; ++k) {
    const double ang = kTwoPi * static_cast<double>(k) / static_cast<double>(n);
    w[k] = cplx(std::cos(ang), -std::sin(ang));
  }
  return cache.emplace(n, std::move(w)).first->second;
}

void fft_pow2(cplx* a, size_t n, int sign) {
  // bit reversal
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  const std::vector<cplx>& w = twiddles(n);
  for (size_t len = 2; len <= n; len <<= 1) {
    const size_t half = len >> 1;
    const size_t step = n / len;
    for (size_t i = 0; i < n; i += len) {
      for (size_t k = 0; k < half; ++k) {
        cplx t = w[k * step];
        if (sign > 0) t = std::conj(t);
        const cplx u = a[i + k];
        const cplx v = a[i + k + half] * t;
        a[i + k] = u + v;
        a[i + k + half] = u - v;
      }
    }
  }
}

void dft_direct(cplx* a, size_t n, int sign) {
  const std::vector<cplx>& w = twiddles(n);
  std::vector<cplx> out(n);
  for (size_t k = 0; k < n; ++k) {
    cplx s = 0.0;
    for (size_t j = 0; j < n; ++j) {
      cplx t = w[(j * k) % n];
      if (sign > 0) t = std::conj(t);
      s += a[j] * t;
    }
    out[k] = s;
  }
  for (size_t k = 0; k < n; ++k) a[k] = out[k];
}

void fft_any(cplx* a, size_t n, int sign) {
  if (n <= 1) return;
  if (is_pow2(n)) fft_pow2(a, n, sign);
  else dft_direct(a, n, sign);
}

}  // namespace

void cfft(std::vector<cplx>& a, int sign) { fft_any(a.data(), a.size(), sign); }

void cfft_strided(cplx* a, size_t n, size_t stride, int sign,
                  std::vector<cplx>& work) {
  work.resize(n);
  for (size_t i = 0; i < n; ++i) work[i] = a[i * stride];
  fft_any(work.data(), n, sign);
  for (size_t i = 0; i < n; ++i) a[i * stride] = work[i];
}

namespace {
std::atomic<bool> g_fast_fft{false};
}

void set_fast_fft(bool on) { g_fast_fft.store(on); }
bool fast_fft() { return g_fast_fft.load(); }

void rfft(size_t n, const double* in, cplx* out) {
  if (fast_fft() && fastfft_supported(n)) return rfft_fast(n, in, out);
  std::vector<cplx> a(n);
  for (size_t i = 0; i < n; ++i) a[i] = cplx(in[i], 0.0);
  fft_any(a.data(), n, -1);
  for (size_t k = 0; k <= n / 2; ++k) out[k] = a[k];
}

void irfft(size_t n, const cplx* in, double* out) {
  if (fast_fft() && fastfft_supported(n)) return irfft_fast(n, in, out);
  const size_t nc = n / 2 + 1;
  std::vector<cplx> a(n);
  a[0] = cplx(in[0].real(), 0.0);
  for (size_t k = 1; k < nc; ++k) {
    a[k] = in[k];
    if (n - k != k) a[n - k] = std::conj(in[k]);
  }
  if (n % 2 == 0) a[n / 2] = cplx(in[n / 2].real(), 0.0);
  fft_any(a.data(), n, +1);
  for (size_t i = 0; i < n; ++i) out[i] = a[i].real();
}

void rfft2(size_t n, const double* in, cplx* out) {
  if (fast_fft() && fastfft_supported(n)) return rfft2_fast(n, in, out);
  const size_t nc = n / 2 + 1;
  std::vector<cplx> row(n), work;
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = 0; j < n; ++j) row[j] = cplx(in[i * n + j], 0.0);
    fft_any(row.data(), n, -1);
    for (size_t j = 0; j < nc; ++j) out[i * nc + j] = row[j];
  }
  for (size_t j = 0; j < nc; ++j) cfft_strided(out + j, n, nc, -1, work);
}

void irfft2(size_t n, const cplx* in, double* out) {
  if (fast_fft() && fastfft_supported(n)) return irfft2_fast(n, in, out);
  const size_t nc = n / 2 + 1;
  std::vector<cplx> a(in, in + n * nc), work;
  // Hermitian projection of the self-conjugate columns.
  std::vector<size_t> cols = {0};
  if (n % 2 == 0 && n / 2 != 0) cols.push_back(n / 2);
  for (size_t j : cols) {
    std::vector<cplx> col(n);
    for (size_t i = 0; i < n; ++i) col[i] = a[i * nc + j];
    for (size_t i = 0; i < n; ++i) {
      const size_t im = (n - i) % n;
      a[i * nc + j] = 0.5 * (col[i] + std::conj(col[im]));
    }
  }
  for (size_t j = 0; j < nc; ++j) cfft_strided(a.data() + j, n, nc, +1, work);
  for (size_t i = 0; i < n; ++i) irfft(n, a.data() + i * nc, out + i * n);
}

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  const double pi = 3.141592653589793238462643383279502884197;
  const int m = (n + 1) / 2;
  for (int i = 0; i < m; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 0; j < n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j + 1.0) * z * p2 - j * p3) / (j + 1);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-15) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - 1 - i] = w[i];
  }
}

}  // namespace orc
