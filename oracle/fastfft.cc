// fastfft.cc -- fast real DFTs for the timed CPU baseline of the oracle.
// TEST AND BASELINE INFRASTRUCTURE ONLY (see fastfft.hh).
#include "fastfft.hh"

#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace orc {

namespace {

using cplx = std::complex<double>;

bool pow2(size_t n) { return n && !(n & (n - 1)); }

// Twiddles of one complex length m: per radix-4 stage of sub-length n the
// values W_n^p, W_n^2p, W_n^3p (p < n/4), W_n = e^{-2 pi i / n}, from the
// angles directly (long double, then rounded).
struct CPlan {
  size_t m = 0;
  std::vector<size_t> off;  // per radix-4 stage, into tw
  std::vector<double> tw;   // 6 doubles per p
  bool radix2_last = false;
};

// Split factors W_{2m}^k = e^{-2 pi i k / (2m)}, k <= m, of a real
// transform of 2m points.
struct RPlan {
  std::vector<double> wr, wi;
};

std::mutex g_mtx;

const CPlan& cplan(size_t m) {
  static std::map<size_t, std::unique_ptr<CPlan>> cache;
  std::lock_guard<std::mutex> lk(g_mtx);
  auto it = cache.find(m);
  if (it != cache.end()) return *it->second;
  auto p = std::make_unique<CPlan>();
  p->m = m;
  const long double tp = 6.283185307179586476925286766559005768L;
  size_t n = m;
  while (n >= 4) {
    p->off.push_back(p->tw.size());
    for (size_t q = 0; q < n / 4; ++q)
      for (int k = 1; k <= 3; ++k) {
        const long double a = tp * static_cast<long double>(k * q) / static_cast<long double>(n);
        p->tw.push_back(static_cast<double>(std::cos(a)));
        p->tw.push_back(static_cast<double>(-std::sin(a)));
      }
    n /= 4;
  }
  p->radix2_last = (n == 2);
  return *cache.emplace(m, std::move(p)).first->second;
}

const RPlan& rplan(size_t n) {
  static std::map<size_t, std::unique_ptr<RPlan>> cache;
  std::lock_guard<std::mutex> lk(g_mtx);
  auto it = cache.find(n);
  if (it != cache.end()) return *it->second;
  auto p = std::make_unique<RPlan>();
  const size_t m = n / 2;
  const long double tp = 6.283185307179586476925286766559005768L;
  p->wr.resize(m + 1);
  p->wi.resize(m + 1);
  for (size_t k = 0; k <= m; ++k) {
    const long double a = tp * static_cast<long double>(k) / static_cast<long double>(n);
    p->wr[k] = static_cast<double>(std::cos(a));
    p->wi[k] = static_cast<double>(-std::sin(a));
  }
  return *cache.emplace(n, std::move(p)).first->second;
}

// One radix-4 Stockham stage of sub-length n over L = stride * batch
// contiguous elements per index: reads index p + k n/4, writes 4p + k.
__attribute__((always_inline)) inline void stage4_body(size_t n, size_t L, const double* tw,
                                                       const double* __restrict__ xr,
                                                       const double* __restrict__ xi,
                                                       double* __restrict__ yr,
                                                       double* __restrict__ yi) {
  const size_t n1 = n / 4;
  for (size_t p = 0; p < n1; ++p) {
    const double* w = tw + 6 * p;
    const double w1r = w[0], w1i = w[1], w2r = w[2], w2i = w[3], w3r = w[4], w3i = w[5];
    const double* __restrict__ ar = xr + p * L;
    const double* __restrict__ ai = xi + p * L;
    const double* __restrict__ br = xr + (p + n1) * L;
    const double* __restrict__ bi = xi + (p + n1) * L;
    const double* __restrict__ cr = xr + (p + 2 * n1) * L;
    const double* __restrict__ ci = xi + (p + 2 * n1) * L;
    const double* __restrict__ dr = xr + (p + 3 * n1) * L;
    const double* __restrict__ di = xi + (p + 3 * n1) * L;
    double* __restrict__ y0r = yr + 4 * p * L;
    double* __restrict__ y0i = yi + 4 * p * L;
    double* __restrict__ y1r = y0r + L;
    double* __restrict__ y1i = y0i + L;
    double* __restrict__ y2r = y0r + 2 * L;
    double* __restrict__ y2i = y0i + 2 * L;
    double* __restrict__ y3r = y0r + 3 * L;
    double* __restrict__ y3i = y0i + 3 * L;
    for (size_t t = 0; t < L; ++t) {
      const double apcr = ar[t] + cr[t], apci = ai[t] + ci[t];
      const double amcr = ar[t] - cr[t], amci = ai[t] - ci[t];
      const double bpdr = br[t] + dr[t], bpdi = bi[t] + di[t];
      const double bmdr = br[t] - dr[t], bmdi = bi[t] - di[t];
      y0r[t] = apcr + bpdr;
      y0i[t] = apci + bpdi;
      const double t1r = amcr + bmdi, t1i = amci - bmdr;  // (a - c) - i (b - d)
      const double t2r = apcr - bpdr, t2i = apci - bpdi;  // (a + c) - (b + d)
      const double t3r = amcr - bmdi, t3i = amci + bmdr;  // (a - c) + i (b - d)
      y1r[t] = w1r * t1r - w1i * t1i;
      y1i[t] = w1r * t1i + w1i * t1r;
      y2r[t] = w2r * t2r - w2i * t2i;
      y2i[t] = w2r * t2i + w2i * t2r;
      y3r[t] = w3r * t3r - w3i * t3i;
      y3i[t] = w3r * t3i + w3i * t3r;
    }
  }
}

__attribute__((always_inline)) inline void stage2_body(size_t L, const double* __restrict__ xr,
                                                       const double* __restrict__ xi,
                                                       double* __restrict__ yr,
                                                       double* __restrict__ yi) {
  for (size_t t = 0; t < L; ++t) {
    const double ar = xr[t], ai = xi[t], br = xr[t + L], bi = xi[t + L];
    yr[t] = ar + br;
    yi[t] = ai + bi;
    yr[t + L] = ar - br;
    yi[t + L] = ai - bi;
  }
}

using Stage4Fn = void (*)(size_t, size_t, const double*, const double*, const double*, double*,
                          double*);
using Stage2Fn = void (*)(size_t, const double*, const double*, double*, double*);

void stage4_plain(size_t n, size_t L, const double* tw, const double* xr, const double* xi,
                  double* yr, double* yi) {
  stage4_body(n, L, tw, xr, xi, yr, yi);
}
void stage2_plain(size_t L, const double* xr, const double* xi, double* yr, double* yi) {
  stage2_body(L, xr, xi, yr, yi);
}
__attribute__((target("avx2,fma"))) void stage4_avx2(size_t n, size_t L, const double* tw,
                                                     const double* xr, const double* xi,
                                                     double* yr, double* yi) {
  stage4_body(n, L, tw, xr, xi, yr, yi);
}
__attribute__((target("avx2,fma"))) void stage2_avx2(size_t L, const double* xr,
                                                     const double* xi, double* yr, double* yi) {
  stage2_body(L, xr, xi, yr, yi);
}

struct Dispatch {
  Stage4Fn s4;
  Stage2Fn s2;
  Dispatch() {
    __builtin_cpu_init();
    const bool v = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
    s4 = v ? stage4_avx2 : stage4_plain;
    s2 = v ? stage2_avx2 : stage2_plain;
  }
};
const Dispatch& dispatch() {
  static const Dispatch d;
  return d;
}

// Forward complex DFT of `batch` interleaved transforms of length m held
// as [m][batch] split arrays (x), with y as scratch of the same size.
// Returns the buffer pair that holds the result (x or y).
std::pair<double*, double*> cfft_split(const CPlan& pl, size_t batch, double* xr, double* xi,
                                       double* yr, double* yi) {
  const Dispatch& d = dispatch();
  size_t n = pl.m, L = batch;
  double *ir = xr, *ii = xi, *orr = yr, *oi = yi;
  for (size_t s = 0; s < pl.off.size(); ++s) {
    d.s4(n, L, pl.tw.data() + pl.off[s], ir, ii, orr, oi);
    std::swap(ir, orr);
    std::swap(ii, oi);
    n /= 4;
    L *= 4;
  }
  if (pl.radix2_last) {
    d.s2(L, ir, ii, orr, oi);
    std::swap(ir, orr);
    std::swap(ii, oi);
  }
  return {ir, ii};
}

struct Work {
  std::vector<double> a, b, c, e;
  void size(size_t n) {
    if (a.size() < n) {
      a.resize(n);
      b.resize(n);
      c.resize(n);
      e.resize(n);
    }
  }
};
Work& work() {
  thread_local Work w;
  return w;
}

void rfft_core(size_t n, const double* in, cplx* out, Work& w) {
  const size_t m = n / 2;
  const CPlan& pl = cplan(m);
  const RPlan& rp = rplan(n);
  w.size(m);
  double *zr = w.a.data(), *zi = w.b.data();
  for (size_t j = 0; j < m; ++j) {
    zr[j] = in[2 * j];
    zi[j] = in[2 * j + 1];
  }
  auto r = cfft_split(pl, 1, zr, zi, w.c.data(), w.e.data());
  const double* Zr = r.first;
  const double* Zi = r.second;
  out[0] = cplx(Zr[0] + Zi[0], 0.0);
  out[m] = cplx(Zr[0] - Zi[0], 0.0);
  for (size_t k = 1; k < m; ++k) {
    const double ar = Zr[k], ai = Zi[k];
    const double br = Zr[m - k], bi = -Zi[m - k];  // conj Z_{m-k}
    const double er = 0.5 * (ar + br), ei = 0.5 * (ai + bi);
    const double dr = ar - br, di = ai - bi;
    const double orr = 0.5 * di, oi = -0.5 * dr;  // -i (Zk - conj Z_{m-k}) / 2
    const double wr = rp.wr[k], wi = rp.wi[k];
    out[k] = cplx(er + wr * orr - wi * oi, ei + wr * oi + wi * orr);
  }
}

void irfft_core(size_t n, const cplx* in, double* out, Work& w) {
  const size_t m = n / 2;
  const CPlan& pl = cplan(m);
  const RPlan& rp = rplan(n);
  w.size(m);
  double *zr = w.a.data(), *zi = w.b.data();
  for (size_t k = 0; k < m; ++k) {
    const double ar = in[k].real(), ai = (k == 0) ? 0.0 : in[k].imag();
    const double br = in[m - k].real(), bi = (k == 0) ? 0.0 : -in[m - k].imag();
    const double sr = ar + br, si = ai + bi;
    const double dr = ar - br, di = ai - bi;
    // i conj(W^k) (Xk - conj X_{m-k})
    const double wr = rp.wr[k], wi = -rp.wi[k];
    const double pr = wr * dr - wi * di, pi = wr * di + wi * dr;
    // conjugated input of the forward transform (inverse by conjugation)
    zr[k] = sr - pi;
    zi[k] = -(si + pr);
  }
  auto r = cfft_split(pl, 1, zr, zi, w.c.data(), w.e.data());
  for (size_t j = 0; j < m; ++j) {
    out[2 * j] = r.first[j];
    out[2 * j + 1] = -r.second[j];
  }
}

constexpr size_t kColBlock = 32;

// Complex DFTs of length n down the columns c0 .. c0+bw-1 of an
// n x nc complex array (row-major), sign -1, or +1 by conjugation.
void column_block(size_t n, size_t nc, size_t c0, size_t bw, cplx* a, int sign, Work& w) {
  const CPlan& pl = cplan(n);
  const size_t tot = n * bw;
  w.size(tot);
  double *xr = w.a.data(), *xi = w.b.data();
  const double s = sign > 0 ? -1.0 : 1.0;
  for (size_t i = 0; i < n; ++i)
    for (size_t c = 0; c < bw; ++c) {
      const cplx v = a[i * nc + c0 + c];
      xr[i * bw + c] = v.real();
      xi[i * bw + c] = s * v.imag();
    }
  auto r = cfft_split(pl, bw, xr, xi, w.c.data(), w.e.data());
  for (size_t i = 0; i < n; ++i)
    for (size_t c = 0; c < bw; ++c)
      a[i * nc + c0 + c] = cplx(r.first[i * bw + c], s * r.second[i * bw + c]);
}

}  // namespace

bool fastfft_supported(size_t n) { return pow2(n) && n >= 8; }

void rfft_fast(size_t n, const double* in, cplx* out) { rfft_core(n, in, out, work()); }

void irfft_fast(size_t n, const cplx* in, double* out) { irfft_core(n, in, out, work()); }

void rfft2_fast(size_t n, const double* in, cplx* out) {
  const size_t nc = n / 2 + 1;
  Work& w = work();
  for (size_t i = 0; i < n; ++i) rfft_core(n, in + i * n, out + i * nc, w);
  for (size_t c0 = 0; c0 < nc; c0 += kColBlock)
    column_block(n, nc, c0, std::min(kColBlock, nc - c0), out, -1, w);
}

void irfft2_fast(size_t n, const cplx* in, double* out) {
  const size_t nc = n / 2 + 1;
  Work& w = work();
  std::vector<cplx> a(in, in + n * nc);
  // Hermitian part of the self-conjugate columns 0 and n/2
  for (size_t j : {static_cast<size_t>(0), n / 2}) {
    for (size_t i = 0; i <= n / 2; ++i) {
      const size_t im = (n - i) % n;
      const cplx h = 0.5 * (a[i * nc + j] + std::conj(a[im * nc + j]));
      a[i * nc + j] = h;
      a[im * nc + j] = std::conj(h);
    }
  }
  for (size_t c0 = 0; c0 < nc; c0 += kColBlock)
    column_block(n, nc, c0, std::min(kColBlock, nc - c0), a.data(), +1, w);
  for (size_t i = 0; i < n; ++i) irfft_core(n, a.data() + i * nc, out + i * n, w);
}

}  // namespace orc
