// setup.cc -- host-side set-up of the P(D) likelihood (see setup.hh).
#include "setup.hh"

#include <algorithm>
#include <cstring>

namespace pofd {

// ---------------------------------------------------------------- Beam1
// Pixel selection (|v| > minval, NaN/inf skipped), ascending sort, totals
// and inverses: beam.cc:331-458.
void Beam1::build(const double* pix, size_t n, double PIXSIZE,
                  double MINVAL) {
  if (PIXSIZE <= 0.0) throw Error(POFD_E_ARG, "Invalid (non-positive) pixel size");
  minval = (MINVAL <= 0.0) ? 0.0 : MINVAL;
  pixsize = PIXSIZE;
  pos.clear();
  neg.clear();
  for (size_t i = 0; i < n; ++i) {
    const double v = pix[i];
    if (!std::isfinite(v)) continue;
    if (v > minval) pos.push_back(v);
    if (v < -minval) neg.push_back(std::fabs(v));
  }
  if (pos.empty() && neg.empty())
    throw Error(POFD_E_ARG, "Beam file has only zero values");
  haspos = !pos.empty();
  hasneg = !neg.empty();
  std::sort(pos.begin(), pos.end());
  std::sort(neg.begin(), neg.end());
  totpos = 0.0;
  totneg = 0.0;
  if (haspos) {
    totpos = pos[0];
    for (size_t i = 1; i < pos.size(); ++i) totpos += pos[i];
  }
  if (hasneg) {
    totneg = neg[0];
    for (size_t i = 1; i < neg.size(); ++i) totneg += neg[i];
  }
  posinv.resize(pos.size());
  neginv.resize(neg.size());
  for (size_t i = 0; i < pos.size(); ++i) posinv[i] = 1.0 / pos[i];
  for (size_t i = 0; i < neg.size(); ++i) neginv[i] = 1.0 / neg[i];
  poshist = neghist = false;
  poswt.clear(); posival.clear(); negwt.clear(); negival.clear();
}

namespace {
// Log2-spaced histogram of sorted values with 0.1% padding on both ends;
// non-empty bins keep (count, 1/mean): beam.cc:487-553.
void loghist(const std::vector<double>& v, unsigned nbins,
             std::vector<double>& wt, std::vector<double>& ival) {
  const double pad = 0.0014419741739063218;  // log2(1.001)
  const double lo = std::log2(v.front()) - pad;
  const double hi = std::log2(v.back()) + pad;
  const double step = (hi - lo) / static_cast<double>(nbins);
  std::vector<unsigned> cnt(nbins, 0);
  std::vector<double> sum(nbins, 0.0);
  for (double x : v) {
    const unsigned b = static_cast<unsigned>((std::log2(x) - lo) / step);
    cnt[b] += 1;
    sum[b] += x;
  }
  wt.clear();
  ival.clear();
  for (unsigned b = 0; b < nbins; ++b) {
    if (cnt[b] == 0) continue;
    const double w = static_cast<double>(cnt[b]);
    wt.push_back(w);
    ival.push_back(1.0 / (sum[b] / w));
  }
}
}  // namespace

void Beam1::histogram(unsigned nbins) {
  if (nbins == 0) throw Error(POFD_E_ARG, "Invalid (non-positive) nbins");
  const unsigned thresh = 20;  // beam.h:31
  poshist = neghist = false;
  poswt.clear(); posival.clear(); negwt.clear(); negival.clear();
  if (haspos && pos.size() >= thresh) {
    loghist(pos, nbins, poswt, posival);
    poshist = true;
  }
  if (hasneg && neg.size() >= thresh) {
    loghist(neg, nbins, negwt, negival);
    neghist = true;
  }
}

void Beam1::terms(bool negside, std::vector<double>& w,
                  std::vector<double>& ieta) const {
  const bool hist = poshist;  // beam::isNegHist() returns the positive flag
  if (!negside) {
    if (!haspos) { w.clear(); ieta.clear(); return; }
    if (hist) { w = poswt; ieta = posival; }
    else { ieta = posinv; w.assign(posinv.size(), 1.0); }
  } else {
    if (!hasneg) { w.clear(); ieta.clear(); return; }
    if (hist) { w = negwt; ieta = negival; }
    else { ieta = neginv; w.assign(neginv.size(), 1.0); }
  }
}

// ---------------------------------------------------------- SplineSystem
// The x-dependent half of the natural-spline equations: diag 2(h_i+h_i+1),
// off-diagonal h_i+1, factored as L D L^T (the factorisation the reference's
// spline library performs each time it fits the spline, e.g.
// PDFactory.cc:522 for the R nodes).
void SplineSystem::factor(const std::vector<double>& xn) {
  x = xn;
  const size_t n = x.size();
  if (n < 3) throw Error(POFD_E_ARG, "spline needs at least 3 nodes");
  ih.resize(n - 1);
  for (size_t i = 0; i + 1 < n; ++i) {
    const double h = x[i + 1] - x[i];
    if (!(h > 0)) throw Error(POFD_E_ARG, "spline nodes must increase");
    ih[i] = 1.0 / h;
  }
  const size_t N = n - 2;
  std::vector<double> diag(N), off(N);
  for (size_t i = 0; i < N; ++i) {
    const double h_i = x[i + 1] - x[i];
    const double h_ip1 = x[i + 2] - x[i + 1];
    off[i] = h_ip1;
    diag[i] = 2.0 * (h_ip1 + h_i);
  }
  alpha.assign(N, 0.0);
  gamma.assign(N, 0.0);
  alpha[0] = diag[0];
  gamma[0] = off[0] / alpha[0];
  for (size_t i = 1; i + 1 < N; ++i) {
    alpha[i] = diag[i] - off[i - 1] * gamma[i - 1];
    gamma[i] = off[i] / alpha[i];
  }
  if (N > 1) alpha[N - 1] = diag[N - 1] - off[N - 2] * gamma[N - 2];
}

// ---------------------------------------------------------------- Data1
void Data1::meanSubtract() {
  double m = data[0];
  for (size_t i = 1; i < data.size(); ++i) m += data[i];
  m /= static_cast<double>(data.size());
  for (auto& v : data) v -= m;
  if (binned) bincent0 -= m;
}

std::pair<double, double> Data1::minmax() const {
  if (binned)
    return {bincent0, bincent0 + static_cast<double>(nbins - 1) * bindelta};
  double lo = data[0], hi = data[0];
  for (size_t i = 1; i < data.size(); ++i) {
    if (data[i] < lo) lo = data[i];
    if (data[i] > hi) hi = data[i];
  }
  return {lo, hi};
}

// Bin centres at min and max: fitsData.cc:406-437.
void Data1::applyBinning(unsigned NB) {
  if (NB == 0) throw Error(POFD_E_ARG, "Trying to bin with no bins");
  binned = false;
  const auto mm = minmax();
  nbins = NB;
  bins.assign(NB, 0u);
  bincent0 = mm.first;
  bindelta = (NB == 1) ? 2 * (mm.second - mm.first)
                       : (mm.second - mm.first) / static_cast<double>(NB - 1);
  const double ib = 1.0 / bindelta;
  for (double v : data) {
    const unsigned idx = static_cast<unsigned>((v - bincent0) * ib + 0.5);
    bins[idx] += 1;
  }
  binned = true;
}

// --------------------------------------------------------------- RGrid1
void RGrid1::init(unsigned N, double minflux, double maxflux) {
  if (N == 0) throw Error(POFD_E_ARG, "Invalid (0) n");
  if (maxflux < minflux) std::swap(minflux, maxflux);
  n = N;
  if (N == 1) {
    if (minflux < 0.0) throw Error(POFD_E_ARG, "n must be > 1 with negative fluxes");
    dflux = maxflux - minflux;
    minflux_R = minflux;
    wrapRidx = 0;
    return;
  }
  const double inm1 = 1.0 / static_cast<double>(N - 1);
  if (maxflux > 0) {
    if (minflux > 0) minflux = 0.0;
    if (minflux == 0) {
      wrapRidx = N - 1;
      minflux_R = 0.0;
      dflux = maxflux * inm1;
    } else {
      dflux = (maxflux - minflux) * inm1;
      dflux = maxflux / (N - std::floor(-minflux / dflux) - 1.0);
      wrapRidx = static_cast<unsigned>(maxflux / dflux + 0.9999999999);
      minflux_R = (wrapRidx + 1) * dflux - static_cast<double>(N) * dflux;
    }
  } else {
    if (minflux >= 0) throw Error(POFD_E_ARG, "No effective range in R fluxes");
    dflux = -minflux * inm1;
    wrapRidx = 0;
    minflux_R = minflux;
  }
}

std::pair<double, double> rrange_knots(double maxknot, const Beam1& bm) {
  if (bm.haspos)
    return {bm.hasneg ? -maxknot * bm.maxneg() : 0.0, maxknot * bm.maxpos()};
  return {-maxknot * bm.maxneg(), 0.0};
}

// ---------------------------------------------------------------- Beam2
// Sign components pp/pn/np/nn of pixels with |v1|,|v2| > minval, input
// order kept: doublebeam.cc:331-462.
void Beam2::build(const double* b1, const double* b2, size_t n,
                  double PIXSIZE, double MINVAL) {
  if (n == 0) throw Error(POFD_E_ARG, "Invalid (zero) n");
  if (MINVAL < 0.0) throw Error(POFD_E_ARG, "Invalid (negative) MINVAL");
  if (PIXSIZE <= 0.0) throw Error(POFD_E_ARG, "Invalid (non-positive) pixel size");
  minval = MINVAL;
  pixsize = PIXSIZE;
  for (int s = 0; s < 4; ++s) {
    hassign[s] = ishist[s] = false;
    pix1[s].clear(); pix2[s].clear();
    minbm1[s] = maxbm1[s] = minbm2[s] = maxbm2[s] = nan();
  }
  for (size_t i = 0; i < n; ++i) {
    const double v1 = b1[i], v2 = b2[i];
    const double a1 = std::fabs(v1), a2 = std::fabs(v2);
    if (a1 > minval && a2 > minval) {
      const int s = (v1 > 0) ? ((v2 > 0) ? 0 : 1) : ((v2 > 0) ? 2 : 3);
      pix1[s].push_back(a1);
      pix2[s].push_back(a2);
    }
  }
  if (!(pix1[0].size() + pix1[1].size() + pix1[2].size() + pix1[3].size()))
    throw Error(POFD_E_ARG, "No acceptable values found");
  for (int s = 0; s < 4; ++s) {
    const size_t m = pix1[s].size();
    if (!m) continue;
    hassign[s] = true;
    inv1[s].resize(m); inv2[s].resize(m); logratio[s].resize(m);
    for (size_t j = 0; j < m; ++j) inv1[s][j] = 1.0 / pix1[s][j];
    for (size_t j = 0; j < m; ++j) inv2[s][j] = 1.0 / pix2[s][j];
    for (size_t j = 0; j < m; ++j)
      logratio[s][j] = std::log(pix1[s][j] * inv2[s][j]);
    double lo = pix1[s][0], hi = pix1[s][0];
    for (size_t j = 1; j < m; ++j) {
      const double v = pix1[s][j];
      if (v > hi) hi = v; else if (v < lo) lo = v;
    }
    minbm1[s] = lo; maxbm1[s] = hi;
    lo = hi = pix2[s][0];
    for (size_t j = 1; j < m; ++j) {
      const double v = pix2[s][j];
      if (v > hi) hi = v; else if (v < lo) lo = v;
    }
    minbm2[s] = lo; maxbm2[s] = hi;
  }
}

// 2D log2 histogram, components with at least 30 pixels:
// doublebeam.cc:467-584; log ratios doublebeam.cc:750-772.
void Beam2::histogram(unsigned nbins) {
  if (!hasData()) throw Error(POFD_E_ARG, "Trying to histogram empty beam");
  if (nbins == 0) throw Error(POFD_E_ARG, "Invalid (zero) NBINS");
  const double pad = 0.0014419741739063218;
  const unsigned nb2 = nbins * nbins;
  const double dn = static_cast<double>(nbins);
  for (int s = 0; s < 4; ++s) {
    ishist[s] = false;
    binwt[s].clear(); binv1[s].clear(); binv2[s].clear(); binlogratio[s].clear();
    if (!(hassign[s] && pix1[s].size() >= 30)) continue;
    const double lo1 = std::log2(minbm1[s]) - pad, hi1 = std::log2(maxbm1[s]) + pad;
    const double is1 = dn / (hi1 - lo1);
    const double lo2 = std::log2(minbm2[s]) - pad, hi2 = std::log2(maxbm2[s]) + pad;
    const double is2 = dn / (hi2 - lo2);
    std::vector<unsigned> cnt(nb2, 0);
    std::vector<double> s1(nb2, 0.0), s2(nb2, 0.0);
    for (size_t i = 0; i < pix1[s].size(); ++i) {
      const double v1 = pix1[s][i], v2 = pix2[s][i];
      const unsigned i1 = static_cast<unsigned>((std::log2(v1) - lo1) * is1);
      const unsigned i2 = static_cast<unsigned>((std::log2(v2) - lo2) * is2);
      const unsigned t = i1 * nbins + i2;
      cnt[t] += 1; s1[t] += v1; s2[t] += v2;
    }
    for (unsigned t = 0; t < nb2; ++t) {
      if (!cnt[t]) continue;
      const double w = static_cast<double>(cnt[t]);
      binwt[s].push_back(w);
      binv1[s].push_back(w / s1[t]);
      binv2[s].push_back(w / s2[t]);
    }
    for (size_t i = 0; i < binwt[s].size(); ++i)
      binlogratio[s].push_back(std::log(binv2[s][i] / binv1[s][i]));
    ishist[s] = true;
  }
}

// ---------------------------------------------------------------- Data2
void Data2::meanSubtract() {
  const size_t n = d1.size();
  double m = d1[0];
  for (size_t i = 1; i < n; ++i) m += d1[i];
  m /= static_cast<double>(n);
  for (auto& v : d1) v -= m;
  if (binned) bc1 -= m;
  m = d2[0];
  for (size_t i = 1; i < n; ++i) m += d2[i];
  m /= static_cast<double>(n);
  for (auto& v : d2) v -= m;
  if (binned) bc2 -= m;
}

void Data2::minmax(double* mm) const {
  if (binned) {
    mm[0] = bc1; mm[1] = bc1 + static_cast<double>(nbins1 - 1) * bd1;
    mm[2] = bc2; mm[3] = bc2 + static_cast<double>(nbins2 - 1) * bd2;
    return;
  }
  mm[0] = mm[1] = d1[0];
  for (size_t i = 1; i < d1.size(); ++i) {
    if (d1[i] < mm[0]) mm[0] = d1[i];
    if (d1[i] > mm[1]) mm[1] = d1[i];
  }
  mm[2] = mm[3] = d2[0];
  for (size_t i = 1; i < d2.size(); ++i) {
    if (d2[i] < mm[2]) mm[2] = d2[i];
    if (d2[i] > mm[3]) mm[3] = d2[i];
  }
}

void Data2::applyBinning(unsigned nb1, unsigned nb2) {
  if (nb1 == 0 || nb2 == 0) throw Error(POFD_E_ARG, "Trying to bin with no bins");
  binned = false;
  double mm[4];
  minmax(mm);
  for (double v : mm)
    if (!std::isfinite(v)) throw Error(POFD_E_ARG, "Non-valid min or max");
  nbins1 = nb1; nbins2 = nb2;
  bins.assign(static_cast<size_t>(nb1) * nb2, 0u);
  bc1 = mm[0];
  bd1 = (nb1 == 1) ? 2 * (mm[1] - mm[0]) : (mm[1] - mm[0]) / static_cast<double>(nb1 - 1);
  bc2 = mm[2];
  bd2 = (nb2 == 1) ? 2 * (mm[3] - mm[2]) : (mm[3] - mm[2]) / static_cast<double>(nb2 - 1);
  const double ib1 = 1.0 / bd1, ib2 = 1.0 / bd2;
  for (size_t i = 0; i < d1.size(); ++i) {
    const unsigned i1 = static_cast<unsigned>((d1[i] - bc1) * ib1 + 0.5);
    const unsigned i2 = static_cast<unsigned>((d2[i] - bc2) * ib2 + 0.5);
    bins[static_cast<size_t>(i1) * nb2 + i2] += 1;
  }
  binned = true;
}

// ----------------------------------------------------------- RGrid2Axis
void RGrid2Axis::init(unsigned N, double minflux, double maxflux) {
  n = N;
  flux.assign(N, 0.0);
  const double inm1 = 1.0 / static_cast<double>(N - 1);
  dflux = (maxflux - minflux) * inm1;
  if (minflux >= 0.0) {
    flux[0] = minflux;
    for (unsigned i = 1; i < N; ++i) flux[i] = static_cast<double>(i) * dflux + minflux;
    wrapidx = N - 1;
  } else {
    dflux = maxflux / (N - std::floor(-minflux / dflux) - 1.0);
    wrapidx = static_cast<unsigned>(maxflux / dflux + 0.999999999);
    flux[0] = 0.0;
    for (unsigned i = 1; i <= wrapidx; ++i) flux[i] = static_cast<double>(i) * dflux;
    const double wrapval = -static_cast<double>(N) * dflux;
    for (unsigned i = wrapidx + 1; i < N; ++i)
      flux[i] = static_cast<double>(i) * dflux + wrapval;
  }
}

}  // namespace pofd

namespace pofd {

// ------------------------------------------------------------- NatSpline
void NatSpline::init(const double* xa, const double* ya, size_t n) {
  if (n < 3) throw Error(POFD_E_ARG, "spline needs at least 3 points");
  SplineSystem sys;
  std::vector<double> xv(xa, xa + n);
  sys.factor(xv);
  x = xv;
  y.assign(ya, ya + n);
  const size_t N = n - 2;
  std::vector<double> cc(n, 0.0), z(N);
  for (size_t i = 0; i < N; ++i)
    z[i] = 3.0 * ((y[i + 2] - y[i + 1]) * sys.ih[i + 1] - (y[i + 1] - y[i]) * sys.ih[i]);
  for (size_t i = 1; i < N; ++i) z[i] = z[i] - sys.gamma[i - 1] * z[i - 1];
  for (size_t i = 0; i < N; ++i) z[i] = z[i] / sys.alpha[i];
  cc[N] = z[N - 1];
  for (size_t k = N - 1; k-- > 0;) cc[1 + k] = z[k] - sys.gamma[k] * cc[2 + k];
  b.assign(n - 1, 0.0);
  c.assign(n, 0.0);
  d.assign(n - 1, 0.0);
  for (size_t i = 0; i < n; ++i) c[i] = cc[i];
  for (size_t i = 0; i + 1 < n; ++i) {
    const double dx = x[i + 1] - x[i], dy = y[i + 1] - y[i];
    b[i] = (dy / dx) - dx * (c[i + 1] + 2.0 * c[i]) / 3.0;
    d[i] = (c[i + 1] - c[i]) / (3.0 * dx);
  }
}

size_t NatSpline::find(double v) const {
  size_t lo = 0, hi = x.size() - 1;
  while (hi > lo + 1) {
    const size_t m = (hi + lo) / 2;
    if (x[m] > v) hi = m; else lo = m;
  }
  return lo;
}

double NatSpline::eval(double v) const {
  const size_t i = find(v);
  const double dl = v - x[i];
  return y[i] + dl * (b[i] + dl * (c[i] + dl * d[i]));
}

// ---------------------------------------------------------- Model2Host
void Model2Host::set(const std::vector<double>& k, const std::vector<double>& s,
                     const std::vector<double>& o, const float* th) {
  knots = k;
  sigk = s;
  offk = o;
  const size_t nk = k.size(), ns = s.size(), no = o.size();
  for (size_t i = 0; i < nk; ++i)
    if (std::isnan(static_cast<double>(th[i])))
      throw Error(POFD_E_INVALID_MODEL, "Model is not valid");
  sigv.resize(ns);
  offv.resize(no);
  for (size_t i = 0; i < ns; ++i) {
    sigv[i] = static_cast<double>(th[nk + i]);
    if (!std::isfinite(sigv[i])) throw Error(POFD_E_INVALID_MODEL, "Model is not valid");
  }
  for (size_t i = 0; i < no; ++i) {
    offv[i] = static_cast<double>(th[nk + ns + i]);
    if (std::isnan(offv[i])) throw Error(POFD_E_INVALID_MODEL, "Model is not valid");
  }
  if (ns > 2) sigspl.init(sigk.data(), sigv.data(), ns);
  if (no > 2) offspl.init(offk.data(), offv.data(), no);
}

double Model2Host::sigma(double f1) const {
  const size_t ns = sigk.size();
  if (ns == 1) return sigv[0];
  if (f1 <= sigk[0]) return sigv[0];
  if (f1 >= sigk[ns - 1]) return sigv[ns - 1];
  double val;
  if (ns == 2) {
    val = sigv[0] + (f1 - sigk[0]) / (sigk[1] - sigk[0]) * (sigv[1] - sigv[0]);
  } else {
    val = sigspl.eval(f1);
  }
  return (val < min_sigma) ? min_sigma : val;
}

double Model2Host::offset(double f1) const {
  const size_t no = offk.size();
  if (no == 1) return offv[0];
  if (f1 <= offk[0]) return offv[0];
  if (f1 >= offk[no - 1]) return offv[no - 1];
  if (no == 2)
    return offv[0] + (f1 - offk[0]) / (offk[1] - offk[0]) * (offv[1] - offv[0]);
  return offspl.eval(f1);
}

namespace {
struct LogNormF {
  double mu, isig, isig2, target;
  double operator()(double u) const {
    const double prefac = 1.0 / std::sqrt(2 * kPi);
    const double eu = std::exp(-u);
    const double arg = u - mu;
    return prefac * std::exp(-0.5 * arg * arg * isig2) * isig * eu - target;
  }
};
}  // namespace

// Brent's method (Brent 1973, ch. 4) with the bracket and the relative
// interval test the reference applies (numberCountsDoubleLogNormal.cc:
// 1426-1471).
double Model2Host::logNormalSolver(double mu, double sig, double nsig) const {
  const double prefac = 1.0 / std::sqrt(kTwoPi);
  if (sig <= 0.0) throw Error(POFD_E_ARG, "Invalid (non-positive) sigma");
  const double sig2 = sig * sig;
  const double mode_u = mu - sig2;
  if (nsig == 0) return std::exp(mode_u);
  const double isig = 1.0 / sig;
  const double val_mode = prefac * isig * std::exp(0.5 * sig2 - mu);
  LogNormF F{mu, isig, isig * isig, val_mode * std::exp(-0.5 * nsig * nsig)};
  double u_low = mode_u;
  double delta_u = std::log(std::exp(mode_u) + 2 * sig) - mode_u;
  double fval = F(u_low + delta_u);
  if (fval >= 0.0) {
    for (int i = 0; i < 20; ++i) {
      delta_u *= 1.5;
      fval = F(u_low + delta_u);
      if (fval < 0.0) break;
    }
    if (fval >= 0.0) throw Error(POFD_E_ARG, "Unable to bracket Log Normal");
  }
  double u_high = u_low + delta_u;
  // Brent state
  double a = u_low, b = u_high, c = u_high;
  double fa = F(a), fb = F(b), fc = fb;
  double d = b - a, e = b - a;
  if ((fa < 0.0 && fb < 0.0) || (fa > 0.0 && fb > 0.0))
    throw Error(POFD_E_ARG, "endpoints do not straddle y=0");
  const double eps = 2.2204460492503131e-16;
  double root = 0.5 * (u_low + u_high);
  for (int it = 0; it < 20; ++it) {
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
    const double tol = 0.5 * eps * std::fabs(b);
    const double m = 0.5 * (c - b);
    double xl, xu;
    if (fb == 0 || std::fabs(m) <= tol) {
      root = b;
      xl = (b < c) ? b : c;
      xu = (b < c) ? c : b;
      if (fb == 0) xl = xu = b;
    } else {
      if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
        d = m; e = m;
      } else {
        double p, q, r;
        const double s = fb / fa;
        if (ac_equal) {
          p = 2 * m * s;
          q = 1 - s;
        } else {
          q = fa / fc;
          r = fb / fc;
          p = s * (2 * m * q * (q - r) - (b - a) * (r - 1));
          q = (q - 1) * (r - 1) * (s - 1);
        }
        if (p > 0) q = -q; else p = -p;
        const double l1 = 3 * m * q - std::fabs(tol * q), l2 = std::fabs(e * q);
        if (2 * p < (l1 < l2 ? l1 : l2)) { e = d; d = p / q; }
        else { d = m; e = m; }
      }
      a = b; fa = fb;
      if (std::fabs(d) > tol) b += d; else b += (m > 0 ? +tol : -tol);
      fb = F(b);
      root = b;
      double cc = c;
      if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) cc = a;
      xl = (b < cc) ? b : cc;
      xu = (b < cc) ? cc : b;
    }
    const double al = std::fabs(xl), au = std::fabs(xu);
    const double min_abs = ((xl > 0 && xu > 0) || (xl < 0 && xu < 0)) ? (al < au ? al : au) : 0.0;
    if (std::fabs(xu - xl) < 1e-3 * min_abs) return std::exp(root);
  }
  throw Error(POFD_E_ARG, "Unable to brent bracket Log Normal");
}

std::pair<double, double> Model2Host::maxFlux() const {
  const double kv = knots.back();
  return {kv, kv * logNormalSolver(offset(kv), sigma(kv), 3.0)};
}

void Model2Host::rrange(const Beam2& bm, double* r) const {
  double min1 = 0, max1 = 0, min2 = 0, max2 = 0, cv;
  const auto mf = maxFlux();
  if (bm.hassign[0]) {
    cv = mf.first * bm.maxbm1[0]; if (cv > max1) max1 = cv;
    cv = mf.second * bm.maxbm2[0]; if (cv > max2) max2 = cv;
  }
  if (bm.hassign[1]) {
    cv = mf.first * bm.maxbm1[1]; if (cv > max1) max1 = cv;
    cv = -mf.second * bm.maxbm2[1]; if (cv < min2) min2 = cv;
  }
  if (bm.hassign[2]) {
    cv = -mf.first * bm.maxbm1[2]; if (cv < min1) min1 = cv;
    cv = mf.second * bm.maxbm2[2]; if (cv > max2) max2 = cv;
  }
  if (bm.hassign[3]) {
    cv = -mf.first * bm.maxbm1[3]; if (cv < min1) min1 = cv;
    cv = -mf.second * bm.maxbm2[3]; if (cv < min2) min2 = cv;
  }
  r[0] = min1; r[1] = max1; r[2] = min2; r[3] = max2;
}

void gauss_legendre(int q, std::vector<double>& x, std::vector<double>& w) {
  if (q < 1) throw Error(POFD_E_ARG, "quadrature order must be positive");
  x.assign(q, 0.0);
  w.assign(q, 0.0);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < (q + 1) / 2; ++i) {
    // initial guess (Tricomi) for the i-th largest root, then Newton
    long double t = std::cos(pi * (i + 0.75L) / (q + 0.5L));
    long double dp = 1.0L;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1.0L, p1 = t;
      for (int k = 2; k <= q; ++k) {
        const long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      // P_q = p1, P_{q-1} = p0; P_q' = q (t P_q - P_{q-1}) / (t^2 - 1)
      dp = q * (t * p1 - p0) / (t * t - 1.0L);
      const long double dt = p1 / dp;
      t -= dt;
      if (std::fabs(static_cast<double>(dt)) < 1e-19) break;
    }
    long double p0 = 1.0L, p1 = t;
    for (int k = 2; k <= q; ++k) {
      const long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = (q == 1) ? 1.0L : q * (t * p1 - p0) / (t * t - 1.0L);
    const long double wt = 2.0L / ((1.0L - t * t) * dp * dp);
    x[q - 1 - i] = static_cast<double>(t);
    x[i] = static_cast<double>(-t);
    w[i] = w[q - 1 - i] = static_cast<double>(wt);
  }
}

void KnotQuadrature::build(const double* logknots, int K, int panels, int q) {
  build_breaks(logknots, K, {}, panels, q);
}

void KnotQuadrature::build_breaks(const double* logknots, int K, std::vector<double> extra,
                                  int panels, int q) {
  std::vector<double> gx, gw;
  gauss_legendre(q, gx, gw);
  nper = panels * q;
  u.clear();
  s.clear();
  w.clear();
  kidx.clear();
  if (K < 2) return;
  std::vector<double> br(logknots, logknots + K);
  for (double e : extra)
    if (e > logknots[0] && e < logknots[K - 1]) br.push_back(e);
  std::sort(br.begin(), br.end());
  br.erase(std::unique(br.begin(), br.end()), br.end());
  const long double ln2 = 0.693147180559945309417232121458176568L;
  int k = 0;
  for (size_t i = 0; i + 1 < br.size(); ++i) {
    while (k + 2 < K && br[i] >= logknots[k + 1]) ++k;
    const long double a = br[i], b = br[i + 1];
    const long double h = (b - a) / panels;
    for (int p = 0; p < panels; ++p) {
      const long double lo = a + p * h;
      for (int g = 0; g < q; ++g) {
        const long double uu = lo + 0.5L * h * (gx[g] + 1.0L);
        u.push_back(static_cast<double>(uu));
        s.push_back(static_cast<double>(std::exp2(uu)));
        w.push_back(static_cast<double>(ln2 * 0.5L * h * gw[g]));
        kidx.push_back(k);
      }
    }
  }
}

}  // namespace pofd
