// pofd_oracle.cc -- CPU FP64 restatement of pofd_affine's P(D) likelihood
// path (reference version 0.5.1), used as the checker for the CUDA path.
//
// TEST INFRASTRUCTURE ONLY: see pofd_oracle.h.  Parity status: the counts,
// R and R-range pieces are pinned by the reference's own golden values
// (test/model_test.cc); the full P(D) and log-likelihood have no reference
// golden vectors (the reference's tests never call PDFactory or calcLike and
// the reference cannot be built here: GSL, FFTW, cfitsio, HDF5 and MPI are
// absent), so at that level this restatement is the parity anchor.
//
// Every function cites the reference file:line it restates.  Deliberate,
// documented departures (all at places where the reference has undefined
// behaviour or calls a library whose behaviour is not defined there):
//   * spline evaluations one rounding step outside the node range are
//     evaluated on the end interval instead of aborting (GSL would raise
//     EDOM and abort the program);
//   * split-point neighbour scans clamp indices to the array (the 1D
//     reference may read pofd[-3], PDFactory.cc:858);
//   * the 2D binned likelihood clamps the bilinear cell to the grid (the
//     reference may read one row past the array, PDDouble.cc:1171);
//   * c2r inputs: the self-conjugate DC/Nyquist bins (1D) and columns (2D)
//     are reduced to their Hermitian part before the inverse DFT.
#include "pofd_oracle.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <thread>

#include "numerics.hh"

namespace orc {

// global_settings.h:24-26, 67-74
const double kPi = 3.141592653589793238462643383279502884197;
const double kTwoPi = 2.0 * kPi;
const double kLogfac = std::log2(10.0);
const double kSmallLogVal = -30.0;
const double kLog2toe = std::log(2.);
const double kILog2toe = 1.0 / std::log(2.);
const double kNZeroPad = 7.5;
const double kNaN = std::numeric_limits<double>::quiet_NaN();
const double kBadLike = 1e25;  // calcLike.h:71

thread_local std::string g_err;

// Error codes shared with the product library's status codes.
enum {
  E_INVALID_MODEL = -1,
  E_SPLIT_RANGE = -2,
  E_SPLIT_PEAK = -3,
  E_SPLIT_MIN = -4,
  E_SPLIT_LOGIC = -5,
  E_SPLIT_TOP = -6,
  E_SPLIT_NONE = -7,
  E_UNSHIFT = -8,
  E_ARG = -10,
};

// ============================================================ 1D beam
// beam.cc:295-458 (readFile; the pixel array replaces the FITS read) and
// beam.cc:467-556 (makeHistogram).
struct Beam1 {
  static constexpr unsigned histothresh = 20;  // beam.h:31
  bool haspos = false, hasneg = false;
  double pixsize = 0, minval = 0;
  std::vector<double> pos, neg, posinv, neginv;
  double totpos = 0, totpossq = 0, totneg = 0, totnegsq = 0;
  bool posh = false, negh = false;
  std::vector<double> poswt, posval, negwt, negval;

  void set(const double* pix, size_t n, double PIXSIZE, double MINVAL) {
    minval = (MINVAL <= 0.0) ? 0.0 : MINVAL;
    const double negminval = -minval;
    pixsize = PIXSIZE;
    pos.clear(); neg.clear();
    for (size_t i = 0; i < n; ++i) {
      const double v = pix[i];
      if (std::isnan(v) || std::isinf(v)) continue;
      if (v > minval) pos.push_back(v);
      if (v < negminval) neg.push_back(std::fabs(v));
    }
    if (pos.empty() && neg.empty())
      throw OrcError(E_ARG, "Beam file has only zero values");
    haspos = !pos.empty();
    hasneg = !neg.empty();
    std::sort(pos.begin(), pos.end());
    std::sort(neg.begin(), neg.end());
    if (haspos) {
      totpos = pos[0]; totpossq = totpos * totpos;
      for (size_t i = 1; i < pos.size(); ++i) {
        totpos += pos[i]; totpossq += pos[i] * pos[i];
      }
    }
    if (hasneg) {
      totneg = neg[0]; totnegsq = totneg * totneg;
      for (size_t i = 1; i < neg.size(); ++i) {
        totneg += neg[i]; totnegsq += neg[i] * neg[i];
      }
    }
    posinv.resize(pos.size());
    for (size_t i = 0; i < pos.size(); ++i) posinv[i] = 1.0 / pos[i];
    neginv.resize(neg.size());
    for (size_t i = 0; i < neg.size(); ++i) neginv[i] = 1.0 / neg[i];
    posh = negh = false;
  }

  static void hist(const std::vector<double>& arr, unsigned nbins,
                   std::vector<double>& wt, std::vector<double>& val) {
    const double log2outscale = 0.0014419741739063218;  // log2(1.001)
    const size_t np = arr.size();
    const double minlog2val = std::log2(arr[0]) - log2outscale;
    const double maxlog2val = std::log2(arr[np - 1]) + log2outscale;
    const double histstep =
        (maxlog2val - minlog2val) / static_cast<double>(nbins);
    std::vector<unsigned> tw(nbins, 0);
    std::vector<double> tv(nbins, 0.0);
    for (size_t i = 0; i < np; ++i) {
      const double cv = arr[i];
      const unsigned idx =
          static_cast<unsigned>((std::log2(cv) - minlog2val) / histstep);
      tw[idx] += 1;
      tv[idx] += cv;
    }
    wt.clear(); val.clear();
    for (unsigned i = 0; i < nbins; ++i)
      if (tw[i] > 0) {
        const double w = static_cast<double>(tw[i]);
        wt.push_back(w);
        val.push_back(tv[i] / w);
      }
    for (auto& v : val) v = 1.0 / v;
  }

  void makeHistogram(unsigned nbins) {
    if (nbins == 0) throw OrcError(E_ARG, "Invalid (non-positive) nbins");
    posh = negh = false;
    poswt.clear(); posval.clear(); negwt.clear(); negval.clear();
    const bool do_pos = haspos && pos.size() >= histothresh;
    const bool do_neg = hasneg && neg.size() >= histothresh;
    if (do_pos) { hist(pos, nbins, poswt, posval); posh = true; }
    if (do_neg) { hist(neg, nbins, negwt, negval); negh = true; }
  }

  double maxpos() const { return haspos ? pos.back() : kNaN; }
  double maxneg() const { return hasneg ? neg.back() : kNaN; }

  // The (weight, inverse beam) lists the array getR sums over
  // (numberCountsKnotsSpline.cc:463-477).  The negative side asks
  // beam::isNegHist(), which returns the *positive* flag (beam.h:86): when
  // the positive beam is histogrammed the negative side uses the negative
  // histogram (empty if that side was too small to histogram).
  void terms(bool negside, bool& hashist, const std::vector<double>*& w,
             const std::vector<double>*& iv) const {
    if (!negside) {
      hashist = posh;
      w = posh ? &poswt : nullptr;
      iv = posh ? &posval : &posinv;
    } else {
      hashist = posh;  // isNegHist() quirk
      w = posh ? &negwt : nullptr;
      iv = posh ? &negval : &neginv;
    }
  }
};

// ================================================ 1D counts: knots spline
// numberCountsKnots.cc:257-284 (setParams/isValid), 345-365 (R range);
// numberCountsKnotsSpline.cc:265-289 (setParams, counts), 352-529 (getR).
struct Counts1 {
  std::vector<double> knots, logknots, logknotvals;
  NatSpline spl;
  bool loaded = false;

  void setKnots(int n, const double* kp) {
    knots.assign(kp, kp + n);
    logknots.resize(n);
    for (int i = 0; i < n; ++i) logknots[i] = std::log2(knots[i]);
    logknotvals.assign(n, kNaN);
    loaded = false;
  }
  void setParams(const float* F, int npar) {
    const int n = static_cast<int>(knots.size());
    if (n > npar) throw OrcError(E_ARG, "Number of knot values different than expected");
    for (int i = 0; i < n; ++i)
      logknotvals[i] = kLogfac * static_cast<double>(F[i]);
    loaded = true;
    bool finite = true;
    for (double v : logknotvals) if (std::isnan(v)) finite = false;
    if (finite) spl.init(logknots.data(), logknotvals.data(), n);
  }
  bool isValid() const {
    const size_t n = knots.size();
    if (n == 0 || !loaded) return false;
    for (double k : knots) if (std::isnan(k)) return false;
    if (knots[0] <= 0.0) return false;
    for (size_t i = 1; i < n; ++i) if (knots[i] <= knots[i - 1]) return false;
    for (double v : logknotvals) if (std::isnan(v)) return false;
    return true;
  }
  double minflux() const { return knots.front(); }
  double maxflux() const { return knots.back(); }
  double counts(double s) const {
    if (knots.size() < 2 || !isValid()) return kNaN;
    if (s < knots.front() || s >= knots.back()) return 0.0;
    return std::exp2(spl.eval(std::log2(s)));
  }
  std::pair<double, double> rrangeInternal(const Beam1& bm) const {
    const double maxknot = knots.back();
    double minRF, maxRF;
    if (bm.haspos) {
      maxRF = maxknot * bm.maxpos();
      minRF = bm.hasneg ? -maxknot * bm.maxneg() : 0.0;
    } else {
      maxRF = 0.0;
      minRF = -maxknot * bm.maxneg();
    }
    return {minRF, maxRF};
  }
  std::pair<double, double> rrange(const Beam1& bm) const {
    if (!isValid()) throw OrcError(E_INVALID_MODEL, "Model is not valid");
    return rrangeInternal(bm);
  }
  // Array getR, numberCountsKnotsSpline.cc:436-529.
  void getR(size_t n, const double* flux, const Beam1& bm, double* R) const {
    if (n == 0) return;
    if (!isValid()) {
      for (size_t i = 0; i < n; ++i) R[i] = kNaN;
      return;
    }
    const auto rr = rrangeInternal(bm);
    const double minknot = knots.front(), maxknot = knots.back();
    double prefac = bm.pixsize / 3600.0;
    prefac = prefac * prefac;
    bool ph, nh;
    const std::vector<double>*pw, *pv, *nw, *nv;
    bm.terms(false, ph, pw, pv);
    bm.terms(true, nh, nw, nv);
    for (size_t i = 0; i < n; ++i) {
      const double f = flux[i];
      double workval = 0.0;
      if (f > 0 && bm.haspos && f <= rr.second) {
        for (size_t j = 0; j < pv->size(); ++j) {
          const double ieta = (*pv)[j];
          const double currarg = f * ieta;
          if (currarg < minknot || currarg >= maxknot) continue;
          const double cts = std::exp2(spl.eval(std::log2(currarg)));
          if (cts > 0) {
            if (ph) workval += (*pw)[j] * cts * ieta;
            else workval += cts * ieta;
          }
        }
      } else if (bm.hasneg && f < 0 && f >= rr.first) {
        for (size_t j = 0; j < nv->size(); ++j) {
          const double ieta = (*nv)[j];
          const double currarg = -f * ieta;
          if (currarg < minknot || currarg >= maxknot) continue;
          const double cts = std::exp2(spl.eval(std::log2(currarg)));
          if (cts > 0) {
            if (nh) workval += (*nw)[j] * cts * ieta;
            else workval += cts * ieta;
          }
        }
      }
      R[i] = prefac * workval;
    }
  }
  // Scalar getR, numberCountsKnotsSpline.cc:352-427.
  double getRScalar(double f, const Beam1& bm) const {
    if (!isValid()) return kNaN;
    if (f > 0 && !bm.haspos) return 0.0;
    else if (f < 0 && !bm.hasneg) return 0.0;
    else if (f == 0) return 0.0;
    const double minknot = knots.front(), maxknot = knots.back();
    const auto rr = rrangeInternal(bm);
    if (f >= rr.second) return 0.0;
    if (f <= rr.first) return 0.0;
    double prefac = bm.pixsize / 3600.0;
    prefac = prefac * prefac;
    double retval = 0.0;
    const bool negside = f < 0;
    bool hh;
    const std::vector<double>*w, *iv;
    bm.terms(negside, hh, w, iv);
    const double af = negside ? -f : f;
    for (size_t i = 0; i < iv->size(); ++i) {
      const double ieta = (*iv)[i];
      const double currarg = af * ieta;
      if (currarg < minknot || currarg >= maxknot) continue;
      const double cts = std::exp2(spl.eval(std::log2(currarg)));
      if (hh) retval += (*w)[i] * ieta * cts;
      else retval += cts * ieta;
    }
    return prefac * retval;
  }
  // numberCountsKnotsSpline::differenceRegularize (numberCountsKnotsSpline.cc:
  // 540-559): minus alpha times the spread of the log2-log2 slopes.
  double differenceRegularize(double alpha) const {
    const size_t nk = knots.size();
    if (nk < 2) return 0.0;
    double mean_deriv = 0.0;
    for (size_t i = 1; i < nk; ++i)
      mean_deriv += (logknotvals[i] - logknotvals[i - 1]) / (logknots[i] - logknots[i - 1]);
    mean_deriv /= static_cast<double>(nk - 1);
    double pen = 0.0;
    for (size_t i = 1; i < nk; ++i) {
      const double d = (logknotvals[i] - logknotvals[i - 1]) / (logknots[i] - logknots[i - 1]) -
                       mean_deriv;
      pen -= d * d;
    }
    return alpha * pen;
  }
  // Integral of S^alpha dN/dS over the knot range
  // (numberCountsKnotsSpline.cc:300-343 integrates the same function with
  // adaptive GK41 to epsrel 1e-5; here a fixed high-order Gauss-Legendre
  // rule in ln S, accurate well beyond that tolerance).
  double splineInt(double alpha) const {
    if (knots.size() < 2 || !isValid()) return kNaN;
    std::vector<double> gx, gw;
    gauss_legendre(20, gx, gw);
    double tot = 0.0;
    for (size_t k = 0; k + 1 < knots.size(); ++k) {
      const double a = std::log(knots[k]), b = std::log(knots[k + 1]);
      const int npanel = 64;
      const double h = (b - a) / npanel;
      for (int p = 0; p < npanel; ++p) {
        const double lo = a + p * h;
        for (int g = 0; g < 20; ++g) {
          const double u = lo + 0.5 * h * (gx[g] + 1.0);
          const double s = std::exp(u);
          double c = (s >= knots.back()) ? 0.0
                                         : std::exp2(spl.eval(std::log2(s)));
          tot += 0.5 * h * gw[g] * std::pow(s, alpha + 1.0) * c;
        }
      }
    }
    return tot;
  }
};

// ============================================================ 1D P(D)
// PD.cc:123-184 (integral/normalise/log), 245-274 (mean), 557-677
// (binned/unbinned log-likelihood).
struct PD1 {
  std::vector<double> pd;
  double minflux = 0, dflux = 1;
  bool logflat = false;

  double integral() const {
    const size_t n = pd.size();
    if (n == 0) return kNaN;
    double tot = 0.5 * pd[0];
    for (size_t i = 1; i < n - 1; ++i) tot += pd[i];
    tot += 0.5 * pd[n - 1];
    return tot * dflux;
  }
  void normalize() {
    if (pd.empty()) throw OrcError(E_ARG, "No information present to normalize");
    const double tot = integral();
    const double itot = 1.0 / tot;
    for (auto& v : pd) v *= itot;
  }
  void applyLog() {
    if (logflat) return;
    for (auto& v : pd) v = (v > 0.0) ? std::log2(v) : kSmallLogVal;
    logflat = true;
  }
  double meanNoNorm() const {
    const size_t n = pd.size();
    if (n == 0) return kNaN;
    double mean = 0.0;
    for (size_t i = 1; i < n - 1; ++i) mean += static_cast<double>(i) * pd[i];
    mean += 0.5 * static_cast<double>(n - 1) * pd[n - 1];
    mean *= dflux * dflux;
    mean += minflux;
    return mean;
  }
  double logLikeBinned(const std::vector<unsigned>& bins, double bincent0,
                       double bindelta) const {
    const size_t n = pd.size();
    const double maxflux = minflux + static_cast<double>(n - 1) * dflux;
    const double idflux = 1.0 / dflux;
    const double maxfluxval = maxflux - dflux;
    double loglike = 0.0;
    for (size_t i = 0; i < bins.size(); ++i) {
      const unsigned ninbin = bins[i];
      if (ninbin == 0) continue;
      const double cflux = bincent0 + static_cast<double>(i) * bindelta;
      if (cflux < minflux) loglike += static_cast<double>(ninbin) * pd[0];
      else if (cflux > maxfluxval)
        loglike += static_cast<double>(ninbin) * pd[n - 1];
      else {
        const double delt = (cflux - minflux) * idflux;
        const int idx = static_cast<int>(delt);
        const double t = delt - static_cast<double>(idx);
        loglike += ((1.0 - t) * pd[idx] + t * pd[idx + 1]) *
                   static_cast<double>(ninbin);
      }
    }
    return kLog2toe * loglike;
  }
  double logLikeUnbinned(const std::vector<double>& flux) const {
    const size_t n = pd.size();
    const double maxflux = minflux + static_cast<double>(n - 1) * dflux;
    const double idflux = 1.0 / dflux;
    const double maxfluxval = maxflux - dflux;
    double loglike = 0.0;
    for (double cflux : flux) {
      if (cflux <= minflux) loglike += pd[0];
      else if (cflux >= maxfluxval) loglike += pd[n - 1];
      else {
        const double delt = (cflux - minflux) * idflux;
        const int idx = static_cast<int>(delt);
        const double t = delt - static_cast<double>(idx);
        loglike += (1.0 - t) * pd[idx] + t * pd[idx + 1];
      }
    }
    return kLog2toe * loglike;
  }
};

// ===================================================== 1D P(D) factory
// PDFactory.cc:361-414 (initRFlux), 426-527 (initRInterp), 541-620 (initR),
// 625-679 (getMeanVarFromR), 691-921 (findSplitPoint), 934-1009
// (unwrapAndNormalizePD), 1031-1141 (initPD), 1154-1243 (getPD).
struct PDF1 {
  static constexpr double subedgemult = 1e-5;  // PDFactory.h:30
  unsigned ninterp = 2048;
  unsigned n = 0;
  double dflux = 0, minflux_R = 0;
  unsigned wrapRidx = 0;
  std::vector<double> rvals, pofd;
  std::vector<cplx> prtrans, pval;
  NatSpline spos, sneg;
  std::vector<double> xpos, ypos, xneg, yneg;  // R nodes (log2 R in y)
  std::vector<double> rpos, rneg;              // R nodes before the log
  double mn = kNaN, var_noi = kNaN, sgpos = kNaN, sgneg = kNaN;
  bool doshift = false;
  double shift = 0.0;
  unsigned lastsplit = 0;

  void initRFlux(unsigned N, double minflux, double maxflux) {
    if (N == 0) throw OrcError(E_ARG, "Invalid (0) n");
    if (maxflux < minflux) std::swap(minflux, maxflux);
    n = N;
    if (N == 1) {
      if (minflux < 0.0) throw OrcError(E_ARG, "n must be > 1 with negative fluxes");
      dflux = maxflux - minflux; minflux_R = minflux; wrapRidx = 0;
      return;
    }
    const double inm1 = 1.0 / static_cast<double>(N - 1);
    if (maxflux > 0) {
      if (minflux > 0) minflux = 0.0;
      if (minflux == 0) {
        wrapRidx = N - 1; minflux_R = 0.0; dflux = maxflux * inm1;
      } else {
        dflux = (maxflux - minflux) * inm1;
        dflux = maxflux / (N - std::floor(-minflux / dflux) - 1.0);
        wrapRidx = static_cast<unsigned>(maxflux / dflux + 0.9999999999);
        minflux_R = (wrapRidx + 1) * dflux - static_cast<double>(N) * dflux;
      }
    } else {
      if (minflux >= 0) throw OrcError(E_ARG, "No effective range in R fluxes");
      dflux = -minflux * inm1; wrapRidx = 0; minflux_R = minflux;
    }
  }

  void initRInterp(const Counts1& model, const Beam1& bm) {
    if (!(bm.haspos || bm.hasneg))
      throw OrcError(E_ARG, "Beam has neither positive nor negative bits");
    const double modelmin = model.minflux(), modelmax = model.maxflux();
    const double ininterpm1 = 1.0 / static_cast<double>(ninterp - 1);
    if (bm.haspos) {
      const double mininterpflux = modelmin * subedgemult;
      double maxinterpflux = modelmax * bm.maxpos();
      const double dinterp =
          0.001 * (maxinterpflux - mininterpflux) * ininterpm1;
      maxinterpflux -= dinterp;
      const double dinterpflux =
          (std::log2(maxinterpflux / mininterpflux)) * ininterpm1;
      xpos.resize(ninterp); rpos.resize(ninterp); ypos.resize(ninterp);
      for (unsigned i = 0; i < ninterp; ++i)
        xpos[i] = mininterpflux * std::exp2(static_cast<double>(i) * dinterpflux);
      model.getR(ninterp, xpos.data(), bm, rpos.data());
      for (unsigned i = 0; i < ninterp; ++i) {
        const double v = rpos[i];
        ypos[i] = (v > 0) ? std::log2(v) : kSmallLogVal;
      }
      spos.init(xpos.data(), ypos.data(), ninterp);
    }
    if (bm.hasneg) {
      double maxinterpflux = -modelmin * subedgemult;
      double mininterpflux = -modelmax * bm.maxneg();
      const double dinterp =
          0.001 * (maxinterpflux - mininterpflux) * ininterpm1;
      mininterpflux += dinterp;
      maxinterpflux -= dinterp;
      const double dinterpflux =
          (std::log2(mininterpflux / maxinterpflux)) * ininterpm1;
      xneg.resize(ninterp); rneg.resize(ninterp); yneg.resize(ninterp);
      for (unsigned i = 0; i < ninterp; ++i)
        xneg[i] = maxinterpflux *
                  std::exp2(static_cast<double>(ninterp - i - 1) * dinterpflux);
      model.getR(ninterp, xneg.data(), bm, rneg.data());
      for (unsigned i = 0; i < ninterp; ++i) {
        const double v = rneg[i];
        yneg[i] = (v > 0) ? std::log2(v) : kSmallLogVal;
      }
      sneg.init(xneg.data(), yneg.data(), ninterp);
    }
  }

  static double splineClamped(const NatSpline& s, double v) {
    const size_t nn = s.x.size();
    size_t i;
    if (v < s.x[0]) i = 0;
    else if (v > s.x[nn - 1]) i = nn - 2;
    else i = s.find(v);
    return s.eval_at(i, v);
  }

  void initR(unsigned N, double minflux, double maxflux, const Counts1& model,
             const Beam1& bm) {
    initRInterp(model, bm);
    initRFlux(N, minflux, maxflux);
    const bool haspos = bm.haspos && (maxflux > 0);
    const bool hasneg = bm.hasneg && (minflux < 0) && (wrapRidx > 0);
    rvals.assign(N, 0.0);
    if (haspos) {
      const double minI = xpos[0], maxI = xpos[ninterp - 1];
      const unsigned minitidx =
          static_cast<unsigned>(minI / dflux + 0.9999999999999999);
      unsigned maxitidx = static_cast<unsigned>(maxI / dflux);
      if (maxitidx > wrapRidx) maxitidx = wrapRidx;
      for (unsigned i = minitidx; i <= maxitidx; ++i) {
        const double cflux = static_cast<double>(i) * dflux;
        rvals[i] = std::exp2(splineClamped(spos, cflux));
      }
    }
    if (hasneg) {
      const double minI = xneg[0], maxI = xneg[ninterp - 1];
      unsigned minitidx = static_cast<unsigned>(
          (minI - minflux_R) / dflux + wrapRidx + 1 + 0.9999999999999999);
      if (minitidx <= wrapRidx) minitidx = wrapRidx + 1;
      unsigned maxitidx =
          static_cast<unsigned>((maxI - minflux_R) / dflux + wrapRidx + 1);
      if (maxitidx > N - 1) maxitidx = N - 1;
      const double mval = minflux_R - static_cast<double>(wrapRidx + 1) * dflux;
      for (unsigned i = minitidx; i <= maxitidx; ++i) {
        const double cflux = static_cast<double>(i) * dflux + mval;
        rvals[i] = std::exp2(splineClamped(sneg, cflux));
      }
    }
    for (unsigned i = 0; i < N; ++i) rvals[i] *= dflux;
  }

  void getMeanVarFromR() {
    double cf, prod;
    mn = 0.0; var_noi = 0.0;
    for (unsigned i = 1; i <= wrapRidx - 1; ++i) {
      cf = static_cast<double>(i) * dflux;
      prod = cf * rvals[i];
      mn += prod;
      var_noi += cf * prod;
    }
    cf = static_cast<double>(wrapRidx) * dflux;
    prod = 0.5 * cf * rvals[wrapRidx];
    mn += prod;
    var_noi += cf * prod;
    for (unsigned i = wrapRidx + 1; i < n; ++i) {
      cf = static_cast<double>(i - wrapRidx - 1) * dflux + minflux_R;
      prod = cf * rvals[i];
      mn += prod;
      var_noi += cf * prod;
    }
    if (wrapRidx < n - 1) {
      cf = minflux_R;
      prod = 0.5 * cf * rvals[wrapRidx - 1];  // reference reads wrapRidx-1
      mn -= prod;
      var_noi -= cf * prod;
    }
  }

  void initPD(unsigned N, double minflux, double maxflux, const Counts1& model,
              const Beam1& bm) {
    if (N == 0) throw OrcError(E_ARG, "Invalid (zero) n");
    if (N == 1) throw OrcError(E_ARG, "Invalid (==0) n");
    if (maxflux <= 0.0) throw OrcError(E_ARG, "Invalid (non-positive) maxflux");
    if (minflux == maxflux) throw OrcError(E_ARG, "Invalid (0) range between min/max flux");
    if (!model.isValid()) throw OrcError(E_INVALID_MODEL, "Invalid model");
    if (!(bm.haspos || bm.hasneg)) throw OrcError(E_ARG, "Empty beam");
    initR(N, minflux, maxflux, model, bm);
    getMeanVarFromR();
    sgpos = std::sqrt(var_noi);
    doshift = (sgpos > dflux) && (std::fabs(mn) > dflux);
    shift = doshift ? -mn : 0.0;
    const unsigned ncplx = N / 2 + 1;
    prtrans.assign(ncplx, 0.0);
    rfft(N, rvals.data(), prtrans.data());
    const double iflux = kTwoPi / (N * dflux);
    const double r0 = prtrans[0].real();
    prtrans[0] = cplx(1.0, 0.0);
    const double wfac = shift * iflux;
    for (unsigned idx = 1; idx < ncplx; ++idx) {
      const double expfac = std::exp(prtrans[idx].real() - r0);
      const double ival = doshift
          ? prtrans[idx].imag() - wfac * static_cast<double>(idx)
          : prtrans[idx].imag();
      prtrans[idx] = cplx(expfac * std::cos(ival), expfac * std::sin(ival));
    }
  }

  unsigned findSplitPoint() const {
    const double n1 = 2.5, f1 = 5e-14, f2 = 1e-5, f3 = 5;
    if (sgpos <= 0) throw OrcError(E_SPLIT_RANGE, "Invalid (non-positive) sigma positive");
    if (sgneg <= 0) throw OrcError(E_SPLIT_RANGE, "Invalid (non-positive) sigma negative");
    const int cs = static_cast<int>(n);
    const double fluxrange = n * dflux;
    const double n1sigpos = n1 * sgpos, n1signeg = n1 * sgneg;
    if (fluxrange < (n1sigpos + n1signeg))
      throw OrcError(E_SPLIT_RANGE, "Not enough flux range");
    double peak = pofd[0];
    for (unsigned i = 1; i < n; ++i) if (pofd[i] > peak) peak = pofd[i];
    if (peak <= 0.0) throw OrcError(E_SPLIT_PEAK, "Peak P(D) value was zero");
    int botidx, topidx;
    botidx = static_cast<int>(n1sigpos / dflux);
    if (n1sigpos > std::fabs(minflux_R)) topidx = wrapRidx;
    else
      topidx = static_cast<int>(-(n1signeg + minflux_R) / dflux + wrapRidx + 1);
    if (botidx >= cs) throw OrcError(E_SPLIT_LOGIC, "Logic error; invalid botidx (wrapped) in split search");
    if (topidx >= cs) throw OrcError(E_SPLIT_LOGIC, "Logic error; invalid (large) topidx in split search");
    int minidx = botidx;
    double minval = pofd[minidx];
    for (int i = botidx + 1; i <= topidx; ++i)
      if (pofd[i] < minval) { minidx = i; minval = pofd[i]; }
    if (minval > f2 * peak)
      throw OrcError(E_SPLIT_MIN, "Minimum in pd is too large relative to peak");
    const int pre_jitter_n = 17;
    double jitter = 0.0;
    if (minidx > pre_jitter_n) {
      bool mono = true;
      const int initidx = minidx - pre_jitter_n;
      double prevval;
      jitter = prevval = pofd[initidx];
      for (int i = initidx + 1; i < minidx; ++i) {
        const double cv = pofd[i];
        if (cv >= prevval) mono = false;
        jitter += cv;
        prevval = cv;
      }
      if (mono) return static_cast<unsigned>(minidx);
      jitter += minval;
      jitter = 1.1 * jitter / static_cast<double>(pre_jitter_n + 1);
    } else {
      jitter = f1 * peak;
      if (minval > jitter) return static_cast<unsigned>(minidx);
    }
    if (minval <= 0.0) {
      const int nminup = 3;
      int bi, ti;
      if (minidx < botidx) bi = botidx; else bi = minidx - nminup;
      if (minidx > topidx - nminup) ti = topidx - nminup; else ti = minidx + nminup;
      if (bi < 0) bi = 0;  // reference would read before the array
      for (int i = bi; i < ti; ++i) if (pofd[i] > minval) minval = pofd[i];
    }
    if (minval > 0) jitter = (f3 * minval) < jitter ? (f3 * minval) : jitter;
    if ((botidx >= topidx) || (std::abs(topidx - botidx) < 1))
      throw OrcError(E_SPLIT_LOGIC, "Topidx vs. botidx search issue");
    if (pofd[topidx] < jitter)
      throw OrcError(E_SPLIT_TOP, "Topidx is already below jitter estimate");
    for (int i = topidx - 1; i >= botidx; --i)
      if (pofd[i] < jitter) return static_cast<unsigned>(i + 1);
    throw OrcError(E_SPLIT_NONE, "Unable to find split point");
  }

  void getPD(double sigma, PD1& pd, bool setLog) {
    const unsigned ncplx = n / 2 + 1;
    pofd.assign(n, 0.0);
    if (sigma > 0) {
      const double iflux = kTwoPi / (n * dflux);
      const double sigfac = -0.5 * sigma * sigma;
      pval.assign(ncplx, 0.0);
      pval[0] = cplx(1.0, 0.0);
      for (unsigned idx = 1; idx < ncplx; ++idx) {
        const double w = iflux * static_cast<double>(idx);
        const double expfac = std::exp(sigfac * w * w);
        pval[idx] = cplx(expfac * prtrans[idx].real(), expfac * prtrans[idx].imag());
      }
      irfft(n, pval.data(), pofd.data());
    } else {
      irfft(n, prtrans.data(), pofd.data());
    }
    sgpos = std::sqrt(var_noi + sigma * sigma);
    if (9 * sigma * sigma > var_noi) sgneg = sigma; else sgneg = sgpos;
    // unwrapAndNormalizePD
    for (auto& v : pofd) if (v < 0) v = 0.0;
    const unsigned splitidx = findSplitPoint();
    lastsplit = splitidx;
    pd.pd.resize(n);
    std::memcpy(pd.pd.data(), pofd.data() + splitidx, (n - splitidx) * sizeof(double));
    std::memcpy(pd.pd.data() + n - splitidx, pofd.data(), splitidx * sizeof(double));
    pd.logflat = false;
    pd.minflux = 0.0;
    pd.dflux = dflux;
    pd.normalize();
    const double tmn = pd.meanNoNorm();
    if (std::isinf(tmn) || std::isnan(tmn))
      throw OrcError(E_UNSHIFT, "Un-shift amounts not finite");
    pd.minflux = -tmn;
    if (setLog) pd.applyLog();
  }
};

// ======================================================= 1D data binning
// fitsData.cc:380-437.
struct Data1 {
  std::vector<double> data;
  bool binned = false;
  unsigned nbins = 0;
  std::vector<unsigned> bins;
  double bincent0 = 0, bindelta = 0;
  void meanSubtract() {
    const size_t n = data.size();
    double mnval = data[0];
    for (size_t i = 1; i < n; ++i) mnval += data[i];
    mnval /= static_cast<double>(n);
    for (auto& v : data) v -= mnval;
    if (binned) bincent0 -= mnval;
  }
  std::pair<double, double> minmax() const {
    if (binned)
      return {bincent0, bincent0 + static_cast<double>(nbins - 1) * bindelta};
    double mn = data[0], mx = data[0];
    for (size_t i = 1; i < data.size(); ++i) {
      if (data[i] < mn) mn = data[i];
      if (data[i] > mx) mx = data[i];
    }
    return {mn, mx};
  }
  void applyBinning(unsigned NBINS) {
    if (data.empty()) return;
    if (NBINS == 0) throw OrcError(E_ARG, "Trying to bin with no bins");
    nbins = NBINS;
    bins.assign(nbins, 0);
    binned = false;
    const auto mm = minmax();
    bincent0 = mm.first;
    if (nbins == 1) bindelta = 2 * (mm.second - mm.first);
    else bindelta = (mm.second - mm.first) / static_cast<double>(nbins - 1);
    const double ibindelta = 1.0 / bindelta;
    for (double v : data) {
      const unsigned idx = static_cast<unsigned>((v - bincent0) * ibindelta + 0.5);
      bins[idx] += 1;
    }
    binned = true;
  }
};

// ============================================================ 1D likelihood
// calcLike.cc:283-371 (sigma base, R range), 389-443 (single getLogLike),
// 688-758 (readDataFromFiles grouping), 827-831, 884-955 (getLogLike).
struct BeamSet1 {
  Beam1 bm;
  std::vector<Data1> data;
  std::vector<double> sigma_base, like_offset, like_norm;
  double exp_conf = 0.0;
  double maxsigma_base = kNaN;
  double minDataFlux = kNaN, maxDataFlux = kNaN;
  double minRFlux = kNaN, maxRFlux = kNaN;
  PDF1 pdfac;
  PD1 pd;
};

struct Like1 {
  // per-thread copies used by eval_batch; rebuilt after any set-up change
  std::vector<std::shared_ptr<Like1>> pool;
  unsigned fftsize = 131072, ninterp = 2048, nbins = 1000;
  bool bin_data = true;
  Counts1 model;
  std::vector<BeamSet1> sets;
  // priors and regularisation (calcLike.h:96-116)
  bool has_sigma_prior = false, has_cfirb_prior = false, has_poisson_prior = false;
  double sigma_prior_width = 0, cfirb_prior_mean = 0, cfirb_prior_sigma = 0;
  double poisson_prior_mean = 0, poisson_prior_sigma = 0, regularization_alpha = 0;
  double mean_flux_per_area = kNaN, mean_fluxsq_per_area = kNaN;

  void refreshSet(BeamSet1& s) {
    s.maxsigma_base = s.sigma_base[0];
    for (size_t i = 1; i < s.sigma_base.size(); ++i)
      if (s.sigma_base[i] > s.maxsigma_base) s.maxsigma_base = s.sigma_base[i];
    for (size_t i = 0; i < s.data.size(); ++i) {
      const double var = s.sigma_base[i] * s.sigma_base[i] + s.exp_conf * s.exp_conf;
      if (var > 0) {
        const double ndd = static_cast<double>(s.data[i].data.size());
        s.like_offset[i] = -0.5 * ndd * (std::log(kTwoPi * var) + 1.0);
      }
    }
    auto mm = s.data[0].minmax();
    s.minDataFlux = mm.first; s.maxDataFlux = mm.second;
    for (size_t i = 1; i < s.data.size(); ++i) {
      mm = s.data[i].minmax();
      if (mm.first < s.minDataFlux) s.minDataFlux = mm.first;
      if (mm.second > s.maxDataFlux) s.maxDataFlux = mm.second;
    }
    s.minRFlux = s.maxRFlux = kNaN;
  }

  void setRRanges(const float* p, int npar) {
    model.setParams(p, npar);
    const double safetyfac = 1.05;
    for (auto& s : sets) {
      const auto raw = model.rrange(s.bm);
      const double sigma = std::sqrt(s.exp_conf * s.exp_conf +
                                     s.maxsigma_base * s.maxsigma_base);
      s.minRFlux = safetyfac * raw.first;
      s.maxRFlux = safetyfac * raw.second + kNZeroPad * sigma;
      if (s.minDataFlux < s.minRFlux && s.bm.hasneg) s.minRFlux = s.minDataFlux;
      if (s.maxDataFlux > s.maxRFlux && s.bm.haspos) s.maxRFlux = s.maxDataFlux;
    }
  }

  double singleLogLike(BeamSet1& s, double sigmult) {
    const double max_sigma = s.maxsigma_base * sigmult;
    if (max_sigma < 0.0) return kBadLike;
    if (std::isnan(s.minRFlux) || std::isnan(s.maxRFlux))
      throw OrcError(E_ARG, "R range not set");
    s.pdfac.ninterp = ninterp;
    s.pdfac.initPD(fftsize, s.minRFlux, s.maxRFlux, model, s.bm);
    double LogLike = 0.0;
    for (size_t i = 0; i < s.data.size(); ++i) {
      s.pdfac.getPD(sigmult * s.sigma_base[i], s.pd, true);
      double cur;
      if (s.data[i].binned)
        cur = s.pd.logLikeBinned(s.data[i].bins, s.data[i].bincent0, s.data[i].bindelta);
      else
        cur = s.pd.logLikeUnbinned(s.data[i].data);
      LogLike += (cur - s.like_offset[i]) / s.like_norm[i];
    }
    return LogLike;
  }

  double getLogLike(const float* p, int npar) {
    if (sets.empty()) return kNaN;
    const int nknots = static_cast<int>(model.knots.size());
    if (npar < 2) throw OrcError(E_ARG, "Not enough elements in params");
    if (nknots > npar - 1) throw OrcError(E_ARG, "Not enough elements in paramSet");
    model.setParams(p, npar);
    const double sigmult = p[nknots];
    double LogLike = 0.0;
    for (auto& s : sets) LogLike += singleLogLike(s, sigmult);
    // priors, bonus parameters and regularisation (calcLike.cc:918-952)
    const double half_log_2pi = 0.918938517570495605469;
    if (has_sigma_prior) {
      const double val = (sigmult - 1.0) / sigma_prior_width;
      LogLike -= half_log_2pi + std::log(sigma_prior_width) + 0.5 * val * val;
    }
    mean_flux_per_area = model.splineInt(1.0);
    if (has_cfirb_prior) {
      const double val = (cfirb_prior_mean - mean_flux_per_area) / cfirb_prior_sigma;
      LogLike -= half_log_2pi + std::log(cfirb_prior_sigma) + 0.5 * val * val;
    }
    mean_fluxsq_per_area = model.splineInt(2.0);
    if (has_poisson_prior) {
      const double val = (poisson_prior_mean - mean_fluxsq_per_area) / poisson_prior_sigma;
      LogLike -= half_log_2pi + std::log(poisson_prior_sigma) + 0.5 * val * val;
    }
    if (regularization_alpha > 0.0) LogLike += model.differenceRegularize(regularization_alpha);
    return LogLike;
  }
};

// ============================================================ 2D beam
// doublebeam.cc:331-462 (setBeams), 467-584 (makeHistogram), 722-772
// (log ratios).
struct Beam2 {
  static constexpr unsigned histothresh = 30;  // doublebeam.h:36
  double pixsize = 0, minval = 0;
  bool hassign[4] = {false, false, false, false};
  std::vector<double> pix1[4], pix2[4], inv1[4], inv2[4], logratio[4];
  double minbm1[4], maxbm1[4], minbm2[4], maxbm2[4];
  bool ishist[4] = {false, false, false, false};
  std::vector<double> binwt[4], binv1[4], binv2[4], binlogratio[4];

  void set(const double* b1, const double* b2, size_t n, double PIXSIZE,
           double MINVAL) {
    if (n == 0) throw OrcError(E_ARG, "Invalid (zero) n");
    if (MINVAL < 0.0) throw OrcError(E_ARG, "Invalid (negative) MINVAL");
    minval = MINVAL;
    for (int s = 0; s < 4; ++s) {
      hassign[s] = false; ishist[s] = false;
      pix1[s].clear(); pix2[s].clear();
      minbm1[s] = maxbm1[s] = minbm2[s] = maxbm2[s] = kNaN;
    }
    for (size_t i = 0; i < n; ++i) {
      const double v1 = b1[i], v2 = b2[i];
      const double a1 = std::fabs(v1), a2 = std::fabs(v2);
      if ((a1 > minval) && (a2 > minval)) {
        unsigned sgn;
        if (v1 > 0) sgn = (v2 > 0) ? 0 : 1;
        else sgn = (v2 > 0) ? 2 : 3;
        pix1[sgn].push_back(a1);
        pix2[sgn].push_back(a2);
      }
    }
    size_t tot = 0;
    for (int s = 0; s < 4; ++s) tot += pix1[s].size();
    if (tot == 0) throw OrcError(E_ARG, "No acceptable values found");
    for (int s = 0; s < 4; ++s) {
      const size_t cn = pix1[s].size();
      if (cn == 0) continue;
      hassign[s] = true;
      inv1[s].resize(cn); inv2[s].resize(cn); logratio[s].resize(cn);
      for (size_t j = 0; j < cn; ++j) inv1[s][j] = 1.0 / pix1[s][j];
      for (size_t j = 0; j < cn; ++j) inv2[s][j] = 1.0 / pix2[s][j];
      for (size_t j = 0; j < cn; ++j) logratio[s][j] = std::log(pix1[s][j] * inv2[s][j]);
      double cmin = pix1[s][0], cmax = pix1[s][0];
      for (size_t j = 1; j < cn; ++j) {
        const double v = pix1[s][j];
        if (v > cmax) cmax = v; else if (v < cmin) cmin = v;
      }
      minbm1[s] = cmin; maxbm1[s] = cmax;
      cmin = cmax = pix2[s][0];
      for (size_t j = 1; j < cn; ++j) {
        const double v = pix2[s][j];
        if (v > cmax) cmax = v; else if (v < cmin) cmin = v;
      }
      minbm2[s] = cmin; maxbm2[s] = cmax;
    }
    if (PIXSIZE <= 0.0) throw OrcError(E_ARG, "Invalid (non-positive) pixel size");
    pixsize = PIXSIZE;
  }

  void makeHistogram(unsigned nbins) {
    if (nbins == 0) throw OrcError(E_ARG, "Invalid (zero) NBINS");
    const double log2outscale = 0.0014419741739063218;
    const unsigned nb2 = nbins * nbins;
    const double dnbins = static_cast<double>(nbins);
    for (int s = 0; s < 4; ++s) {
      ishist[s] = false;
      binwt[s].clear(); binv1[s].clear(); binv2[s].clear(); binlogratio[s].clear();
      if (!(hassign[s] && pix1[s].size() >= histothresh)) continue;
      const double minb1 = std::log2(minbm1[s]) - log2outscale;
      const double maxb1 = std::log2(maxbm1[s]) + log2outscale;
      const double ih1 = dnbins / (maxb1 - minb1);
      const double minb2 = std::log2(minbm2[s]) - log2outscale;
      const double maxb2 = std::log2(maxbm2[s]) + log2outscale;
      const double ih2 = dnbins / (maxb2 - minb2);
      std::vector<unsigned> tw(nb2, 0);
      std::vector<double> th1(nb2, 0.0), th2(nb2, 0.0);
      for (size_t i = 0; i < pix1[s].size(); ++i) {
        const double v1 = pix1[s][i], v2 = pix2[s][i];
        const unsigned i1 = static_cast<unsigned>((std::log2(v1) - minb1) * ih1);
        const unsigned i2 = static_cast<unsigned>((std::log2(v2) - minb2) * ih2);
        const unsigned t = i1 * nbins + i2;
        tw[t] += 1; th1[t] += v1; th2[t] += v2;
      }
      for (unsigned i = 0; i < nb2; ++i)
        if (tw[i] > 0) {
          const double w = static_cast<double>(tw[i]);
          binwt[s].push_back(w);
          binv1[s].push_back(w / th1[i]);
          binv2[s].push_back(w / th2[i]);
        }
      for (size_t i = 0; i < binwt[s].size(); ++i)
        binlogratio[s].push_back(std::log(binv2[s][i] / binv1[s][i]));
      ishist[s] = true;
    }
  }
  bool hasData() const {
    return hassign[0] || hassign[1] || hassign[2] || hassign[3];
  }
};

// ============================================ 2D counts: log-normal colour
// numberCountsDoubleLogNormal.cc: interp choice 109-139, setParams
// 1010-1052, validity 1060-1110, getSigmaInner 1172-1179, getOffsetInner
// 1187-1193, counts 1230-1247, getMaxFlux 1365-1379, logNormalSolver
// 1389-1472, R range 1481-1521, scalar getR 1682-1724, array getR 1788-2007.
struct Counts2 {
  std::vector<double> knots, logknots, logknotvals;
  std::vector<double> sigmaknots, sigmavals, offsetknots, offsetvals;
  NatSpline spl, sigspl, offspl;
  double min_sigma = 0.0;
  bool knots_valid = false, sigmas_valid = false, offsets_valid = false;

  void setPositions(int nk, const double* kp, int ns, const double* sp, int no,
                    const double* op) {
    if (nk <= 2) throw OrcError(E_ARG, "nknots must be > 2");
    knots.assign(kp, kp + nk);
    logknots.resize(nk);
    for (int i = 0; i < nk; ++i) logknots[i] = std::log2(knots[i]);
    logknotvals.assign(nk, kNaN);
    sigmaknots.assign(sp, sp + ns);
    sigmavals.assign(ns, kNaN);
    offsetknots.assign(op, op + no);
    offsetvals.assign(no, kNaN);
  }
  int nparams() const {
    return static_cast<int>(knots.size() + sigmaknots.size() + offsetknots.size());
  }
  void setParams(const float* F, int npar) {
    const int nk = static_cast<int>(knots.size());
    const int ns = static_cast<int>(sigmaknots.size());
    const int no = static_cast<int>(offsetknots.size());
    if (nk + ns + no > npar) throw OrcError(E_ARG, "Not enough parameters present to set");
    for (int i = 0; i < nk; ++i) logknotvals[i] = kLogfac * static_cast<double>(F[i]);
    bool fin = true;
    for (double v : logknotvals) if (std::isnan(v)) fin = false;
    if (fin) spl.init(logknots.data(), logknotvals.data(), nk);
    knots_valid = fin;
    for (int i = 1; i < nk; ++i) if (knots[i] <= knots[i - 1]) knots_valid = false;
    if (knots[0] <= 0.0) knots_valid = false;
    for (int i = 0; i < ns; ++i) sigmavals[i] = static_cast<double>(F[nk + i]);
    sigmas_valid = ns > 0 && min_sigma >= 0.0 && sigmaknots[0] > 0.0;
    for (int i = 1; i < ns; ++i) if (sigmaknots[i] <= sigmaknots[i - 1]) sigmas_valid = false;
    for (double v : sigmavals) if (std::isnan(v) || std::isinf(v)) sigmas_valid = false;
    if (sigmas_valid && ns > 2) sigspl.init(sigmaknots.data(), sigmavals.data(), ns);
    for (int i = 0; i < no; ++i) offsetvals[i] = static_cast<double>(F[nk + ns + i]);
    offsets_valid = no > 0 && offsetknots[0] > 0.0;
    for (int i = 1; i < no; ++i) if (offsetknots[i] <= offsetknots[i - 1]) offsets_valid = false;
    for (double v : offsetvals) if (std::isnan(v)) offsets_valid = false;
    if (offsets_valid && no > 2) offspl.init(offsetknots.data(), offsetvals.data(), no);
  }
  bool isValid() const { return knots_valid && sigmas_valid && offsets_valid; }

  // Breakpoints of the band-1 integrals in ln S1: the knots, plus the sigma
  // and offset knots inside the knot range (where the colour curves have
  // kinks: linear interpolation, clamping).
  std::vector<double> lnBreaks() const {
    std::vector<double> b;
    for (double k : knots) b.push_back(std::log(k));
    for (const auto* v : {&sigmaknots, &offsetknots})
      for (double k : *v)
        if (k > knots.front() && k < knots.back()) b.push_back(std::log(k));
    std::sort(b.begin(), b.end());
    b.erase(std::unique(b.begin(), b.end()), b.end());
    return b;
  }
  // numberCountsDoubleLogNormal::splineInt (numberCountsDoubleLogNormal.cc:
  // 1549-1631) with the integrand of evalPowfNDoubleLogNormal (2424-2512):
  // S1^(a+b) n1(S1) exp(b mu(S1) + b^2/2 sigma^2(S1)) over [S_0, S_{K-1}),
  // sigma floored at min_sigma in every branch there.  32 panels of 20-point
  // Gauss-Legendre per breakpoint interval, in ln S1.
  double splineInt(double alpha, double beta) const {
    if (knots.size() < 2 || !isValid()) return kNaN;
    std::vector<double> gx, gw;
    gauss_legendre(20, gx, gw);
    const double power = alpha + beta, c1 = beta, c2 = 0.5 * beta * beta;
    const auto br = lnBreaks();
    double tot = 0.0;
    for (size_t k = 0; k + 1 < br.size(); ++k) {
      const int npanel = 32;
      const double h = (br[k + 1] - br[k]) / npanel;
      for (int p = 0; p < npanel; ++p) {
        const double lo = br[k] + p * h;
        for (int g = 0; g < 20; ++g) {
          const double s1 = std::exp(lo + 0.5 * h * (gx[g] + 1.0));
          if (s1 < knots.front() || s1 >= knots.back()) continue;
          double prefac = std::pow(s1, power);
          if (c1 != 0.0 || c2 != 0.0) {
            double e = 0.0;
            if (c1 != 0.0) e = c1 * offsetInner(s1);
            if (c2 != 0.0) {
              const size_t ns = sigmaknots.size();
              double sg;
              if (ns == 1) sg = sigmavals[0];
              else if (s1 <= sigmaknots[0]) sg = sigmavals[0];
              else if (s1 >= sigmaknots[ns - 1]) sg = sigmavals[ns - 1];
              else sg = (ns == 2) ? linear_interp(sigmaknots, sigmavals, s1) : sigspl.eval(s1);
              if (sg < min_sigma) sg = min_sigma;
              e += c2 * sg * sg;
            }
            prefac *= std::exp(e);
          }
          tot += 0.5 * h * gw[g] * s1 * prefac * std::exp2(spl.eval(std::log2(s1)));
        }
      }
    }
    return tot;
  }
  // differenceRegularize of the band-1 knots (numberCountsDoubleLogNormal.cc:
  // 2154-2173)
  double differenceRegularize(double alpha) const {
    if (!knots_valid) return kNaN;
    const size_t nk = knots.size();
    if (nk < 2) return 0.0;
    double mean_deriv = 0.0;
    for (size_t i = 1; i < nk; ++i)
      mean_deriv += (logknotvals[i] - logknotvals[i - 1]) / (logknots[i] - logknots[i - 1]);
    mean_deriv /= static_cast<double>(nk - 1);
    double pen = 0.0;
    for (size_t i = 1; i < nk; ++i) {
      const double d = (logknotvals[i] - logknotvals[i - 1]) / (logknots[i] - logknots[i - 1]) -
                       mean_deriv;
      pen -= d * d;
    }
    return alpha * pen;
  }

  double sigmaInner(double f1) const {
    const size_t ns = sigmaknots.size();
    if (ns == 1) return sigmavals[0];
    if (f1 <= sigmaknots[0]) return sigmavals[0];
    if (f1 >= sigmaknots[ns - 1]) return sigmavals[ns - 1];
    const double val = (ns == 2) ? linear_interp(sigmaknots, sigmavals, f1)
                                 : sigspl.eval(f1);
    return (val < min_sigma) ? min_sigma : val;
  }
  double offsetInner(double f1) const {
    const size_t no = offsetknots.size();
    if (no == 1) return offsetvals[0];
    if (f1 <= offsetknots[0]) return offsetvals[0];
    if (f1 >= offsetknots[no - 1]) return offsetvals[no - 1];
    return (no == 2) ? linear_interp(offsetknots, offsetvals, f1)
                     : offspl.eval(f1);
  }
  double countsInner(double f1, double f2) const {
    const double normfac = 1.0 / std::sqrt(2 * kPi);
    const double prefac = -0.5 * kILog2toe;
    if (f1 < knots.front() || f1 >= knots.back() || f2 <= 0.0) return 0.0;
    double cnts = std::exp2(spl.eval(std::log2(f1)));
    const double if1 = 1.0 / f1;
    const double isigma = 1.0 / sigmaInner(f1);
    const double tfac = (std::log(f2 * if1) - offsetInner(f1)) * isigma;
    cnts *= normfac * isigma * std::exp2(prefac * tfac * tfac) / f2;
    return cnts;
  }
  double counts(double f1, double f2) const {
    if (!isValid()) return kNaN;
    if (std::isnan(f1) || std::isinf(f1) || std::isnan(f2) || std::isinf(f2)) return kNaN;
    return countsInner(f1, f2);
  }

  static double lognorm(double u, double mu, double isig, double isig2,
                        double target) {
    const double prefac = 1.0 / std::sqrt(2 * kPi);
    const double eu = std::exp(-u);
    const double arg = u - mu;
    const double L = prefac * std::exp(-0.5 * arg * arg * isig2) * isig * eu;
    return L - target;
  }
  double logNormalSolver(double mu, double sig, double nsig) const {
    const unsigned max_bracket_iters = 20;
    const double prefac = 1.0 / std::sqrt(kTwoPi);
    const double tol = 1e-3;
    if (sig <= 0.0) throw OrcError(E_ARG, "Invalid (non-positive) sigma");
    if (nsig < 0.0) throw OrcError(E_ARG, "Invalid (negative) nsig");
    const double sig2 = sig * sig;
    const double mode_u = mu - sig2;
    if (nsig == 0) return std::exp(mode_u);
    const double isig = 1.0 / sig;
    const double val_mode = prefac * isig * std::exp(0.5 * sig2 - mu);
    const double target = val_mode * std::exp(-0.5 * nsig * nsig);
    const double isig2 = isig * isig;
    auto F = [&](double u) { return lognorm(u, mu, isig, isig2, target); };
    double u_low = mode_u;
    double delta_u = std::log(std::exp(mode_u) + 2 * sig) - mode_u;
    double fval = F(u_low + delta_u);
    if (fval >= 0.0) {
      for (unsigned i = 0; i < max_bracket_iters; ++i) {
        delta_u *= 1.5;
        fval = F(u_low + delta_u);
        if (fval < 0.0) break;
      }
      if (fval >= 0.0) throw OrcError(E_ARG, "Unable to bracket Log Normal");
    }
    double u_high = u_low + delta_u;
    BrentState st;
    brent_init(st, F, u_low, u_high);
    bool ok = false;
    double u = 0.5 * (u_low + u_high);
    for (unsigned i = 0; i < max_bracket_iters; ++i) {
      u = brent_iterate(st, F, u_low, u_high);
      if (root_interval_ok(u_low, u_high, 0, tol)) { ok = true; break; }
    }
    if (!ok) throw OrcError(E_ARG, "Unable to brent bracket Log Normal");
    return std::exp(u);
  }
  std::pair<double, double> maxFlux() const {
    const double nsig = 3.0;
    const double kv = knots.back();
    const double sg = sigmaInner(kv);
    const double mu = offsetInner(kv);
    const double m2 = logNormalSolver(mu, sg, nsig);
    return {kv, kv * m2};
  }
  // returns (min1, max1, min2, max2)
  void rrangeInternal(const Beam2& bm, double* r) const {
    double minflux1 = 0, maxflux1 = 0, minflux2 = 0, maxflux2 = 0;
    const auto maxf = maxFlux();
    double cval;
    if (bm.hassign[0]) {
      cval = maxf.first * bm.maxbm1[0]; if (cval > maxflux1) maxflux1 = cval;
      cval = maxf.second * bm.maxbm2[0]; if (cval > maxflux2) maxflux2 = cval;
    }
    if (bm.hassign[1]) {
      cval = maxf.first * bm.maxbm1[1]; if (cval > maxflux1) maxflux1 = cval;
      cval = -maxf.second * bm.maxbm2[1]; if (cval < minflux2) minflux2 = cval;
    }
    if (bm.hassign[2]) {
      cval = -maxf.first * bm.maxbm1[2]; if (cval < minflux1) minflux1 = cval;
      cval = maxf.second * bm.maxbm2[2]; if (cval > maxflux2) maxflux2 = cval;
    }
    if (bm.hassign[3]) {
      cval = -maxf.first * bm.maxbm1[3]; if (cval < minflux1) minflux1 = cval;
      cval = -maxf.second * bm.maxbm2[3]; if (cval < minflux2) minflux2 = cval;
    }
    r[0] = minflux1; r[1] = maxflux1; r[2] = minflux2; r[3] = maxflux2;
  }

  double getRScalar(double f1, double f2, const Beam2& bm) const {
    if (!isValid()) return kNaN;
    if (!bm.hasData()) return kNaN;
    if ((f1 == 0) || (f2 == 0)) return 0.0;
    unsigned sgn;
    if (f1 >= 0) sgn = (f2 >= 0) ? 0 : 1; else sgn = (f2 >= 0) ? 2 : 3;
    if (!bm.hassign[sgn]) return 0.0;
    const double af1 = std::fabs(f1), af2 = std::fabs(f2);
    double retval = 0.0;
    if (bm.ishist[sgn]) {
      for (size_t i = 0; i < bm.binwt[sgn].size(); ++i) {
        const double i1 = bm.binv1[sgn][i], i2 = bm.binv2[sgn][i];
        retval += bm.binwt[sgn][i] * i1 * i2 * countsInner(af1 * i1, af2 * i2);
      }
    } else {
      for (size_t i = 0; i < bm.inv1[sgn].size(); ++i) {
        const double i1 = bm.inv1[sgn][i], i2 = bm.inv2[sgn][i];
        retval += i1 * i2 * countsInner(af1 * i1, af2 * i2);
      }
    }
    const double prefac = bm.pixsize / 3600.0;
    return prefac * prefac * retval;
  }

  // Array getR (row precompute + column loop), .cc:1788-2007.
  void getR(size_t n1, const double* f1, size_t n2, const double* f2,
            const Beam2& bm, double* R) const {
    if (!isValid() || !bm.hasData() || n1 == 0 || n2 == 0) {
      for (size_t i = 0; i < n1 * n2; ++i) R[i] = kNaN;
      return;
    }
    const double minknot = knots.front(), maxknot = knots.back();
    bool hs[4];
    size_t npsf[4];
    const std::vector<double>*wt[4], *ib1[4], *lr[4];
    double maxf1[4];
    for (int s = 0; s < 4; ++s) {
      hs[s] = bm.hassign[s];
      const bool ih = bm.ishist[s];
      npsf[s] = hs[s] ? (ih ? bm.binwt[s].size() : bm.pix1[s].size()) : 0;
      wt[s] = ih ? &bm.binwt[s] : nullptr;
      ib1[s] = ih ? &bm.binv1[s] : &bm.inv1[s];
      lr[s] = ih ? &bm.binlogratio[s] : &bm.logratio[s];
      maxf1[s] = hs[s] ? maxknot * bm.maxbm1[s] : 0.0;
    }
    const size_t maxnpsf = std::max(npsf[0] + npsf[1], npsf[2] + npsf[3]);
    std::vector<double> RWork(3 * (maxnpsf + 1), 0.0);
    const double normfac = 1.0 / std::sqrt(2 * kPi);
    const double pixsizedeg = bm.pixsize / 3600.0;
    const double prefac = pixsizedeg * pixsizedeg * normfac;
    const bool hasNegX1 = hs[2] || hs[3];
    std::fill(R, R + n1 * n2, 0.0);
    std::vector<unsigned> f2sgn(n2, 0);
    std::vector<double> f2inv(n2, 0.0), f2log(n2, 0.0);
    for (size_t j = 0; j < n2; ++j) {
      double v = f2[j];
      if (v == 0) { f2inv[j] = 0.0; continue; }
      if (v > 0) f2sgn[j] = 0;
      else { f2sgn[j] = 1; v = std::fabs(v); }
      f2inv[j] = 1.0 / v;
      f2log[j] = std::log(v);
    }
    for (size_t i = 0; i < n1; ++i) {
      double f1val = f1[i];
      if ((f1val == 0) || (f1val < 0 && !hasNegX1)) continue;
      unsigned sgn1;
      if (f1val > 0) sgn1 = 0; else { sgn1 = 2; f1val = std::fabs(f1val); }
      const double logf1val = std::log(f1val);
      const size_t np = hs[sgn1] ? npsf[sgn1] : 0;
      const size_t nn = hs[sgn1 + 1] ? npsf[sgn1 + 1] : 0;
      for (unsigned k = 0; k < 2; ++k) {
        const unsigned sgn = sgn1 + k;
        const size_t curr_n = (k == 0) ? np : nn;
        if (curr_n > 0 && f1val < maxf1[sgn]) {
          double* RWptr = RWork.data() + k * np * 3;
          for (size_t j = 0; j < curr_n; ++j) {
            const double ieta1 = (*ib1[sgn])[j];
            const double f1prod = f1val * ieta1;
            double* cRW = RWptr + 3 * j;
            if (f1prod >= minknot && f1prod < maxknot) {
              const double cts = std::exp2(spl.eval(std::log2(f1prod)));
              if (cts > 0) {
                const double isigma = 1.0 / sigmaInner(f1prod);
                if (wt[sgn]) cRW[0] = (*wt[sgn])[j] * ieta1 * isigma * cts * prefac;
                else cRW[0] = cts * ieta1 * isigma * prefac;
                cRW[1] = logf1val + offsetInner(f1prod) - (*lr[sgn])[j];
                cRW[2] = -0.5 * isigma * isigma * kILog2toe;
              } else cRW[0] = 0;
            } else cRW[0] = 0;
          }
        } else {
          const size_t mi = (k == 0) ? 0 : np;
          const size_t ma = (k == 0) ? np : (np + nn);
          for (size_t j = mi; j < ma; ++j) RWork[3 * j] = 0.0;
        }
      }
      double* rowptr = R + i * n2;
      for (size_t j = 0; j < n2; ++j) {
        const double if2val = f2inv[j];
        if (if2val == 0) continue;
        const unsigned fs = f2sgn[j];
        const unsigned sgn = sgn1 + fs;
        if (hs[sgn]) {
          double workval = 0;
          const size_t curr_n = npsf[sgn];
          const double* RWptr = RWork.data() + fs * np * 3;
          const double logf2val = f2log[j];
          for (size_t k = 0; k < curr_n; ++k) {
            const double* cRW = RWptr + k * 3;
            const double c0 = cRW[0];
            if (c0 != 0) {
              const double tfac = logf2val - cRW[1];
              workval += c0 * std::exp2(tfac * tfac * cRW[2]);
            }
          }
          rowptr[j] = workval * f2inv[j];
        }
      }
    }
  }
};

// =================================================================== 2D P(D)
// PDDouble.cc:142-230 (integral, normalise, log), 355-447 (means),
// 1103-1222 (binned log-likelihood).
struct PD2 {
  size_t n1 = 0, n2 = 0;
  std::vector<double> pd;
  double minflux1 = 0, dflux1 = 1, minflux2 = 0, dflux2 = 1;
  bool logflat = false;

  double integral() const {
    double tot = 0.5 * pd[0];
    for (size_t j = 1; j < n2 - 1; ++j) tot += pd[j];
    tot += 0.5 * pd[n2 - 1];
    tot *= 0.5;
    for (size_t i = 1; i < n1 - 1; ++i) {
      const double* r = pd.data() + i * n2;
      tot += 0.5 * r[0];
      for (size_t j = 1; j < n2 - 1; ++j) tot += r[j];
      tot += 0.5 * r[n2 - 1];
    }
    const double* r = pd.data() + (n1 - 1) * n2;
    tot += 0.25 * r[0];
    for (size_t j = 1; j < n2 - 1; ++j) tot += 0.5 * r[j];
    tot += 0.25 * r[n2 - 1];
    return tot * dflux1 * dflux2;
  }
  void normalize() {
    const double itot = 1.0 / integral();
    for (auto& v : pd) v *= itot;
  }
  void applyLog() {
    if (logflat) return;
    for (auto& v : pd) v = (v <= 0.0) ? kSmallLogVal : std::log2(v);
    logflat = true;
  }
  std::pair<double, double> meansNoNorm() const {
    double mean1 = 0.0, mean2 = 0.0, xsum, pval;
    for (size_t j = 1; j < n2 - 1; ++j) mean2 += j * pd[j];
    mean2 += 0.5 * (n2 - 1) * pd[n2 - 1];
    mean2 *= 0.5;
    for (size_t i = 1; i < n1 - 1; ++i) {
      const double* r = pd.data() + n2 * i;
      xsum = 0.5 * r[0];
      for (size_t j = 1; j < n2 - 1; ++j) {
        pval = r[j];
        xsum += pval;
        mean2 += static_cast<double>(j) * pval;
      }
      xsum += 0.5 * r[n2 - 1];
      mean1 += xsum * static_cast<double>(i);
      mean2 += 0.5 * (n2 - 1) * r[n2 - 1];
    }
    const double* r = pd.data() + (n1 - 1) * n2;
    xsum = 0.5 * r[0];
    for (size_t j = 1; j < n2 - 1; ++j) {
      pval = r[j];
      xsum += pval;
      mean2 += 0.5 * static_cast<double>(j) * pval;
    }
    xsum += 0.5 * r[n2 - 1];
    mean1 += 0.5 * xsum * (n1 - 1);
    mean2 += 0.25 * (n2 - 1) * r[n2 - 1];
    mean1 *= dflux1 * dflux1 * dflux2;
    mean2 *= dflux1 * dflux2 * dflux2;
    mean1 += minflux1;
    mean2 += minflux2;
    return {mean1, mean2};
  }
  // PDDouble::getLogLikeUnbinned, log-stored branch (PDDouble.cc:994-1051):
  // edge tests are inclusive here, unlike the binned form.
  double logLikeUnbinned(const std::vector<double>& f1, const std::vector<double>& f2) const {
    const double maxflux1 = minflux1 + static_cast<double>(n1 - 1) * dflux1;
    const double maxflux2 = minflux2 + static_cast<double>(n2 - 1) * dflux2;
    const size_t n2n1 = n2 * n1;
    const double idflux1 = 1.0 / dflux1, idflux2 = 1.0 / dflux2;
    double loglike = 0.0;
    for (size_t i = 0; i < f1.size(); ++i) {
      const double cflux1 = f1[i], cflux2 = f2[i];
      const double delt1 = (cflux1 - minflux1) * idflux1;
      const double delt2 = (cflux2 - minflux2) * idflux2;
      const int idx1 = static_cast<int>(delt1);
      const int idx2 = static_cast<int>(delt2);
      const size_t n2idx1 = n2 * static_cast<size_t>(idx1);
      double iv;
      if (cflux1 <= minflux1) {
        if (cflux2 <= minflux2) iv = pd[0];
        else if (cflux2 >= maxflux2) iv = pd[n2 - 1];
        else iv = pd[idx2];
      } else if (cflux1 >= maxflux1) {
        if (cflux2 <= minflux2) iv = pd[n2n1 - n1];
        else if (cflux2 >= maxflux2) iv = pd[n2n1 - 1];
        else iv = pd[n2n1 - n1 + idx2];
      } else if (cflux2 <= minflux2) {
        iv = pd[n2idx1];
      } else if (cflux2 >= maxflux2) {
        iv = pd[n2idx1 + n2 - 1];
      } else {
        const double t = delt1 - static_cast<double>(idx1);
        const double u = delt2 - static_cast<double>(idx2);
        const double omu = 1.0 - u, omt = 1.0 - t;
        const size_t b = n2idx1 + idx2;
        iv = omt * (omu * pd[b] + u * pd[b + 1]) + t * (omu * pd[b + n2] + u * pd[b + n2 + 1]);
      }
      loglike += iv;
    }
    return kLog2toe * loglike;
  }
  double logLikeBinned(const std::vector<unsigned>& bins, unsigned nb1,
                       unsigned nb2, double bc1, double bc2, double bd1,
                       double bd2) const {
    const double maxflux1 = minflux1 + static_cast<double>(n1 - 1) * dflux1;
    const double maxflux2 = minflux2 + static_cast<double>(n2 - 1) * dflux2;
    const size_t n2n1 = n2 * n1;
    const double idflux1 = 1.0 / dflux1, idflux2 = 1.0 / dflux2;
    double loglike = 0.0;
    for (unsigned i = 0; i < nb1; ++i) {
      const double cflux1 = bc1 + static_cast<double>(i) * bd1;
      int idx1 = static_cast<int>((cflux1 - minflux1) * idflux1);
      const unsigned* binptr = bins.data() + static_cast<size_t>(i) * nb2;
      for (unsigned j = 0; j < nb2; ++j) {
        const unsigned ninbin = binptr[j];
        if (ninbin == 0) continue;
        const double cflux2 = bc2 + static_cast<double>(j) * bd2;
        int idx2 = static_cast<int>((cflux2 - minflux2) * idflux2);
        double iv;
        if (cflux1 < minflux1) {
          if (cflux2 < minflux2) iv = pd[0];
          else if (cflux2 > maxflux2) iv = pd[n2 - 1];
          else iv = pd[idx2];
        } else if (cflux1 > maxflux1) {
          if (cflux2 < minflux2) iv = pd[n2n1 - n1];
          else if (cflux2 > maxflux2) iv = pd[n2n1 - 1];
          else iv = pd[n2n1 - n1 + idx2];
        } else if (cflux2 < minflux2) {
          iv = pd[n2 * idx1];
        } else if (cflux2 > maxflux2) {
          iv = pd[n2 * idx1 + n2 - 1];
        } else {
          double t = (cflux1 - minflux1) * idflux1 - static_cast<double>(idx1);
          double u = (cflux2 - minflux2) * idflux2 - static_cast<double>(idx2);
          // The reference reads one cell past the grid when the point lies
          // in the last row/column; clamp to the last cell instead.
          int i1 = idx1, i2 = idx2;
          if (i1 > static_cast<int>(n1) - 2) { i1 = static_cast<int>(n1) - 2; t = 1.0; }
          if (i2 > static_cast<int>(n2) - 2) { i2 = static_cast<int>(n2) - 2; u = 1.0; }
          const double omu = 1.0 - u, omt = 1.0 - t;
          const size_t b = n2 * i1 + i2;
          iv = omt * (omu * pd[b] + u * pd[b + 1]) +
               t * (omu * pd[b + n2] + u * pd[b + n2 + 1]);
        }
        loglike += static_cast<double>(ninbin) * iv;
      }
    }
    return kLog2toe * loglike;
  }
};

// ===================================================== 2D P(D) factory
// PDFactoryDouble.cc:18-49 (initRFluxInternal), 313-338 (initRFlux),
// 355-585 (initR with edges), 593-722 (getRStats), 784-968 (findSplitPoint),
// 978-1118 (unwrap), 1145-1349 (initPD), 1362-1499 (getPD).
struct PDF2 {
  static constexpr double lowEdgeRMult = 1e-9;  // PDFactoryDouble.h:33
  unsigned nedge = 256;
  unsigned n = 0;
  double dflux1 = 0, dflux2 = 0;
  unsigned wrap1 = 0, wrap2 = 0;
  std::vector<double> RFlux1, RFlux2, rvals, pofd, rsum;
  std::vector<cplx> prtrans, pval;
  double mn1 = 0, mn2 = 0, var1 = 0, var2 = 0;
  double sg1pos = 0, sg1neg = 0, sg2pos = 0, sg2neg = 0;
  bool doshift1 = false, doshift2 = false;
  double shift1 = 0, shift2 = 0;
  unsigned lastsplit1 = 0, lastsplit2 = 0;

  static void rfluxInternal(unsigned N, double minflux, double maxflux,
                            std::vector<double>& rflux, double& dflux,
                            unsigned& wrapidx) {
    rflux.assign(N, 0.0);
    const double inm1 = 1.0 / static_cast<double>(N - 1);
    dflux = (maxflux - minflux) * inm1;
    if (minflux >= 0.0) {
      rflux[0] = minflux;
      for (unsigned i = 1; i < N; ++i) rflux[i] = static_cast<double>(i) * dflux + minflux;
      wrapidx = N - 1;
    } else {
      dflux = maxflux / (N - std::floor(-minflux / dflux) - 1.0);
      wrapidx = static_cast<unsigned>(maxflux / dflux + 0.999999999);
      rflux[0] = 0.0;
      for (unsigned i = 1; i <= wrapidx; ++i) rflux[i] = static_cast<double>(i) * dflux;
      const double wrapval = -static_cast<double>(N) * dflux;
      for (unsigned i = wrapidx + 1; i < N; ++i) rflux[i] = static_cast<double>(i) * dflux + wrapval;
    }
  }

  void initRFlux(unsigned N, double min1, double max1, double min2, double max2) {
    if (N == 0) throw OrcError(E_ARG, "Invalid (0) n");
    n = N;
    if (max1 < min1) std::swap(min1, max1);
    if (max2 < min2) std::swap(min2, max2);
    rfluxInternal(N, min1, max1, RFlux1, dflux1, wrap1);
    rfluxInternal(N, min2, max2, RFlux2, dflux2, wrap2);
  }

  void initR(unsigned N, double min1, double max1, double min2, double max2,
             const Counts2& model, const Beam2& bm, bool setEdge) {
    initRFlux(N, min1, max1, min2, max2);
    rvals.assign(static_cast<size_t>(N) * N, 0.0);
    double r00val = 0.0;
    std::vector<double> RxEdge, RyEdge;
    if (setEdge) {
      if (N < nedge) throw OrcError(E_ARG, "Nedge is less than R fill size");
      const double minedge1 = dflux1 * lowEdgeRMult;
      const double minedge2 = dflux2 * lowEdgeRMult;
      const double inedgem1 = 1.0 / static_cast<double>(nedge - 1);
      std::vector<double> E1(nedge), E2(nedge);
      const double dife1 = -std::log(lowEdgeRMult) * inedgem1;  // log x
      for (unsigned i = 0; i < nedge; ++i)
        E1[i] = minedge1 * std::exp(static_cast<double>(i) * dife1);
      const double dife2 = (dflux2 - minedge2) * inedgem1;  // linear y
      for (unsigned i = 0; i < nedge; ++i)
        E2[i] = minedge2 + static_cast<double>(i) * dife2;
      const double iRxnorm = dife1 / (dflux1 - minedge1);
      const double iRynorm = dife2 / (dflux2 - minedge2);
      const double iR00norm = dife1 * dife2 / ((dflux1 - minedge1) * (dflux2 - minedge2));
      std::vector<double> work(static_cast<size_t>(nedge) * std::max(nedge, N));
      // r[0,0]
      model.getR(nedge, E1.data(), nedge, E2.data(), bm, work.data());
      std::vector<double> rx(std::max(nedge, N));
      for (unsigned i = 0; i < nedge; ++i) {
        const double* rp = work.data() + static_cast<size_t>(i) * nedge;
        double s = 0.5 * rp[0];
        for (unsigned j = 1; j < nedge - 1; ++j) s += rp[j];
        s += 0.5 * rp[nedge - 1];
        rx[i] = s;
      }
      double s = 0.5 * E1[0] * rx[0];
      for (unsigned i = 1; i < nedge - 1; ++i) s += E1[i] * rx[i];
      s += 0.5 * E1[nedge - 1] * rx[nedge - 1];
      r00val = s * iR00norm;
      // Rx = R[0, y]
      model.getR(nedge, E1.data(), N, RFlux2.data(), bm, work.data());
      RxEdge.assign(N, 0.0);
      {
        double rf = E1[0];
        for (unsigned j = 0; j < N; ++j) RxEdge[j] = 0.5 * rf * work[j];
        for (unsigned i = 1; i < nedge - 1; ++i) {
          rf = E1[i];
          const double* rp = work.data() + static_cast<size_t>(i) * N;
          for (unsigned j = 0; j < N; ++j) RxEdge[j] += rf * rp[j];
        }
        rf = E1[nedge - 1];
        const double* rp = work.data() + static_cast<size_t>(nedge - 1) * N;
        for (unsigned j = 0; j < N; ++j) RxEdge[j] += 0.5 * rf * rp[j];
      }
      for (unsigned j = 0; j < N; ++j) RxEdge[j] *= iRxnorm;
      // Ry = R[x, 0]
      model.getR(N, RFlux1.data(), nedge, E2.data(), bm, work.data());
      RyEdge.assign(N, 0.0);
      for (unsigned i = 0; i < N; ++i) {
        const double* rp = work.data() + static_cast<size_t>(i) * nedge;
        double t = 0.5 * rp[0];
        for (unsigned j = 1; j < nedge - 1; ++j) t += rp[j];
        t += 0.5 * rp[nedge - 1];
        RyEdge[i] = t;
      }
      for (unsigned i = 0; i < N; ++i) RyEdge[i] *= iRynorm;
    }
    model.getR(N, RFlux1.data(), N, RFlux2.data(), bm, rvals.data());
    if (setEdge) {
      for (unsigned j = 1; j < N; ++j) rvals[j] = RxEdge[j];
      for (unsigned i = 1; i < N; ++i) rvals[static_cast<size_t>(i) * N] = RyEdge[i];
      rvals[0] = r00val;
    } else {
      for (unsigned j = 0; j < N; ++j) rvals[j] = 0.0;
      for (unsigned i = 1; i < N; ++i) rvals[static_cast<size_t>(i) * N] = 0.0;
    }
    const double fluxfac = dflux1 * dflux2;
    for (auto& v : rvals) v *= fluxfac;
  }

  void getRStats() {
    const unsigned cs = n;
    double cf1, cf2, cR, mean1, mean2, v1, v2, prod1, prod2;
    const double* rowptr = rvals.data();
    cf1 = RFlux1[0];
    cR = 0.5 * rowptr[0];
    prod1 = 0.5 * cf1 * cR; mean1 = prod1; v1 = cf1 * prod1;
    cf2 = RFlux2[0];
    prod2 = 0.5 * cf2 * cR; mean2 = prod2; v2 = cf2 * prod2;
    for (unsigned j = 1; j < cs - 1; ++j) {
      cR = 0.5 * rowptr[j];
      prod1 = cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
      cf2 = RFlux2[j];
      prod2 = cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
    }
    cR = 0.5 * rowptr[cs - 1];
    prod1 = 0.5 * cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
    cf2 = RFlux2[cs - 1];
    prod2 = 0.5 * cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
    for (unsigned i = 1; i < cs - 1; ++i) {
      rowptr = rvals.data() + static_cast<size_t>(i) * cs;
      cf1 = RFlux1[i];
      cR = rowptr[0];
      prod1 = 0.5 * cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
      cf2 = RFlux2[0];
      prod2 = 0.5 * cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
      for (unsigned j = 1; j < cs - 1; ++j) {
        cR = rowptr[j];
        prod1 = cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
        cf2 = RFlux2[j];
        prod2 = cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
      }
      cR = rowptr[cs - 1];
      prod1 = 0.5 * cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
      cf2 = RFlux2[cs - 1];
      prod2 = 0.5 * cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
    }
    rowptr = rvals.data() + static_cast<size_t>(cs - 1) * cs;
    cf1 = RFlux1[cs - 1];
    cR = 0.5 * rowptr[0];
    prod1 = 0.5 * cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
    cf2 = RFlux2[0];
    prod2 = 0.5 * cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
    for (unsigned j = 1; j < cs - 1; ++j) {
      cR = 0.5 * rowptr[j];
      prod1 = cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
      cf2 = RFlux2[j];
      prod2 = cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
    }
    cR = 0.5 * rowptr[cs - 1];
    prod1 = 0.5 * cf1 * cR; mean1 += prod1; v1 += cf1 * prod1;
    cf2 = RFlux2[cs - 1];
    prod2 = 0.5 * cf2 * cR; mean2 += prod2; v2 += cf2 * prod2;
    mn1 = mean1; mn2 = mean2; var1 = v1; var2 = v2;
  }

  void initPD(unsigned N, double min1, double max1, double min2, double max2,
              const Counts2& model, const Beam2& bm, bool setEdge) {
    if (N == 0) throw OrcError(E_ARG, "Invalid (zero) n");
    if (N == 1) throw OrcError(E_ARG, "Invalid n (==1)");
    if (max1 <= 0.0) throw OrcError(E_ARG, "Invalid (non-positive) maxflux1");
    if (max2 <= 0.0) throw OrcError(E_ARG, "Invalid (non-positive) maxflux2");
    if (max1 == min1) throw OrcError(E_ARG, "Invalid range (0) between min/max flux in band 1");
    if (max2 == min2) throw OrcError(E_ARG, "Invalid range (0) between min/max flux in band 2");
    if (!model.isValid()) throw OrcError(E_INVALID_MODEL, "Invalid model");
    initR(N, min1, max1, min2, max2, model, bm, setEdge);
    getRStats();
    sg1pos = std::sqrt(var1);
    sg2pos = std::sqrt(var2);
    doshift1 = (sg1pos > dflux1) && (std::fabs(mn1) > dflux1);
    shift1 = doshift1 ? -mn1 : 0.0;
    doshift2 = (sg2pos > dflux2) && (std::fabs(mn2) > dflux2);
    shift2 = doshift2 ? -mn2 : 0.0;
    const unsigned ncplx = N / 2 + 1;
    prtrans.assign(static_cast<size_t>(N) * ncplx, 0.0);
    rfft2(N, rvals.data(), prtrans.data());
    const double iflux1 = kTwoPi / (N * dflux1);
    const double iflux2 = kTwoPi / (N * dflux2);
    const double r0 = prtrans[0].real();
    const double shiftfac1 = doshift1 ? shift1 * iflux1 : 0.0;
    const double shiftfac2 = doshift2 ? shift2 * iflux2 : 0.0;
    for (unsigned idx1 = 0; idx1 < N; ++idx1) {
      cplx* row = prtrans.data() + static_cast<size_t>(idx1) * ncplx;
      double shiftprod1 = 0.0;
      if (doshift1)
        shiftprod1 = (idx1 < ncplx) ? shiftfac1 * static_cast<double>(idx1)
                                    : -shiftfac1 * static_cast<double>(N - idx1);
      for (unsigned idx2 = 0; idx2 < ncplx; ++idx2) {
        const double rval = row[idx2].real() - r0;
        double ival = row[idx2].imag();
        if (doshift1) ival = ival - shiftprod1;
        if (doshift2) ival = ival - shiftfac2 * static_cast<double>(idx2);
        const double expfac = std::exp(rval);
        row[idx2] = cplx(expfac * std::cos(ival), expfac * std::sin(ival));
      }
    }
    prtrans[0] = cplx(1.0, 0.0);
  }

  unsigned findSplitPoint(const double* data, double dflux, double sigmapos,
                          double sigmaneg) const {
    const double n1 = 2.25, f1 = 5e-14, f2 = 1.5e-5, f3 = 5;
    if (sigmapos <= 0) throw OrcError(E_SPLIT_RANGE, "Invalid (non-positive) sigma pos");
    if (sigmaneg <= 0) throw OrcError(E_SPLIT_RANGE, "Invalid (non-positive) sigma neg");
    const int cs = static_cast<int>(n);
    const double fluxrange = n * dflux;
    const double n1sigpos = n1 * sigmapos, n1signeg = n1 * sigmaneg;
    if (fluxrange < (n1sigpos + n1signeg)) throw OrcError(E_SPLIT_RANGE, "Not enough flux range");
    double peak = data[0];
    for (int i = 1; i < cs; ++i) if (data[i] > peak) peak = data[i];
    if (peak <= 0.0) throw OrcError(E_SPLIT_PEAK, "Peak P(D) value was zero");
    const int topidx = cs - static_cast<int>(n1signeg / dflux) - 1;
    const int botidx = static_cast<int>(n1sigpos / dflux);
    if (topidx >= cs || botidx < 0 || botidx > topidx)
      throw OrcError(E_SPLIT_LOGIC, "Logic error in topidx/botidx");
    int minidx = botidx;
    double minval = data[minidx];
    for (int i = botidx + 1; i <= topidx; ++i)
      if (data[i] < minval) { minidx = i; minval = data[i]; }
    if (minval > f2 * peak) throw OrcError(E_SPLIT_MIN, "Minimum in marginalized pd is too large");
    const int pre_jitter_n = 17;
    double jitter = 0.0;
    if (minidx > pre_jitter_n) {
      bool mono = true;
      const int initidx = minidx - pre_jitter_n;
      double prevval;
      jitter = prevval = data[initidx];
      for (int i = initidx + 1; i < minidx; ++i) {
        const double cv = data[i];
        if (cv >= prevval) mono = false;
        jitter += cv;
        prevval = cv;
      }
      if (mono) return static_cast<unsigned>(minidx);
      jitter += minval;
      jitter = 1.1 * jitter / static_cast<double>(pre_jitter_n + 1);
    } else {
      jitter = f1 * peak;
      if (minval > jitter) return static_cast<unsigned>(minidx);
    }
    if (minval <= 0.0) {
      const int nminup = 3;
      int bi, ti;
      if (minidx < botidx) bi = botidx;
      else bi = (minidx >= nminup) ? (minidx - nminup) : minidx;
      if (minidx > topidx - nminup) ti = topidx - nminup; else ti = minidx + nminup;
      ti = (ti >= cs) ? (cs - 1) : ti;
      for (int i = bi; i < ti; ++i) if (data[i] > minval) minval = data[i];
    }
    if (minval > 0) jitter = (f3 * minval) < jitter ? (f3 * minval) : jitter;
    if ((botidx >= topidx) || (std::abs(topidx - botidx) < 1))
      throw OrcError(E_SPLIT_LOGIC, "Topidx vs. botidx search issue");
    if (data[topidx] < jitter) throw OrcError(E_SPLIT_TOP, "Topidx is already below jitter estimate");
    for (int i = topidx - 1; i >= botidx; --i)
      if (data[i] < jitter) return static_cast<unsigned>(i + 1);
    throw OrcError(E_SPLIT_NONE, "Unable to find split point");
  }

  void getPD(double sigma1, double sigma2, PD2& pd, bool setLog) {
    const unsigned N = n, ncplx = N / 2 + 1;
    pofd.assign(static_cast<size_t>(N) * N, 0.0);
    if (sigma1 > 0 || sigma2 > 0) {
      const double iflux1 = kTwoPi / (N * dflux1);
      const double iflux2 = kTwoPi / (N * dflux2);
      const double sigfac1 = -0.5 * sigma1 * sigma1 * iflux1 * iflux1;
      const double sigfac2 = -0.5 * sigma2 * sigma2 * iflux2 * iflux2;
      pval.assign(static_cast<size_t>(N) * ncplx, 0.0);
      for (unsigned idx1 = 0; idx1 < N; ++idx1) {
        const double didx1 = (idx1 < ncplx) ? static_cast<double>(idx1)
                                            : static_cast<double>(N - idx1);
        const double sigprod1 = sigfac1 * didx1 * didx1;
        const cplx* in = prtrans.data() + static_cast<size_t>(idx1) * ncplx;
        cplx* out = pval.data() + static_cast<size_t>(idx1) * ncplx;
        for (unsigned idx2 = 0; idx2 < ncplx; ++idx2) {
          const double didx2 = static_cast<double>(idx2);
          const double expfac = std::exp(sigprod1 + sigfac2 * didx2 * didx2);
          out[idx2] = cplx(expfac * in[idx2].real(), expfac * in[idx2].imag());
        }
      }
      pval[0] = cplx(1.0, 0.0);
      irfft2(N, pval.data(), pofd.data());
    } else {
      irfft2(N, prtrans.data(), pofd.data());
    }
    sg1pos = std::sqrt(var1 + sigma1 * sigma1);
    sg2pos = std::sqrt(var2 + sigma2 * sigma2);
    sg1neg = (9 * sigma1 * sigma1 > var1) ? sigma1 : sg1pos;
    sg2neg = (9 * sigma2 * sigma2 > var2) ? sigma2 : sg2pos;
    // unwrapAndNormalizePD
    for (auto& v : pofd) if (v < 0) v = 0.0;
    rsum.assign(N, 0.0);
    for (unsigned i = 0; i < N; ++i) {
      const double* r = pofd.data() + static_cast<size_t>(i) * N;
      double cval = 0.5 * r[0];
      for (unsigned j = 1; j < N - 1; ++j) cval += r[j];
      cval += 0.5 * r[N - 1];
      rsum[i] = cval;
    }
    const unsigned s1 = findSplitPoint(rsum.data(), dflux1, sg1pos, sg1neg);
    for (unsigned j = 0; j < N; ++j) rsum[j] = 0.5 * pofd[j];
    for (unsigned i = 1; i < N - 1; ++i) {
      const double* r = pofd.data() + static_cast<size_t>(i) * N;
      for (unsigned j = 0; j < N; ++j) rsum[j] += r[j];
    }
    {
      const double* r = pofd.data() + static_cast<size_t>(N - 1) * N;
      for (unsigned j = 0; j < N; ++j) rsum[j] += 0.5 * r[j];
    }
    const unsigned s2 = findSplitPoint(rsum.data(), dflux2, sg2pos, sg2neg);
    lastsplit1 = s1; lastsplit2 = s2;
    pd.n1 = pd.n2 = N;
    pd.pd.assign(static_cast<size_t>(N) * N, 0.0);
    for (unsigned a = 0; a < N; ++a) {
      const unsigned i = (a + s1) % N;
      for (unsigned b = 0; b < N; ++b) {
        const unsigned j = (b + s2) % N;
        pd.pd[static_cast<size_t>(a) * N + b] = pofd[static_cast<size_t>(i) * N + j];
      }
    }
    pd.logflat = false;
    pd.minflux1 = 0.0; pd.dflux1 = dflux1;
    pd.minflux2 = 0.0; pd.dflux2 = dflux2;
    pd.normalize();
    const auto tmn = pd.meansNoNorm();
    if (std::isinf(tmn.first) || std::isnan(tmn.first) ||
        std::isinf(tmn.second) || std::isnan(tmn.second))
      throw OrcError(E_UNSHIFT, "Un-shift amounts not finite");
    pd.minflux1 = -tmn.first;
    pd.minflux2 = -tmn.second;
    if (setLog) pd.applyLog();
  }
};

// ======================================================= 2D data binning
// fitsDataDouble.cc:480-608.
struct Data2 {
  std::vector<double> d1, d2;
  bool binned = false;
  unsigned nbins1 = 0, nbins2 = 0;
  std::vector<unsigned> bins;
  double bc1 = 0, bc2 = 0, bd1 = 0, bd2 = 0;
  void meanSubtract() {
    const size_t n = d1.size();
    double m = d1[0];
    for (size_t i = 1; i < n; ++i) m += d1[i];
    m /= static_cast<double>(n);
    for (auto& v : d1) v -= m;
    double m2 = d2[0];
    for (size_t i = 1; i < n; ++i) m2 += d2[i];
    m2 /= static_cast<double>(n);
    for (auto& v : d2) v -= m2;
  }
  void minmax(double* mm) const {
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
  void applyBinning(unsigned nb1, unsigned nb2) {
    nbins1 = nb1; nbins2 = nb2;
    bins.assign(static_cast<size_t>(nb1) * nb2, 0);
    binned = false;
    double mm[4];
    minmax(mm);
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
};

// ============================================================ 2D likelihood
// calcLikeDouble.cc:377-487 (sigma base), 496-534 (R range), 553-616
// (single getLogLike), 1195-1277 (getLogLike).
struct BeamSet2 {
  Beam2 bm;
  std::vector<Data2> data;
  std::vector<double> sb1, sb2, like_offset, like_norm;
  double exp_conf1 = 0, exp_conf2 = 0;
  double maxsb1 = kNaN, maxsb2 = kNaN;
  double mdf[4] = {kNaN, kNaN, kNaN, kNaN};  // min1 max1 min2 max2 data
  double rr[4] = {kNaN, kNaN, kNaN, kNaN};
  PDF2 pdfac;
  PD2 pd;
};

struct Like2 {
  std::vector<std::shared_ptr<Like2>> pool;
  unsigned fftsize = 4096, nedge = 256, nbins = 1000;
  bool edge = true, bin_data = true;
  Counts2 model;
  std::vector<BeamSet2> sets;
  // priors and regularisation (calcLikeDouble.h:213-232)
  bool has_sigma_prior[2] = {false, false}, has_cfirb_prior[2] = {false, false};
  bool has_poisson_prior[2] = {false, false};
  double sigma_prior_width[2] = {0, 0}, cfirb_prior_mean[2] = {0, 0};
  double cfirb_prior_sigma[2] = {0, 0}, poisson_prior_mean[2] = {0, 0};
  double poisson_prior_sigma[2] = {0, 0}, regularization_alpha = 0;

  void refreshSet(BeamSet2& s) {
    s.maxsb1 = s.sb1[0]; s.maxsb2 = s.sb2[0];
    for (size_t i = 1; i < s.sb1.size(); ++i) {
      if (s.sb1[i] > s.maxsb1) s.maxsb1 = s.sb1[i];
      if (s.sb2[i] > s.maxsb2) s.maxsb2 = s.sb2[i];
    }
    for (size_t i = 0; i < s.data.size(); ++i) {
      const double v1 = s.sb1[i] * s.sb1[i] + s.exp_conf1 * s.exp_conf1;
      const double v2 = s.sb2[i] * s.sb2[i] + s.exp_conf2 * s.exp_conf2;
      const double sp = std::sqrt(v1 * v2);
      if (sp > 0) {
        const double ndd = static_cast<double>(s.data[i].d1.size());
        s.like_offset[i] = -ndd * (std::log(kTwoPi * sp) + 1.0);
      }
    }
    double mm[4];
    s.data[0].minmax(mm);
    for (int k = 0; k < 4; ++k) s.mdf[k] = mm[k];
    for (size_t i = 1; i < s.data.size(); ++i) {
      s.data[i].minmax(mm);
      if (mm[0] < s.mdf[0]) s.mdf[0] = mm[0];
      if (mm[1] > s.mdf[1]) s.mdf[1] = mm[1];
      if (mm[2] < s.mdf[2]) s.mdf[2] = mm[2];
      if (mm[3] > s.mdf[3]) s.mdf[3] = mm[3];
    }
  }

  void setRRanges(const float* p, int npar) {
    model.setParams(p, npar);
    if (!model.isValid()) throw OrcError(E_INVALID_MODEL, "Model is not valid");
    const double safetyfac = 1.1;
    for (auto& s : sets) {
      double raw[4];
      model.rrangeInternal(s.bm, raw);
      const double sigma1 = std::sqrt(s.exp_conf1 * s.exp_conf1 + s.maxsb1 * s.maxsb1);
      const double sigma2 = std::sqrt(s.exp_conf2 * s.exp_conf2 + s.maxsb2 * s.maxsb2);
      s.rr[0] = safetyfac * raw[0];
      s.rr[1] = safetyfac * raw[1] + kNZeroPad * sigma1;
      s.rr[2] = safetyfac * raw[2];
      s.rr[3] = safetyfac * raw[3] + kNZeroPad * sigma2;
      const bool* hs = s.bm.hassign;
      if (s.mdf[0] < s.rr[0] && (hs[2] || hs[3])) s.rr[0] = s.mdf[0];
      if (s.mdf[1] > s.rr[1] && (hs[0] || hs[1])) s.rr[1] = s.mdf[1];
      if (s.mdf[2] < s.rr[2] && (hs[1] || hs[3])) s.rr[2] = s.mdf[2];
      if (s.mdf[3] > s.rr[3] && (hs[0] || hs[2])) s.rr[3] = s.mdf[3];
    }
  }

  double singleLogLike(BeamSet2& s, double sm1, double sm2) {
    if (s.maxsb1 * sm1 < 0.0) return kBadLike;
    if (s.maxsb2 * sm2 < 0.0) return kBadLike;
    for (double v : s.rr) if (std::isnan(v)) throw OrcError(E_ARG, "R range not set");
    s.pdfac.nedge = nedge;
    s.pdfac.initPD(fftsize, s.rr[0], s.rr[1], s.rr[2], s.rr[3], model, s.bm, edge);
    double LogLike = 0.0;
    for (size_t i = 0; i < s.data.size(); ++i) {
      s.pdfac.getPD(sm1 * s.sb1[i], sm2 * s.sb2[i], s.pd, true);
      const Data2& d = s.data[i];
      const double cur = d.binned ? s.pd.logLikeBinned(d.bins, d.nbins1, d.nbins2, d.bc1,
                                                       d.bc2, d.bd1, d.bd2)
                                  : s.pd.logLikeUnbinned(d.d1, d.d2);
      LogLike += (cur - s.like_offset[i]) / s.like_norm[i];
    }
    return LogLike;
  }

  double getLogLike(const float* p, int npar) {
    if (sets.empty()) return kNaN;
    const int nm = model.nparams();
    if (npar < nm + 2) throw OrcError(E_ARG, "Not enough elements in params");
    model.setParams(p, npar);
    const double sm1 = p[nm], sm2 = p[nm + 1];
    double LogLike = 0.0;
    for (auto& s : sets) LogLike += singleLogLike(s, sm1, sm2);
    // priors and regularisation (calcLikeDouble.cc:1236-1276)
    const double half_log_2pi = 0.918938517570495605469;
    const double sm[2] = {sm1, sm2};
    for (int b = 0; b < 2; ++b)
      if (has_sigma_prior[b]) {
        const double val = (sm[b] - 1.0) / sigma_prior_width[b];
        LogLike -= half_log_2pi + std::log(sigma_prior_width[b]) + 0.5 * val * val;
      }
    const double mf[2] = {model.splineInt(1.0, 0.0), model.splineInt(0.0, 1.0)};
    for (int b = 0; b < 2; ++b)
      if (has_cfirb_prior[b]) {
        const double val = (cfirb_prior_mean[b] - mf[b]) / cfirb_prior_sigma[b];
        LogLike -= half_log_2pi + std::log(cfirb_prior_sigma[b]) + 0.5 * val * val;
      }
    const double mf2[2] = {model.splineInt(2.0, 0.0), model.splineInt(0.0, 2.0)};
    for (int b = 0; b < 2; ++b)
      if (has_poisson_prior[b]) {
        const double val = (poisson_prior_mean[b] - mf2[b]) / poisson_prior_sigma[b];
        LogLike -= half_log_2pi + std::log(poisson_prior_sigma[b]) + 0.5 * val * val;
      }
    if (regularization_alpha > 0.0) LogLike += model.differenceRegularize(regularization_alpha);
    return LogLike;
  }
};

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const OrcError& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -99;
  }
}

template <class L>
int eval_batch(L* like, int nprop, const float* theta, int npar, double* logl,
               int* status, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > nprop) nthreads = nprop > 0 ? nprop : 1;
  std::atomic<int> next(0);
  auto work = [&](L* L_) {
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= nprop) break;
      double v = kNaN;
      const int st = guard([&] { v = L_->getLogLike(theta + static_cast<size_t>(i) * npar, npar); });
      logl[i] = st == 0 ? v : kNaN;
      status[i] = st;
    }
  };
  if (nthreads == 1) {
    work(like);
    return 0;
  }
  while (static_cast<int>(like->pool.size()) < nthreads - 1) {
    std::shared_ptr<L> c(new L(*like));
    c->pool.clear();
    like->pool.push_back(c);
  }
  std::vector<std::thread> th;
  th.emplace_back(work, like);
  for (int t = 0; t < nthreads - 1; ++t) th.emplace_back(work, like->pool[t].get());
  for (auto& t : th) t.join();
  return 0;
}

}  // namespace orc

using namespace orc;

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_cspline_eval(int n, const double* x, const double* y, int m,
                     const double* xq, double* out) {
  return guard([&] {
    NatSpline s;
    s.init(x, y, n);
    for (int i = 0; i < m; ++i) out[i] = s.eval(xq[i]);
  });
}

int orc_set_fast_fft(int on) {
  set_fast_fft(on != 0);
  return 0;
}
int orc_rfft(int n, const double* in, double* out_c) {
  return guard([&] { rfft(n, in, reinterpret_cast<cplx*>(out_c)); });
}
int orc_irfft(int n, const double* in_c, double* out) {
  return guard([&] { irfft(n, reinterpret_cast<const cplx*>(in_c), out); });
}
int orc_rfft2(int n, const double* in, double* out_c) {
  return guard([&] { rfft2(n, in, reinterpret_cast<cplx*>(out_c)); });
}
int orc_irfft2(int n, const double* in_c, double* out) {
  return guard([&] { irfft2(n, reinterpret_cast<const cplx*>(in_c), out); });
}

// ------------------------------------------------------------- 1D beam
void* orc_beam1_new(const double* pix, int64_t npix, double pixsize,
                    double minval, unsigned nhist) {
  Beam1* b = new Beam1();
  const int st = guard([&] {
    b->set(pix, static_cast<size_t>(npix), pixsize, minval);
    if (nhist > 0) b->makeHistogram(nhist);
  });
  if (st != 0) { delete b; return nullptr; }
  return b;
}
void orc_beam1_free(void* b) { delete static_cast<Beam1*>(b); }
int orc_beam1_info(void* vb, double* o) {
  const Beam1* b = static_cast<Beam1*>(vb);
  o[0] = b->haspos; o[1] = b->hasneg;
  o[2] = static_cast<double>(b->pos.size()); o[3] = static_cast<double>(b->neg.size());
  o[4] = b->posh; o[5] = b->negh;
  o[6] = static_cast<double>(b->poswt.size()); o[7] = static_cast<double>(b->negwt.size());
  o[8] = b->haspos ? b->pos.front() : kNaN; o[9] = b->maxpos();
  o[10] = b->hasneg ? b->neg.front() : kNaN; o[11] = b->maxneg();
  o[12] = b->pixsize; o[13] = b->totpos; o[14] = b->totneg;
  return 0;
}
int orc_beam1_array(void* vb, int which, double* out) {
  const Beam1* b = static_cast<Beam1*>(vb);
  const std::vector<double>* arr[6] = {&b->poswt, &b->posval, &b->negwt,
                                       &b->negval, &b->posinv, &b->neginv};
  if (which < 0 || which > 5) return E_ARG;
  std::copy(arr[which]->begin(), arr[which]->end(), out);
  return 0;
}

// -------------------------------------------------------------- 1D counts
int orc_counts1_eval(int nknots, const double* knotpos, const float* theta,
                     int m, const double* s, double* out) {
  return guard([&] {
    Counts1 c;
    c.setKnots(nknots, knotpos);
    c.setParams(theta, nknots);
    for (int i = 0; i < m; ++i) out[i] = c.counts(s[i]);
  });
}
int orc_counts1_getR(int nknots, const double* knotpos, const float* theta,
                     void* beam, int m, const double* flux, double* out,
                     int scalar_version) {
  return guard([&] {
    Counts1 c;
    c.setKnots(nknots, knotpos);
    c.setParams(theta, nknots);
    const Beam1& bm = *static_cast<Beam1*>(beam);
    if (scalar_version)
      for (int i = 0; i < m; ++i) out[i] = c.getRScalar(flux[i], bm);
    else
      c.getR(m, flux, bm, out);
  });
}
int orc_counts1_rrange(int nknots, const double* knotpos, const float* theta,
                       void* beam, double* r) {
  return guard([&] {
    Counts1 c;
    c.setKnots(nknots, knotpos);
    c.setParams(theta, nknots);
    const auto rr = c.rrange(*static_cast<Beam1*>(beam));
    r[0] = rr.first; r[1] = rr.second;
  });
}
int orc_counts1_integrals(int nknots, const double* knotpos,
                          const float* theta, double* o) {
  return guard([&] {
    Counts1 c;
    c.setKnots(nknots, knotpos);
    c.setParams(theta, nknots);
    o[0] = c.splineInt(0); o[1] = c.splineInt(1); o[2] = c.splineInt(2);
  });
}

// ---------------------------------------------------------- 1D likelihood
void* orc_like1_new(int nknots, const double* knotpos, unsigned fftsize,
                    unsigned ninterp, int bin_data, unsigned nbins) {
  Like1* L = new Like1();
  L->model.setKnots(nknots, knotpos);
  L->fftsize = fftsize; L->ninterp = ninterp;
  L->bin_data = bin_data != 0; L->nbins = nbins;
  return L;
}
void orc_like1_free(void* L) { delete static_cast<Like1*>(L); }
int orc_like1_add_beamset(void* vL, const double* beampix, int64_t nbeampix,
                          double pixsize, double minval, int histogram,
                          unsigned nbeamhist, double exp_conf) {
  static_cast<Like1*>(vL)->pool.clear();
  Like1* L = static_cast<Like1*>(vL);
  int idx = -1;
  const int st = guard([&] {
    BeamSet1 s;
    s.bm.set(beampix, static_cast<size_t>(nbeampix), pixsize, minval);
    if (histogram) s.bm.makeHistogram(nbeamhist);
    s.exp_conf = exp_conf;
    L->sets.push_back(std::move(s));
    idx = static_cast<int>(L->sets.size()) - 1;
  });
  return st != 0 ? st : idx;
}
int orc_like1_add_dataset(void* vL, int bs, const double* data, int64_t nd,
                          int meansub, double sigma_base, double like_norm) {
  static_cast<Like1*>(vL)->pool.clear();
  Like1* L = static_cast<Like1*>(vL);
  return guard([&] {
    if (bs < 0 || bs >= static_cast<int>(L->sets.size())) throw OrcError(E_ARG, "bad beam set");
    if (nd <= 0) throw OrcError(E_ARG, "No pixels in data");
    BeamSet1& s = L->sets[bs];
    Data1 d;
    d.data.assign(data, data + nd);
    if (meansub) d.meanSubtract();
    if (L->bin_data) d.applyBinning(L->nbins);
    s.data.push_back(std::move(d));
    s.sigma_base.push_back(sigma_base);
    s.like_offset.push_back(0.0);
    s.like_norm.push_back(like_norm);
    L->refreshSet(s);
  });
}
int orc_like1_set_rranges(void* vL, const float* theta, int npar) {
  static_cast<Like1*>(vL)->pool.clear();
  return guard([&] { static_cast<Like1*>(vL)->setRRanges(theta, npar); });
}
int orc_like1_get_rrange(void* vL, int bs, double* r) {
  Like1* L = static_cast<Like1*>(vL);
  if (bs < 0 || bs >= static_cast<int>(L->sets.size())) return E_ARG;
  r[0] = L->sets[bs].minRFlux; r[1] = L->sets[bs].maxRFlux;
  return 0;
}
int orc_like1_dataset_info(void* vL, int bs, int ds, double* o) {
  Like1* L = static_cast<Like1*>(vL);
  const BeamSet1& s = L->sets.at(bs);
  const Data1& d = s.data.at(ds);
  o[0] = static_cast<double>(d.data.size()); o[1] = d.nbins;
  o[2] = d.bincent0; o[3] = d.bindelta; o[4] = s.like_offset[ds];
  o[5] = s.sigma_base[ds]; o[6] = s.like_norm[ds];
  o[7] = s.minDataFlux; o[8] = s.maxDataFlux;
  return 0;
}
int orc_like1_dataset_bins(void* vL, int bs, int ds, uint32_t* out) {
  Like1* L = static_cast<Like1*>(vL);
  const Data1& d = L->sets.at(bs).data.at(ds);
  std::copy(d.bins.begin(), d.bins.end(), out);
  return 0;
}
int orc_like1_set_priors(void* vL, const double* p9) {
  Like1* L = static_cast<Like1*>(vL);
  L->pool.clear();
  L->has_sigma_prior = p9[0] != 0.0;
  L->sigma_prior_width = p9[1];
  L->has_cfirb_prior = p9[2] != 0.0;
  L->cfirb_prior_mean = p9[3];
  L->cfirb_prior_sigma = p9[4];
  L->has_poisson_prior = p9[5] != 0.0;
  L->poisson_prior_mean = p9[6];
  L->poisson_prior_sigma = p9[7];
  L->regularization_alpha = p9[8];
  return 0;
}
int orc_like1_bonus(void* vL, const float* theta, int npar, double* out2) {
  Like1* L = static_cast<Like1*>(vL);
  return guard([&] {
    L->model.setParams(theta, npar);
    out2[0] = L->model.splineInt(1.0);
    out2[1] = L->model.splineInt(2.0);
  });
}
int orc_like1_eval(void* vL, const float* theta, int npar, double* logl) {
  return guard([&] { *logl = static_cast<Like1*>(vL)->getLogLike(theta, npar); });
}
int orc_like1_eval_batch(void* vL, int nprop, const float* theta, int npar,
                         double* logl, int* status, int nthreads) {
  return eval_batch(static_cast<Like1*>(vL), nprop, theta, npar, logl, status,
                    nthreads);
}
int orc_like1_pd(void* vL, int bs, int ds, const float* theta, int npar,
                 int setlog, double* pd_out, double* dbg, double* rvals_out) {
  Like1* L = static_cast<Like1*>(vL);
  return guard([&] {
    BeamSet1& s = L->sets.at(bs);
    const int nk = static_cast<int>(L->model.knots.size());
    L->model.setParams(theta, npar);
    const double sigmult = theta[nk];
    s.pdfac.ninterp = L->ninterp;
    s.pdfac.initPD(L->fftsize, s.minRFlux, s.maxRFlux, L->model, s.bm);
    if (rvals_out) std::copy(s.pdfac.rvals.begin(), s.pdfac.rvals.end(), rvals_out);
    const double r0_dbg = 0.0;
    s.pdfac.getPD(sigmult * s.sigma_base.at(ds), s.pd, setlog != 0);
    std::copy(s.pd.pd.begin(), s.pd.pd.end(), pd_out);
    if (dbg) {
      const PDF1& f = s.pdfac;
      dbg[0] = f.dflux; dbg[1] = f.minflux_R; dbg[2] = f.wrapRidx;
      dbg[3] = f.mn; dbg[4] = f.var_noi; dbg[5] = f.doshift; dbg[6] = f.shift;
      dbg[7] = f.lastsplit; dbg[8] = f.sgpos; dbg[9] = f.sgneg;
      dbg[10] = s.pd.minflux; dbg[11] = r0_dbg;
    }
  });
}
int orc_like1_rinterp(void* vL, int bs, const float* theta, int npar, int neg,
                      double* x_out, double* r_out) {
  Like1* L = static_cast<Like1*>(vL);
  return guard([&] {
    BeamSet1& s = L->sets.at(bs);
    L->model.setParams(theta, npar);
    s.pdfac.ninterp = L->ninterp;
    s.pdfac.initRInterp(L->model, s.bm);
    const auto& x = neg ? s.pdfac.xneg : s.pdfac.xpos;
    const auto& r = neg ? s.pdfac.rneg : s.pdfac.rpos;
    std::copy(x.begin(), x.end(), x_out);
    std::copy(r.begin(), r.end(), r_out);
  });
}

// ------------------------------------------------------------- 2D beam
void* orc_beam2_new(const double* p1, const double* p2, int64_t npix,
                    double pixsize, double minval, unsigned nhist) {
  Beam2* b = new Beam2();
  const int st = guard([&] {
    b->set(p1, p2, static_cast<size_t>(npix), pixsize, minval);
    if (nhist > 0) b->makeHistogram(nhist);
  });
  if (st != 0) { delete b; return nullptr; }
  return b;
}
void orc_beam2_free(void* b) { delete static_cast<Beam2*>(b); }
int orc_beam2_info(void* vb, double* o) {
  const Beam2* b = static_cast<Beam2*>(vb);
  for (int s = 0; s < 4; ++s) {
    o[s] = b->hassign[s];
    o[4 + s] = static_cast<double>(b->pix1[s].size());
    o[8 + s] = b->ishist[s];
    o[12 + s] = static_cast<double>(b->binwt[s].size());
  }
  o[16] = b->pixsize;
  return 0;
}
int orc_beam2_array(void* vb, int sgn, int which, double* out) {
  const Beam2* b = static_cast<Beam2*>(vb);
  if (sgn < 0 || sgn > 3) return E_ARG;
  const bool h = b->ishist[sgn];
  switch (which) {
    case 0:
      if (h) std::copy(b->binwt[sgn].begin(), b->binwt[sgn].end(), out);
      else std::fill(out, out + b->pix1[sgn].size(), 1.0);
      break;
    case 1: {
      const auto& a = h ? b->binv1[sgn] : b->inv1[sgn];
      std::copy(a.begin(), a.end(), out);
      break;
    }
    case 2: {
      const auto& a = h ? b->binv2[sgn] : b->inv2[sgn];
      std::copy(a.begin(), a.end(), out);
      break;
    }
    case 3: {
      const auto& a = h ? b->binlogratio[sgn] : b->logratio[sgn];
      std::copy(a.begin(), a.end(), out);
      break;
    }
    default: return E_ARG;
  }
  return 0;
}
int orc_beam2_minmax(void* vb, int s, double* mm) {
  const Beam2* b = static_cast<Beam2*>(vb);
  mm[0] = b->minbm1[s]; mm[1] = b->maxbm1[s]; mm[2] = b->minbm2[s]; mm[3] = b->maxbm2[s];
  return 0;
}

// -------------------------------------------------------------- 2D counts
void* orc_counts2_new(int nk, const double* kp, int ns, const double* sp,
                      int no, const double* op) {
  Counts2* m = new Counts2();
  const int st = guard([&] { m->setPositions(nk, kp, ns, sp, no, op); });
  if (st != 0) { delete m; return nullptr; }
  return m;
}
void orc_counts2_free(void* m) { delete static_cast<Counts2*>(m); }
int orc_counts2_set(void* m, const float* theta, int npar) {
  return guard([&] { static_cast<Counts2*>(m)->setParams(theta, npar); });
}
int orc_counts2_eval(void* vm, int n, const double* f1, const double* f2,
                     double* out) {
  return guard([&] {
    const Counts2* m = static_cast<Counts2*>(vm);
    for (int i = 0; i < n; ++i) out[i] = m->counts(f1[i], f2[i]);
  });
}
int orc_counts2_getR(void* vm, void* beam, int n1, const double* f1, int n2,
                     const double* f2, double* out) {
  return guard([&] {
    static_cast<Counts2*>(vm)->getR(n1, f1, n2, f2, *static_cast<Beam2*>(beam), out);
  });
}
int orc_counts2_getR_scalar(void* vm, void* beam, int n, const double* f1,
                            const double* f2, double* out) {
  return guard([&] {
    const Counts2* m = static_cast<Counts2*>(vm);
    for (int i = 0; i < n; ++i) out[i] = m->getRScalar(f1[i], f2[i], *static_cast<Beam2*>(beam));
  });
}
int orc_counts2_maxflux(void* vm, double* mm) {
  return guard([&] {
    const auto r = static_cast<Counts2*>(vm)->maxFlux();
    mm[0] = r.first; mm[1] = r.second;
  });
}
int orc_counts2_spline_int(void* vm, double alpha, double beta, double* out) {
  return guard([&] { *out = static_cast<Counts2*>(vm)->splineInt(alpha, beta); });
}
int orc_counts2_rrange(void* vm, void* beam, double* r) {
  return guard([&] {
    const Counts2* m = static_cast<Counts2*>(vm);
    if (!m->isValid()) throw OrcError(E_INVALID_MODEL, "Model is not valid");
    m->rrangeInternal(*static_cast<Beam2*>(beam), r);
  });
}
int orc_counts2_sigma_offset(void* vm, int n, const double* f1, double* sig,
                             double* off) {
  return guard([&] {
    const Counts2* m = static_cast<Counts2*>(vm);
    for (int i = 0; i < n; ++i) { sig[i] = m->sigmaInner(f1[i]); off[i] = m->offsetInner(f1[i]); }
  });
}

// ---------------------------------------------------------- 2D likelihood
void* orc_like2_new(int nk, const double* kp, int ns, const double* sp, int no,
                    const double* op, unsigned fftsize, unsigned nedge,
                    int edge_integ, int bin_data, unsigned nbins) {
  Like2* L = new Like2();
  const int st = guard([&] { L->model.setPositions(nk, kp, ns, sp, no, op); });
  if (st != 0) { delete L; return nullptr; }
  L->fftsize = fftsize; L->nedge = nedge; L->edge = edge_integ != 0;
  L->bin_data = bin_data != 0; L->nbins = nbins;
  return L;
}
void orc_like2_free(void* L) { delete static_cast<Like2*>(L); }
int orc_like2_add_beamset(void* vL, const double* p1, const double* p2,
                          int64_t npix, double pixsize, double minval,
                          int histogram, unsigned nbeamhist, double ec1,
                          double ec2) {
  static_cast<Like2*>(vL)->pool.clear();
  Like2* L = static_cast<Like2*>(vL);
  int idx = -1;
  const int st = guard([&] {
    BeamSet2 s;
    s.bm.set(p1, p2, static_cast<size_t>(npix), pixsize, minval);
    if (histogram) s.bm.makeHistogram(nbeamhist);
    s.exp_conf1 = ec1; s.exp_conf2 = ec2;
    L->sets.push_back(std::move(s));
    idx = static_cast<int>(L->sets.size()) - 1;
  });
  return st != 0 ? st : idx;
}
int orc_like2_add_dataset(void* vL, int bs, const double* d1, const double* d2,
                          int64_t nd, int meansub, double sb1, double sb2,
                          double like_norm) {
  static_cast<Like2*>(vL)->pool.clear();
  Like2* L = static_cast<Like2*>(vL);
  return guard([&] {
    if (bs < 0 || bs >= static_cast<int>(L->sets.size())) throw OrcError(E_ARG, "bad beam set");
    if (nd <= 0) throw OrcError(E_ARG, "No pixels in data");
    BeamSet2& s = L->sets[bs];
    Data2 d;
    d.d1.assign(d1, d1 + nd);
    d.d2.assign(d2, d2 + nd);
    if (meansub) d.meanSubtract();
    if (L->bin_data) d.applyBinning(L->nbins, L->nbins);
    s.data.push_back(std::move(d));
    s.sb1.push_back(sb1); s.sb2.push_back(sb2);
    s.like_offset.push_back(0.0);
    s.like_norm.push_back(like_norm);
    L->refreshSet(s);
  });
}
int orc_like2_set_rranges(void* vL, const float* theta, int npar) {
  static_cast<Like2*>(vL)->pool.clear();
  return guard([&] { static_cast<Like2*>(vL)->setRRanges(theta, npar); });
}
int orc_like2_get_rrange(void* vL, int bs, double* r) {
  Like2* L = static_cast<Like2*>(vL);
  if (bs < 0 || bs >= static_cast<int>(L->sets.size())) return E_ARG;
  for (int k = 0; k < 4; ++k) r[k] = L->sets[bs].rr[k];
  return 0;
}
int orc_like2_dataset_info(void* vL, int bs, int ds, double* o) {
  Like2* L = static_cast<Like2*>(vL);
  const BeamSet2& s = L->sets.at(bs);
  const Data2& d = s.data.at(ds);
  o[0] = static_cast<double>(d.d1.size()); o[1] = d.nbins1;
  o[2] = d.bc1; o[3] = d.bc2; o[4] = d.bd1; o[5] = d.bd2;
  o[6] = s.like_offset[ds]; o[7] = s.sb1[ds]; o[8] = s.sb2[ds]; o[9] = s.like_norm[ds];
  return 0;
}
int orc_like2_dataset_bins(void* vL, int bs, int ds, uint32_t* out) {
  Like2* L = static_cast<Like2*>(vL);
  const Data2& d = L->sets.at(bs).data.at(ds);
  std::copy(d.bins.begin(), d.bins.end(), out);
  return 0;
}
int orc_like2_set_priors(void* vL, const double* p17) {
  Like2* L = static_cast<Like2*>(vL);
  L->pool.clear();
  for (int b = 0; b < 2; ++b) {
    const double* q = p17 + 8 * b;
    L->has_sigma_prior[b] = q[0] != 0.0;
    L->sigma_prior_width[b] = q[1];
    L->has_cfirb_prior[b] = q[2] != 0.0;
    L->cfirb_prior_mean[b] = q[3];
    L->cfirb_prior_sigma[b] = q[4];
    L->has_poisson_prior[b] = q[5] != 0.0;
    L->poisson_prior_mean[b] = q[6];
    L->poisson_prior_sigma[b] = q[7];
  }
  L->regularization_alpha = p17[16];
  return 0;
}
int orc_like2_bonus(void* vL, const float* theta, int npar, double* out4) {
  Like2* L = static_cast<Like2*>(vL);
  return guard([&] {
    L->model.setParams(theta, npar);
    out4[0] = L->model.splineInt(1.0, 0.0);
    out4[1] = L->model.splineInt(0.0, 1.0);
    out4[2] = L->model.splineInt(2.0, 0.0);
    out4[3] = L->model.splineInt(0.0, 2.0);
  });
}
int orc_like2_eval(void* vL, const float* theta, int npar, double* logl) {
  return guard([&] { *logl = static_cast<Like2*>(vL)->getLogLike(theta, npar); });
}
int orc_like2_eval_batch(void* vL, int nprop, const float* theta, int npar,
                         double* logl, int* status, int nthreads) {
  return eval_batch(static_cast<Like2*>(vL), nprop, theta, npar, logl, status,
                    nthreads);
}
int orc_like2_pd(void* vL, int bs, int ds, const float* theta, int npar,
                 int setlog, double* pd_out, double* dbg, double* rvals_out) {
  Like2* L = static_cast<Like2*>(vL);
  return guard([&] {
    BeamSet2& s = L->sets.at(bs);
    const int nm = L->model.nparams();
    L->model.setParams(theta, npar);
    const double sm1 = theta[nm], sm2 = theta[nm + 1];
    s.pdfac.nedge = L->nedge;
    s.pdfac.initPD(L->fftsize, s.rr[0], s.rr[1], s.rr[2], s.rr[3], L->model, s.bm, L->edge);
    if (rvals_out) std::copy(s.pdfac.rvals.begin(), s.pdfac.rvals.end(), rvals_out);
    s.pdfac.getPD(sm1 * s.sb1.at(ds), sm2 * s.sb2.at(ds), s.pd, setlog != 0);
    std::copy(s.pd.pd.begin(), s.pd.pd.end(), pd_out);
    if (dbg) {
      const PDF2& f = s.pdfac;
      dbg[0] = f.dflux1; dbg[1] = f.dflux2; dbg[2] = f.mn1; dbg[3] = f.mn2;
      dbg[4] = f.var1; dbg[5] = f.var2; dbg[6] = f.shift1; dbg[7] = f.shift2;
      dbg[8] = f.lastsplit1; dbg[9] = f.lastsplit2;
      dbg[10] = s.pd.minflux1; dbg[11] = s.pd.minflux2;
      dbg[12] = f.sg1pos; dbg[13] = f.sg1neg; dbg[14] = f.sg2pos; dbg[15] = f.sg2neg;
    }
  });
}

}  // extern "C"
