// setup.hh -- host-side, theta-independent set-up of the P(D) likelihood.
//
// This is the once-per-run work the reference does before sampling: beam
// pixel selection and log-binned histogram (beam.cc:295-556,
// doublebeam.cc:331-584), data mean subtraction and binning
// (fitsData.cc:393-437, fitsDataDouble.cc:480-608), likelihood offsets
// (calcLike.cc:283-308, calcLikeDouble.cc:377-487) and the frozen R ranges
// (calcLike.cc:346-371, calcLikeDouble.cc:496-534).  It also precomputes
// everything of the per-proposal path that does not depend on the
// parameters -- the R interpolation nodes, the natural-spline system
// factorisation over them and the wrapped flux grids -- so that the GPU
// kernels only do parameter-dependent work.
#ifndef POFD_SETUP_HH
#define POFD_SETUP_HH

#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pofd_b200.h"

namespace pofd {

struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

constexpr double kPi = 3.141592653589793238462643383279502884197;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kSmallLogVal = -30.0;  // pofd_mcmc::smalllogval
constexpr double kNZeroPad = 7.5;       // pofd_mcmc::n_zero_pad
constexpr double kBadLike = 1e25;       // calcLike::bad_like
inline double logfac() { return std::log2(10.0); }
inline double log2toe() { return std::log(2.0); }
inline double nan() { return std::numeric_limits<double>::quiet_NaN(); }

// ------------------------------------------------------------- 1D beam
struct Beam1 {
  bool haspos = false, hasneg = false;
  double pixsize = 0, minval = 0;
  std::vector<double> pos, neg;        // sorted |values| > minval
  std::vector<double> posinv, neginv;  // 1 / values
  double totpos = 0, totneg = 0;
  bool poshist = false, neghist = false;
  std::vector<double> poswt, posival, negwt, negival;  // histogram

  void build(const double* pix, size_t n, double PIXSIZE, double MINVAL);
  void histogram(unsigned nbins);
  double maxpos() const { return haspos ? pos.back() : nan(); }
  double maxneg() const { return hasneg ? neg.back() : nan(); }
  // Terms the R sum runs over for one side (weights 1 for a raw beam).  The
  // negative side follows beam::isNegHist(), which reports the positive
  // side's histogram flag (beam.h:86).
  void terms(bool negside, std::vector<double>& w,
             std::vector<double>& ieta) const;
};

// Natural cubic spline through nodes x: the x-only part of the tridiagonal
// system (LDL^T factors) and 1/h, so that per-parameter work is the RHS
// and two first-order recurrences.
struct SplineSystem {
  std::vector<double> x, ih, alpha, gamma;  // ih: 1/h_i (n-1); alpha,gamma: n-2
  void factor(const std::vector<double>& xn);
};

// Data set: mean-subtracted pixels, binned.
struct Data1 {
  std::vector<double> data;  // pixels (may be empty once binned elsewhere)
  size_t npix = 0;           // pixel count when data is empty
  size_t count() const { return data.empty() ? npix : data.size(); }
  bool binned = false;
  unsigned nbins = 0;
  std::vector<uint32_t> bins;
  double bincent0 = 0, bindelta = 0;
  void meanSubtract();
  std::pair<double, double> minmax() const;
  void applyBinning(unsigned nbins);
};

// Mean subtraction and binning of maps in device memory (ingest.cu),
// bit-identical to Data1 / Data2's: info3 = {mean, bincent0, bindelta},
// info6 = {mean1, mean2, bincent01, bindelta1, bincent02, bindelta2}.
// stream: a cudaStream_t.
void ingest_bin1(double* x_dev, size_t n, bool meansub, unsigned nb, unsigned* bins_dev,
                 double* info3, void* stream);
void ingest_bin2(double* x1_dev, double* x2_dev, size_t n, bool meansub, unsigned nb1,
                 unsigned nb2, unsigned* bins_dev, double* info6, void* stream);

// The wrapped R flux grid of PDFactory::initRFlux (PDFactory.cc:361-414).
struct RGrid1 {
  unsigned n = 0, wrapRidx = 0;
  double dflux = 0, minflux_R = 0;
  void init(unsigned N, double minflux, double maxflux);
};

// The flux range of a knot model over a beam (numberCountsKnots.cc:345-365).
std::pair<double, double> rrange_knots(double maxknot, const Beam1& bm);

// Gauss-Legendre rule of order q on [-1, 1], nodes ascending: Newton
// iterations on the three-term Legendre recurrence, in long double.
void gauss_legendre(int q, std::vector<double>& x, std::vector<double>& w);

// Quadrature nodes for integrals of S^a dN/dS over [S_0, S_{K-1}] written in
// u = log2 S (dS = ln2 2^u du): each knot interval [u_k, u_{k+1}] is cut into
// `panels` equal panels with a q-point Gauss-Legendre rule each.  Node j lies
// in knot interval j / nper (nper = panels * q); s = 2^u and w = ln2 * h/2 *
// w_g, so that the integral is sum_j w_j s_j^{a+1} 2^{spline(u_j)}.
struct KnotQuadrature {
  std::vector<double> u, s, w;
  std::vector<int> kidx;  // knot interval of each node
  int nper = 0;
  void build(const double* logknots, int K, int panels, int q);
  // The same with extra breakpoints (log2 S, strictly inside the knot range)
  // splitting the knot intervals, for integrands with kinks there; nper is
  // then the nodes per sub-interval and kidx the only interval map.
  void build_breaks(const double* logknots, int K, std::vector<double> extra, int panels,
                    int q);
};

// ------------------------------------------------------------- 2D beam
struct Beam2 {
  double pixsize = 0, minval = 0;
  bool hassign[4] = {false, false, false, false};
  std::vector<double> pix1[4], pix2[4];  // |values|, input order
  std::vector<double> inv1[4], inv2[4], logratio[4];
  double minbm1[4], maxbm1[4], minbm2[4], maxbm2[4];
  bool ishist[4] = {false, false, false, false};
  std::vector<double> binwt[4], binv1[4], binv2[4], binlogratio[4];

  void build(const double* b1, const double* b2, size_t n, double PIXSIZE,
             double MINVAL);
  void histogram(unsigned nbins);
  bool hasData() const {
    return hassign[0] || hassign[1] || hassign[2] || hassign[3];
  }
  // Terms of one sign component: weights (1 for raw), inverse beam 1,
  // inverse beam 2, log(beam1/beam2).
  size_t nterms(int s) const {
    return hassign[s] ? (ishist[s] ? binwt[s].size() : pix1[s].size()) : 0;
  }
};

struct Data2 {
  std::vector<double> d1, d2;  // pixels (may be empty once binned elsewhere)
  size_t npix = 0;             // pixel count when d1 is empty
  size_t count() const { return d1.empty() ? npix : d1.size(); }
  unsigned nbins1 = 0, nbins2 = 0;
  std::vector<uint32_t> bins;
  double bc1 = 0, bc2 = 0, bd1 = 0, bd2 = 0;
  bool binned = false;
  void meanSubtract();
  void minmax(double* mm4) const;
  void applyBinning(unsigned nb1, unsigned nb2);
};

// PDFactoryDouble's wrapped grid along one axis (PDFactoryDouble.cc:18-49).
struct RGrid2Axis {
  unsigned n = 0, wrapidx = 0;
  double dflux = 0;
  std::vector<double> flux;
  void init(unsigned N, double minflux, double maxflux);
};



// Natural cubic spline (host), per-interval y,b,c,d as the reference's
// spline library forms them at evaluation (used for the 2D model's sigma
// and offset curves and its knot counts on the host).
struct NatSpline {
  std::vector<double> x, y, b, c, d;
  void init(const double* xa, const double* ya, size_t n);
  size_t find(double v) const;
  double eval(double v) const;
};

// Log-normal colour model on the host (numberCountsDoubleLogNormal.cc:
// setParams 1010-1052, getSigmaInner 1172-1179, getOffsetInner 1187-1193,
// getMaxFlux 1365-1379, logNormalSolver 1389-1472, getRRangeInternal
// 1481-1521): only what the frozen R range needs.
struct Model2Host {
  std::vector<double> knots, sigk, offk;
  std::vector<double> sigv, offv;
  NatSpline sigspl, offspl;
  double min_sigma = 0.0;
  void set(const std::vector<double>& k, const std::vector<double>& s,
           const std::vector<double>& o, const float* theta);
  double sigma(double f1) const;
  double offset(double f1) const;
  double logNormalSolver(double mu, double sig, double nsig) const;
  std::pair<double, double> maxFlux() const;
  void rrange(const Beam2& bm, double* r4) const;
};

}  // namespace pofd
#endif
