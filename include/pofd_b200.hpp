// pofd_b200.hpp -- header-only C++ shim over the C ABI (pofd_b200.h) with
// the reference's class shapes, for dropping into the pofd_affine C++ code.
//
//   pofd_b200::Context ctx(0);
//   pofd_b200::Beam1 bm(pixels, npix, pixsize, true, 120, 1e-5);
//   pofd_b200::Like1 like(ctx, knotpos, fftsize, ninterp, true, nbins);
//   like.addBeamSet(bm); like.addDataset(0, data, ndata, sigma);
//   like.setRRanges(theta, npar);
//   double L = like.getLogLike(theta, npar, pars_invalid);   // calcLike.h:275
//   like.getLogLikeBatch(nprop, thetas, npar, logl, status); // batched
//
// The 2D likelihood likewise: Beam2 (doublebeam) and Like2 (calcLikeDouble,
// priors per band, fillBonusParams).
//
// Errors are thrown as pofd_b200::Exception carrying the status code and the
// library's message, in the place where the reference throws affineExcept.
#ifndef POFD_B200_HPP
#define POFD_B200_HPP

#include <cmath>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "pofd_b200.h"

namespace pofd_b200 {

class Exception : public std::runtime_error {
 public:
  Exception(int code, const std::string& method)
      : std::runtime_error(method + ": " + pofd_last_error()), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline int check(int st, const char* method) {
  if (st < 0) throw Exception(st, method);
  return st;
}

// FITS reading through the library (fitsData::readData, beam::readFile).
inline std::vector<double> readFitsData(const std::string& path, bool ignore_mask,
                                        bool meansub) {
  size_t n = 0;
  check(pofd_fits_read_data(path.c_str(), ignore_mask, meansub, nullptr, 0, &n),
        "fitsData::readData");
  std::vector<double> d(n);
  check(pofd_fits_read_data(path.c_str(), ignore_mask, meansub, d.data(), n, &n),
        "fitsData::readData");
  return d;
}
inline void readFitsData2(const std::string& p1, const std::string& p2, bool ignore_mask,
                          bool meansub, std::vector<double>& d1, std::vector<double>& d2) {
  size_t n = 0;
  check(pofd_fits_read_data2(p1.c_str(), p2.c_str(), ignore_mask, meansub, nullptr, nullptr,
                             0, &n),
        "fitsDataDouble::readData");
  d1.resize(n);
  d2.resize(n);
  check(pofd_fits_read_data2(p1.c_str(), p2.c_str(), ignore_mask, meansub, d1.data(),
                             d2.data(), n, &n),
        "fitsDataDouble::readData");
}
inline std::vector<double> readFitsBeam(const std::string& path, double& pixsize) {
  size_t nx = 0, ny = 0;
  check(pofd_fits_read_beam(path.c_str(), nullptr, 0, &nx, &ny, &pixsize), "beam::readFile");
  std::vector<double> b(nx * ny);
  check(pofd_fits_read_beam(path.c_str(), b.data(), b.size(), &nx, &ny, &pixsize),
        "beam::readFile");
  return b;
}

class Context {
 public:
  explicit Context(int device = 0) {
    check(pofd_ctx_create(device, &h_), "pofd_ctx_create");
  }
  ~Context() { pofd_ctx_destroy(h_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  pofd_ctx* get() const { return h_; }

 private:
  pofd_ctx* h_ = nullptr;
};

// beam::beam(filename, histogram, NBINS, MINVAL) from a pixel array.
class Beam1 {
 public:
  Beam1(const double* pix, size_t npix, double pixsize, bool histogram = false,
        unsigned nbins = 120, double minval = 1e-5) {
    check(pofd_beam1_create(pix, npix, pixsize, minval,
                            histogram ? nbins : 0u, &h_),
          "beam::beam");
  }
  ~Beam1() { pofd_beam1_destroy(h_); }
  Beam1(const Beam1&) = delete;
  Beam1& operator=(const Beam1&) = delete;
  const pofd_beam1* get() const { return h_; }
  bool hasPos() const { return info(0) != 0.0; }
  bool hasNeg() const { return info(1) != 0.0; }

 private:
  double info(int i) const {
    double o[15];
    check(pofd_beam1_info(h_, o), "beam::info");
    return o[i];
  }
  pofd_beam1* h_ = nullptr;
};

// PDFactory (PDFactory.h:136-140).
class PDFactory1 {
 public:
  explicit PDFactory1(Context& ctx, unsigned ninterp = 2048) {
    check(pofd_pdfactory1_create(ctx.get(), ninterp, &h_), "PDFactory");
  }
  ~PDFactory1() { pofd_pdfactory1_destroy(h_); }
  PDFactory1(const PDFactory1&) = delete;
  PDFactory1& operator=(const PDFactory1&) = delete;
  bool initPD(unsigned n, double minflux, double maxflux, unsigned nknots,
              const double* knotpos, const float* knotvals, const Beam1& bm) {
    check(pofd_pdfactory1_initpd(h_, n, minflux, maxflux, nknots, knotpos,
                                 knotvals, bm.get()),
          "PDFactory::initPD");
    n_ = n;
    return true;
  }
  // Fills pd (n values), returns the flux of element 0; dflux via *dflux.
  double getPD(double sigma, std::vector<double>& pd, bool setLog = true,
               double* dflux = nullptr) {
    pd.resize(n_);
    double mf = 0.0, df = 0.0;
    check(pofd_pdfactory1_getpd(h_, sigma, setLog ? 1 : 0, pd.data(), &mf, &df),
          "PDFactory::getPD");
    if (dflux) *dflux = df;
    return mf;
  }

 private:
  pofd_pdfactory1* h_ = nullptr;
  unsigned n_ = 0;
};

// calcLike (calcLike.h:166-275).
class Like1 {
 public:
  Like1(Context& ctx, unsigned nknots, const double* knotpos,
        unsigned fftsize = 131072, unsigned ninterp = 2048,
        bool bin_data = true, unsigned nbins = 1000) {
    check(pofd_like1_create(ctx.get(), nknots, knotpos, fftsize, ninterp,
                            bin_data ? 1 : 0, nbins, &h_),
          "calcLike::calcLike");
  }
  ~Like1() { pofd_like1_destroy(h_); }
  Like1(const Like1&) = delete;
  Like1& operator=(const Like1&) = delete;
  int addBeamSet(const Beam1& bm, double exp_conf = 0.0) {
    return check(pofd_like1_add_beamset(h_, bm.get(), exp_conf),
                 "calcLike::readDataFromFiles");
  }
  void addDataset(int beamset, const double* data, size_t ndata,
                  double sigma_base, double like_norm = 1.0,
                  bool meansub = true) {
    check(pofd_like1_add_dataset(h_, beamset, data, ndata, meansub ? 1 : 0,
                                 sigma_base, like_norm),
          "calcLike::readDataFromFiles");
  }
  // calcLike::readDataFromFiles (calcLike.h:218-223, calcLike.cc:688-758):
  // datasets grouped by beam file, the groups in file-name order (the
  // reference's std::map), each group's datasets in input order
  void readDataFromFiles(const std::vector<std::string>& datafiles,
                         const std::vector<std::string>& beamfiles,
                         const std::vector<double>& sigmas,
                         const std::vector<double>& like_norms, bool IGNOREMASK = false,
                         bool MEANSUB = false, double MINBEAMVAL = 1e-5,
                         bool HISTOGRAMBEAMS = false, unsigned int NBEAMHIST = 120,
                         double EXPCONF = 0.0) {
    const size_t n = datafiles.size();
    if (n == 0) throw std::runtime_error("calcLike::readDataFromFiles: No datafiles");
    if (n != beamfiles.size() || n != sigmas.size() || n != like_norms.size())
      throw std::runtime_error("calcLike::readDataFromFiles: inputs not same length");
    std::map<std::string, std::vector<size_t>> groups;
    for (size_t i = 0; i < n; ++i) groups[beamfiles[i]].push_back(i);
    for (const auto& g : groups) {
      double ps = 0.0;
      const std::vector<double> pix = readFitsBeam(g.first, ps);
      Beam1 bm(pix.data(), pix.size(), ps, HISTOGRAMBEAMS, NBEAMHIST, MINBEAMVAL);
      const int bs = addBeamSet(bm, EXPCONF);
      for (size_t i : g.second) {
        const std::vector<double> d = readFitsData(datafiles[i], IGNOREMASK, false);
        addDataset(bs, d.data(), d.size(), sigmas[i], like_norms[i], MEANSUB);
      }
    }
  }
  void setRRanges(const float* p, unsigned npar) {
    check(pofd_like1_set_rranges(h_, p, npar), "calcLike::setRRanges");
  }
  void reserve(unsigned max_batch) {
    check(pofd_like1_reserve(h_, max_batch), "calcLike::reserve");
  }
  double getLogLike(const float* p, unsigned npar, bool& pars_invalid) {
    double ll = 0.0;
    int inv = 0;
    check(pofd_like1_loglike(h_, p, npar, &ll, &inv), "calcLike::getLogLike");
    pars_invalid = inv != 0;
    return ll;
  }
  void getLogLikeBatch(unsigned nprop, const float* p, unsigned npar,
                       double* logl, int* status) {
    check(pofd_like1_eval_batch(h_, nprop, p, npar, logl, status),
          "calcLike::getLogLikeBatch");
  }
  // priors (calcLike.h:251-269)
  void setSigmaPrior(double width) {
    check(pofd_like1_set_sigma_prior(h_, 1, width), "calcLike::setSigmaPrior");
  }
  void unsetSigmaPrior() {
    check(pofd_like1_set_sigma_prior(h_, 0, 0.0), "calcLike::unsetSigmaPrior");
  }
  void setCFIRBPrior(double mean, double sigma) {
    check(pofd_like1_set_cfirb_prior(h_, 1, mean, sigma), "calcLike::setCFIRBPrior");
  }
  void unsetCFIRBPrior() {
    check(pofd_like1_set_cfirb_prior(h_, 0, 0.0, 0.0), "calcLike::unsetCFIRBPrior");
  }
  void setPoissonPrior(double mean, double sigma) {
    check(pofd_like1_set_poisson_prior(h_, 1, mean, sigma), "calcLike::setPoissonPrior");
  }
  void unsetPoissonPrior() {
    check(pofd_like1_set_poisson_prior(h_, 0, 0.0, 0.0), "calcLike::unsetPoissonPrior");
  }
  void setRegularizationAlpha(double alpha) {
    check(pofd_like1_set_regularization(h_, alpha), "calcLike::setRegularizationAlpha");
  }
  // calcLike::fillBonusParams (calcLike.cc:958-980) on host rows of npar >=
  // nknots + 3 entries: <S>, <S^2> written after the sigma multiplier
  void fillBonusParams(unsigned nknots, float* p, unsigned npar) {
    if (npar < nknots + 3) throw std::runtime_error("calcLike::fillBonusParams: Not enough room to fill");
    double b[2];
    check(pofd_like1_bonus(h_, 1, p, npar, b), "calcLike::fillBonusParams");
    p[nknots + 1] = static_cast<float>(b[0]);
    p[nknots + 2] = static_cast<float>(b[1]);
  }
  // launch-shape autotuner on nprop representative rows (no counterpart)
  void autotune(unsigned nprop, const float* p, unsigned npar, int reps = 20) {
    check(pofd_like1_autotune(h_, nprop, p, npar, reps, nullptr), "calcLike::autotune");
  }
  pofd_like1* get() const { return h_; }

 private:
  pofd_like1* h_ = nullptr;
};

// doublebeam::doublebeam(file1, file2, histogram, NBINS, MINVAL)
// (doublebeam.h:81) from two pixel arrays of npix values each.
class Beam2 {
 public:
  Beam2(const double* pix1, const double* pix2, size_t npix, double pixsize,
        bool histogram = false, unsigned nbins = 150, double minval = 1e-6) {
    check(pofd_beam2_create(pix1, pix2, npix, pixsize, minval,
                            histogram ? nbins : 0u, &h_),
          "doublebeam::doublebeam");
  }
  ~Beam2() { pofd_beam2_destroy(h_); }
  Beam2(const Beam2&) = delete;
  Beam2& operator=(const Beam2&) = delete;
  const pofd_beam2* get() const { return h_; }

 private:
  pofd_beam2* h_ = nullptr;
};

// calcLikeDouble (calcLikeDouble.h:192-347) with the log-normal colour model.
class Like2 {
 public:
  Like2(Context& ctx, unsigned nknots, const double* knotpos, unsigned nsigma,
        const double* sigmapos, unsigned noffset, const double* offsetpos,
        unsigned fftsize = 4096, unsigned nedge = 256, bool edge_integ = true,
        bool bin_data = true, unsigned nbins = 1000) {
    check(pofd_like2_create(ctx.get(), nknots, knotpos, nsigma, sigmapos, noffset,
                            offsetpos, fftsize, nedge, edge_integ ? 1 : 0,
                            bin_data ? 1 : 0, nbins, &h_),
          "calcLikeDouble::calcLikeDouble");
  }
  ~Like2() { pofd_like2_destroy(h_); }
  Like2(const Like2&) = delete;
  Like2& operator=(const Like2&) = delete;
  int addBeamSet(const Beam2& bm, double exp_conf1 = 0.0, double exp_conf2 = 0.0) {
    return check(pofd_like2_add_beamset(h_, bm.get(), exp_conf1, exp_conf2),
                 "calcLikeDouble::readDataFromFiles");
  }
  void addDataset(int beamset, const double* data1, const double* data2, size_t ndata,
                  double sigma_base1, double sigma_base2, double like_norm = 1.0,
                  bool meansub = true) {
    check(pofd_like2_add_dataset(h_, beamset, data1, data2, ndata, meansub ? 1 : 0,
                                 sigma_base1, sigma_base2, like_norm),
          "calcLikeDouble::readDataFromFiles");
  }
  // calcLikeDouble::readDataFromFiles (calcLikeDouble.cc:932-1030): groups
  // keyed by "beamfile1:beamfile2" in key order, datasets in input order
  void readDataFromFiles(const std::vector<std::string>& datafiles1,
                         const std::vector<std::string>& datafiles2,
                         const std::vector<std::string>& beamfiles1,
                         const std::vector<std::string>& beamfiles2,
                         const std::vector<double>& sigmas1, const std::vector<double>& sigmas2,
                         const std::vector<double>& like_norms, bool IGNOREMASK = false,
                         bool MEANSUB = false, double MINBEAMVAL = 1e-6, bool HISTOGRAM = false,
                         unsigned int NBEAMHIST = 150, double EXPCONF1 = 0.0,
                         double EXPCONF2 = 0.0) {
    const size_t n = datafiles1.size();
    if (n != datafiles2.size())
      throw std::runtime_error("calcLikeDouble::readDataFromFiles: Datafiles1 and datafile2 not same length");
    if (n == 0) throw std::runtime_error("calcLikeDouble::readDataFromFiles: No datafiles");
    if (n != beamfiles1.size() || n != beamfiles2.size() || n != sigmas1.size() ||
        n != sigmas2.size() || n != like_norms.size())
      throw std::runtime_error("calcLikeDouble::readDataFromFiles: inputs not same length");
    std::map<std::string, std::vector<size_t>> groups;
    for (size_t i = 0; i < n; ++i) groups[beamfiles1[i] + ":" + beamfiles2[i]].push_back(i);
    for (const auto& g : groups) {
      const size_t i0 = g.second.front();
      double ps1 = 0.0, ps2 = 0.0;
      const std::vector<double> p1 = readFitsBeam(beamfiles1[i0], ps1);
      const std::vector<double> p2 = readFitsBeam(beamfiles2[i0], ps2);
      if (std::abs((ps1 - ps2) / ps1) > 1e-5)  // doublebeam.cc:263-270
        throw std::runtime_error("doublebeam::readFiles: Pixel scale in " + beamfiles2[i0] +
                                 " doesn't match that of " + beamfiles1[i0]);
      if (p1.size() != p2.size())
        throw std::runtime_error("doublebeam::readFiles: beam sizes differ");
      Beam2 bm(p1.data(), p2.data(), p1.size(), ps1, HISTOGRAM, NBEAMHIST, MINBEAMVAL);
      const int bs = addBeamSet(bm, EXPCONF1, EXPCONF2);
      for (size_t i : g.second) {
        std::vector<double> d1, d2;
        readFitsData2(datafiles1[i], datafiles2[i], IGNOREMASK, false, d1, d2);
        addDataset(bs, d1.data(), d2.data(), d1.size(), sigmas1[i], sigmas2[i], like_norms[i],
                   MEANSUB);
      }
    }
  }
  void setRRanges(const float* p, unsigned npar) {
    check(pofd_like2_set_rranges(h_, p, npar), "calcLikeDouble::setRRanges");
  }
  void reserve(unsigned max_batch) {
    check(pofd_like2_reserve(h_, max_batch), "calcLikeDouble::reserve");
  }
  double getLogLike(const float* p, unsigned npar, bool& pars_invalid) {
    double ll = 0.0;
    int inv = 0;
    check(pofd_like2_loglike(h_, p, npar, &ll, &inv), "calcLikeDouble::getLogLike");
    pars_invalid = inv != 0;
    return ll;
  }
  void getLogLikeBatch(unsigned nprop, const float* p, unsigned npar, double* logl,
                       int* status) {
    check(pofd_like2_eval_batch(h_, nprop, p, npar, logl, status),
          "calcLikeDouble::getLogLikeBatch");
  }
  // priors per band 0/1 (calcLikeDouble.h:310-341)
  void setSigmaPrior(int band, double width) {
    check(pofd_like2_set_sigma_prior(h_, band, 1, width), "calcLikeDouble::setSigmaPrior");
  }
  void unsetSigmaPrior(int band) {
    check(pofd_like2_set_sigma_prior(h_, band, 0, 0.0), "calcLikeDouble::unsetSigmaPrior");
  }
  void setCFIRBPrior(int band, double mean, double sigma) {
    check(pofd_like2_set_cfirb_prior(h_, band, 1, mean, sigma), "calcLikeDouble::setCFIRBPrior");
  }
  void unsetCFIRBPrior(int band) {
    check(pofd_like2_set_cfirb_prior(h_, band, 0, 0.0, 0.0), "calcLikeDouble::unsetCFIRBPrior");
  }
  void setPoissonPrior(int band, double mean, double sigma) {
    check(pofd_like2_set_poisson_prior(h_, band, 1, mean, sigma),
          "calcLikeDouble::setPoissonPrior");
  }
  void unsetPoissonPrior(int band) {
    check(pofd_like2_set_poisson_prior(h_, band, 0, 0.0, 0.0),
          "calcLikeDouble::unsetPoissonPrior");
  }
  void setRegularizationAlpha(double alpha) {
    check(pofd_like2_set_regularization(h_, alpha), "calcLikeDouble::setRegularizationAlpha");
  }
  // calcLikeDouble::fillBonusParams (calcLikeDouble.cc:1283-1310) on a host
  // row: <S1>, <S2>, <S1^2>, <S2^2> after the two sigma multipliers
  // (nmodel = knots + sigma knots + offset knots; npar >= nmodel + 6)
  void fillBonusParams(unsigned nmodel, float* p, unsigned npar) {
    if (npar < nmodel + 6)
      throw std::runtime_error("calcLikeDouble::fillBonusParams: Not enough room to fill");
    double b[4];
    check(pofd_like2_bonus(h_, 1, p, npar, b), "calcLikeDouble::fillBonusParams");
    for (int i = 0; i < 4; ++i) p[nmodel + 2 + i] = static_cast<float>(b[i]);
  }
  // 1: row cuFFT + fused column kernel (default where the size allows),
  // 0: 2D cuFFT (no counterpart: the reference's FFTW plans are internal)
  void setFFT(int mode) { check(pofd_like2_set_fft(h_, mode), "calcLikeDouble::setFFT"); }
  pofd_like2* get() const { return h_; }

 private:
  pofd_like2* h_ = nullptr;
};

}  // namespace pofd_b200
#endif
