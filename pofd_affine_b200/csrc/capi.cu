// capi.cu -- extern "C" entry points of libpofd_b200.so (include/pofd_b200.h).
//
// Each entry point converts C++ exceptions into the status codes of the
// header, so callers see the reference's error behaviour (an affineExcept
// at the same point) as a negative return plus pofd_last_error().
#include <cuda_runtime.h>

#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pofd_b200.h"
#include "engine1d.cuh"
#include "engine2d.cuh"
#include "ensemble.cuh"
#include "fits.hh"
#include "surrogate.cuh"
#include "setup.hh"

namespace {
thread_local std::string g_err;

template <class F>
int guard(F&& f) {
  try {
    return f();
  } catch (const pofd::Error& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return POFD_E_NOMEM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return POFD_E_ARG;
  }
}

void need(bool ok, const char* msg) {
  if (!ok) throw pofd::Error(POFD_E_ARG, msg);
}
}  // namespace

struct pofd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
};

struct pofd_beam1 {
  pofd::Beam1 b;
};

struct pofd_like1 {
  pofd_ctx* ctx = nullptr;
  std::unique_ptr<pofd::Engine1> eng;
};

struct pofd_beam2 {
  pofd::Beam2 b;
};

struct pofd_pdfactory2 {
  pofd_ctx* ctx = nullptr;
  unsigned nedge = 256;
  std::unique_ptr<pofd::Engine2> eng;
  std::vector<float> theta;
  bool inited = false;
};

struct pofd_like2 {
  pofd_ctx* ctx = nullptr;
  std::unique_ptr<pofd::Engine2> eng;
};

struct pofd_surrogate {
  pofd_ctx* ctx = nullptr;
  std::unique_ptr<pofd::Surrogate> s;
};

struct pofd_likesum {
  pofd_ctx* ctx = nullptr;
  std::unique_ptr<pofd::LikeSum> ls;
};

struct pofd_ensemble {
  pofd_ctx* ctx = nullptr;
  std::unique_ptr<pofd::Ensemble> ens;
};

struct pofd_pdfactory1 {
  pofd_ctx* ctx = nullptr;
  unsigned ninterp = 2048;
  std::unique_ptr<pofd::Engine1> eng;
  std::vector<float> theta;  // knot values + noise slot
  bool inited = false;
};

namespace pofd {
// Lets entry points outside this file (the allocation-free one) report a
// message through pofd_last_error().
void set_last_error(const char* msg) { g_err = msg; }
int ctx_device(const pofd_ctx* ctx) { return ctx->device; }
cudaStream_t ctx_stream(const pofd_ctx* ctx) { return ctx->stream; }
}  // namespace pofd

extern "C" {

const char* pofd_last_error(void) { return g_err.c_str(); }

const char* pofd_version(void) { return "pofd_b200 0.1.0 (reference pofd_affine 0.5.1)"; }

// ------------------------------------------------------------- context
int pofd_ctx_create(int device, pofd_ctx** out) {
  return guard([&] {
    need(out != nullptr, "null output pointer");
    if (device == -1) {
      // host-only context: set-up calls (beams, data, R ranges) work,
      // anything that needs a GPU returns POFD_E_CUDA
      std::unique_ptr<pofd_ctx> c(new pofd_ctx());
      c->device = -1;
      *out = c.release();
      return POFD_OK;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
      throw pofd::Error(POFD_E_CUDA, "no CUDA device available");
    need(device >= 0 && device < ndev, "invalid device index");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) throw pofd::Error(POFD_E_CUDA, cudaGetErrorString(e));
    std::unique_ptr<pofd_ctx> c(new pofd_ctx());
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) throw pofd::Error(POFD_E_CUDA, cudaGetErrorString(e));
    *out = c.release();
    return POFD_OK;
  });
}

int pofd_ctx_destroy(pofd_ctx* ctx) {
  if (!ctx) return POFD_OK;
  if (ctx->device < 0) {
    delete ctx;
    return POFD_OK;
  }
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return POFD_OK;
}

int pofd_ctx_stream(pofd_ctx* ctx, void** s) {
  return guard([&] {
    need(ctx && s, "null argument");
    *s = ctx->stream;
    return POFD_OK;
  });
}

int pofd_ctx_synchronize(pofd_ctx* ctx) {
  return guard([&] {
    need(ctx != nullptr, "null context");
    cudaSetDevice(ctx->device);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) throw pofd::Error(POFD_E_CUDA, cudaGetErrorString(e));
    return POFD_OK;
  });
}

// ------------------------------------------------------------- 1D beam
int pofd_fits_read_data(const char* path, int ignore_mask, int meansub, double* out,
                        size_t cap, size_t* n) {
  return guard([&] {
    need(path && n, "null argument");
    const std::vector<double> d = pofd::fits_read_data(path, ignore_mask != 0, meansub != 0);
    *n = d.size();
    if (out) {
      need(cap >= d.size(), "output buffer too small");
      std::memcpy(out, d.data(), d.size() * sizeof(double));
    }
    return POFD_OK;
  });
}

int pofd_fits_read_data2(const char* path1, const char* path2, int ignore_mask, int meansub,
                         double* out1, double* out2, size_t cap, size_t* n) {
  return guard([&] {
    need(path1 && path2 && n, "null argument");
    std::vector<double> a, b;
    pofd::fits_read_data2(path1, path2, ignore_mask != 0, meansub != 0, &a, &b);
    *n = a.size();
    if (out1 || out2) {
      need(out1 && out2, "null argument");
      need(cap >= a.size(), "output buffer too small");
      std::memcpy(out1, a.data(), a.size() * sizeof(double));
      std::memcpy(out2, b.data(), b.size() * sizeof(double));
    }
    return POFD_OK;
  });
}

int pofd_fits_read_beam(const char* path, double* out, size_t cap, size_t* nx, size_t* ny,
                        double* pixsize) {
  return guard([&] {
    need(path && nx && ny && pixsize, "null argument");
    const pofd::FitsBeam b = pofd::fits_read_beam(path);
    *nx = static_cast<size_t>(b.nx);
    *ny = static_cast<size_t>(b.ny);
    *pixsize = b.pixsize;
    if (out) {
      need(cap >= b.pix.size(), "output buffer too small");
      std::memcpy(out, b.pix.data(), b.pix.size() * sizeof(double));
    }
    return POFD_OK;
  });
}

int pofd_beam1_create(const double* pix, size_t npix, double pixsize,
                      double minval, unsigned nhist, pofd_beam1** out) {
  return guard([&] {
    need(pix && out, "null argument");
    std::unique_ptr<pofd_beam1> b(new pofd_beam1());
    b->b.build(pix, npix, pixsize, minval);
    if (nhist > 0) b->b.histogram(nhist);
    *out = b.release();
    return POFD_OK;
  });
}

int pofd_beam1_destroy(pofd_beam1* b) {
  delete b;
  return POFD_OK;
}

int pofd_beam1_info(const pofd_beam1* bp, double* o) {
  return guard([&] {
    need(bp && o, "null argument");
    const pofd::Beam1& b = bp->b;
    o[0] = b.haspos; o[1] = b.hasneg;
    o[2] = static_cast<double>(b.pos.size()); o[3] = static_cast<double>(b.neg.size());
    o[4] = b.poshist; o[5] = b.neghist;
    o[6] = static_cast<double>(b.poswt.size()); o[7] = static_cast<double>(b.negwt.size());
    o[8] = b.haspos ? b.pos.front() : pofd::nan(); o[9] = b.maxpos();
    o[10] = b.hasneg ? b.neg.front() : pofd::nan(); o[11] = b.maxneg();
    o[12] = b.pixsize; o[13] = b.totpos; o[14] = b.totneg;
    return POFD_OK;
  });
}

int pofd_beam1_terms(const pofd_beam1* bp, int negside, size_t* nterms,
                     double* weights, double* inv_beam) {
  return guard([&] {
    need(bp && nterms, "null argument");
    std::vector<double> w, ie;
    bp->b.terms(negside != 0, w, ie);
    *nterms = ie.size();
    if (weights) std::memcpy(weights, w.data(), w.size() * sizeof(double));
    if (inv_beam) std::memcpy(inv_beam, ie.data(), ie.size() * sizeof(double));
    return POFD_OK;
  });
}

// ------------------------------------------------------- 1D P(D) factory
int pofd_pdfactory1_create(pofd_ctx* ctx, unsigned ninterp,
                           pofd_pdfactory1** out) {
  return guard([&] {
    need(ctx && out, "null argument");
    need(ninterp >= 4, "Invalid (0) ninterp");
    std::unique_ptr<pofd_pdfactory1> f(new pofd_pdfactory1());
    f->ctx = ctx;
    f->ninterp = ninterp;
    *out = f.release();
    return POFD_OK;
  });
}

int pofd_pdfactory1_destroy(pofd_pdfactory1* f) {
  if (f && f->ctx) cudaSetDevice(f->ctx->device);
  delete f;
  return POFD_OK;
}

// PDFactory::initPD argument checks (PDFactory.cc:1031-1054), then the
// engine is configured for one beam set with one noise-only dataset.
int pofd_pdfactory1_initpd(pofd_pdfactory1* f, unsigned n, double minflux,
                           double maxflux, unsigned nknots,
                           const double* knotpos, const float* knotvals,
                           const pofd_beam1* beam) {
  return guard([&] {
    need(f && knotpos && knotvals && beam, "null argument");
    if (n == 0) throw pofd::Error(POFD_E_ARG, "Invalid (zero) n");
    if (n == 1) throw pofd::Error(POFD_E_ARG, "Invalid (==0) n");
    if (maxflux <= 0.0) throw pofd::Error(POFD_E_ARG, "Invalid (non-positive) maxflux");
    if (minflux == maxflux) throw pofd::Error(POFD_E_ARG, "Invalid (0) range between min/max flux");
    for (unsigned k = 0; k < nknots; ++k)
      if (std::isnan(static_cast<double>(knotvals[k])))
        throw pofd::Error(POFD_E_INVALID_MODEL, "Invalid model");
    cudaSetDevice(f->ctx->device);
    f->eng.reset(new pofd::Engine1(f->ctx->device, f->ctx->stream));
    f->eng->configure(nknots, knotpos, n, f->ninterp, true, 1);
    const int bs = f->eng->add_beamset(beam->b, 0.0);
    f->eng->add_virtual_dataset(bs, 1.0);
    f->eng->set_rrange_explicit(bs, minflux, maxflux);
    f->eng->reserve(1);
    f->theta.assign(knotvals, knotvals + nknots);
    f->theta.push_back(1.0f);  // sigma multiplier; the noise level is the dataset's
    f->inited = true;
    return POFD_OK;
  });
}

int pofd_pdfactory1_getpd(pofd_pdfactory1* f, double sigma, int setlog,
                          double* pd_out, double* minflux_out,
                          double* dflux_out) {
  return guard([&] {
    need(f && pd_out, "null argument");
    if (!f->inited) throw pofd::Error(POFD_E_ARG, "Must call initPD first");
    cudaSetDevice(f->ctx->device);
    double info[12];
    f->eng->set_virtual_sigma(0, sigma);
    const int st = f->eng->pd_host(0, 0, f->theta.data(),
                                   static_cast<unsigned>(f->theta.size()),
                                   setlog != 0, pd_out, info);
    if (minflux_out) *minflux_out = info[10];
    if (dflux_out) *dflux_out = info[0];
    if (st != 0) throw pofd::Error(st, "P(D) unwrap failed (split point or mean)");
    return POFD_OK;
  });
}

int pofd_pdfactory1_get_r(pofd_pdfactory1* f, double* rvals_out) {
  return guard([&] {
    need(f && rvals_out, "null argument");
    if (!f->inited) throw pofd::Error(POFD_E_ARG, "Must call initPD first");
    cudaSetDevice(f->ctx->device);
    f->eng->rgrid_host(0, f->theta.data(), static_cast<unsigned>(f->theta.size()), rvals_out);
    return POFD_OK;
  });
}

// ---------------------------------------------------------- 1D likelihood
int pofd_like1_create(pofd_ctx* ctx, unsigned nknots, const double* knotpos,
                      unsigned fftsize, unsigned ninterp, int bin_data,
                      unsigned nbins, pofd_like1** out) {
  return guard([&] {
    need(ctx && knotpos && out, "null argument");
    cudaSetDevice(ctx->device);
    std::unique_ptr<pofd_like1> L(new pofd_like1());
    L->ctx = ctx;
    L->eng.reset(new pofd::Engine1(ctx->device, ctx->stream));
    L->eng->configure(nknots, knotpos, fftsize, ninterp, bin_data != 0, nbins);
    *out = L.release();
    return POFD_OK;
  });
}

int pofd_like1_destroy(pofd_like1* L) {
  if (L && L->ctx) cudaSetDevice(L->ctx->device);
  delete L;
  return POFD_OK;
}

int pofd_like1_add_beamset(pofd_like1* L, const pofd_beam1* beam,
                           double exp_conf) {
  return guard([&] {
    need(L && beam, "null argument");
    return L->eng->add_beamset(beam->b, exp_conf);
  });
}

int pofd_like1_add_dataset(pofd_like1* L, int beamset, const double* data,
                           size_t ndata, int meansub, double sigma_base,
                           double like_norm) {
  return guard([&] {
    need(L && data, "null argument");
    L->eng->add_dataset(beamset, data, ndata, meansub != 0, sigma_base, like_norm);
    return POFD_OK;
  });
}

int pofd_like1_add_dataset_device(pofd_like1* L, int beamset, double* data_dev, size_t ndata,
                                  int meansub, double sigma_base, double like_norm) {
  return guard([&] {
    need(L && data_dev, "null argument");
    L->eng->add_dataset_device(beamset, data_dev, ndata, meansub != 0, sigma_base, like_norm);
    return POFD_OK;
  });
}

int pofd_data_bin_device(double* data_dev, size_t ndata, int meansub, unsigned nbins,
                         unsigned* bins_dev, double* info3, void* stream) {
  return guard([&] {
    need(data_dev && bins_dev && info3, "null argument");
    pofd::ingest_bin1(data_dev, ndata, meansub != 0, nbins, bins_dev, info3, stream);
    return POFD_OK;
  });
}

int pofd_data2_bin_device(double* d1_dev, double* d2_dev, size_t ndata, int meansub,
                          unsigned nbins1, unsigned nbins2, unsigned* bins_dev, double* info6,
                          void* stream) {
  return guard([&] {
    need(d1_dev && d2_dev && bins_dev && info6, "null argument");
    pofd::ingest_bin2(d1_dev, d2_dev, ndata, meansub != 0, nbins1, nbins2, bins_dev, info6,
                      stream);
    return POFD_OK;
  });
}

int pofd_like1_set_rranges(pofd_like1* L, const float* theta, unsigned npar) {
  return guard([&] {
    need(L && theta, "null argument");
    L->eng->set_rranges(theta, npar);
    return POFD_OK;
  });
}

int pofd_like1_get_rrange(const pofd_like1* L, int beamset, double* r) {
  return guard([&] {
    need(L && r, "null argument");
    const auto rr = L->eng->rrange(beamset);
    r[0] = rr.first;
    r[1] = rr.second;
    return POFD_OK;
  });
}

int pofd_like1_dataset_info(const pofd_like1* L, int beamset, int dataset,
                            double* info9, uint32_t* bins) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->dataset_info(beamset, dataset, info9, bins);
    return POFD_OK;
  });
}

int pofd_like1_reserve(pofd_like1* L, unsigned max_batch) {
  return guard([&] {
    need(L != nullptr, "null argument");
    cudaSetDevice(L->ctx->device);
    L->eng->reserve(max_batch);
    return POFD_OK;
  });
}

int pofd_like1_loglike(pofd_like1* L, const float* theta, unsigned npar,
                       double* logl, int* pars_invalid) {
  return guard([&] {
    need(L && theta && logl, "null argument");
    cudaSetDevice(L->ctx->device);
    int st = 0;
    L->eng->eval_host(1, theta, npar, logl, &st);
    if (pars_invalid) *pars_invalid = (st == POFD_REJECTED) ? 1 : 0;
    if (st < 0) throw pofd::Error(st, "likelihood evaluation failed");
    return st;
  });
}

int pofd_like1_eval_batch(pofd_like1* L, unsigned nprop, const float* theta,
                          unsigned npar, double* logl, int* status) {
  return guard([&] {
    need(L && theta && logl && status, "null argument");
    cudaSetDevice(L->ctx->device);
    L->eng->eval_host(nprop, theta, npar, logl, status);
    return POFD_OK;
  });
}

int pofd_like1_eval_batch_device(pofd_like1* L, unsigned nprop,
                                 const float* theta_dev, unsigned npar,
                                 double* logl_dev, int* status_dev,
                                 void* stream) {
  return guard([&] {
    need(L && theta_dev && logl_dev && status_dev, "null argument");
    cudaSetDevice(L->ctx->device);
    L->eng->enqueue(nprop, theta_dev, npar, logl_dev, status_dev,
                    static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

int pofd_like1_pd(pofd_like1* L, int beamset, int dataset, const float* theta,
                  unsigned npar, int setlog, double* pd_out, double* info12) {
  return guard([&] {
    need(L && theta && pd_out, "null argument");
    cudaSetDevice(L->ctx->device);
    const int st = L->eng->pd_host(beamset, dataset, theta, npar, setlog != 0,
                                   pd_out, info12);
    if (st != 0) throw pofd::Error(st, "P(D) unwrap failed (split point or mean)");
    return POFD_OK;
  });
}

int pofd_like1_rnodes(pofd_like1* L, int beamset, int negative_side,
                      const float* theta, unsigned npar, double* x_out,
                      double* r_out) {
  return guard([&] {
    need(L && theta && x_out && r_out, "null argument");
    cudaSetDevice(L->ctx->device);
    L->eng->rnodes_host(beamset, negative_side ? 1 : 0, theta, npar, x_out, r_out);
    return POFD_OK;
  });
}

int pofd_like1_kernels_per_eval(const pofd_like1* L, int* nk) {
  return guard([&] {
    need(L && nk, "null argument");
    *nk = L->eng->kernels_per_eval();
    return POFD_OK;
  });
}

int pofd_like1_profile(pofd_like1* L, unsigned nprop, const float* theta,
                       unsigned npar, int reps, double* stage_ms,
                       int* nstages) {
  return guard([&] {
    need(L && theta && stage_ms && nstages, "null argument");
    need(reps > 0, "reps must be > 0");
    cudaSetDevice(L->ctx->device);
    L->eng->profile_stages(nprop, theta, npar, reps, stage_ms);
    *nstages = pofd::Engine1::kNumStages;
    return POFD_OK;
  });
}

const char* pofd_like1_stage_name(const pofd_like1* L, int i) {
  return (L && L->eng) ? L->eng->stage_name(i) : "";
}

int pofd_like1_set_fft(pofd_like1* L, int mode) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_fft_mode(mode);
    return POFD_OK;
  });
}

int pofd_like1_fft_info(pofd_like1* L, int* own) {
  return guard([&] {
    need(L && own, "null argument");
    if (L->ctx->device >= 0) L->eng->reserve(1);
    *own = L->eng->own_fft() ? 1 : 0;
    return POFD_OK;
  });
}

int pofd_like1_autotune(pofd_like1* L, unsigned nprop, const float* theta, unsigned npar,
                        int reps, double* out7) {
  return guard([&] {
    need(L && theta, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->autotune(nprop, theta, npar, reps, out7);
    return POFD_OK;
  });
}

int pofd_like1_get_tuning(const pofd_like1* L, int* knobs5) {
  return guard([&] {
    need(L && knobs5, "null argument");
    const pofd::Tune1& t = L->eng->tuning();
    knobs5[0] = t.own_fft;
    knobs5[1] = t.rfill_per;
    knobs5[2] = t.rnodes_threads;
    knobs5[3] = t.spec_blocks;
    knobs5[4] = t.rfill_mode;
    return POFD_OK;
  });
}

int pofd_like1_set_tuning(pofd_like1* L, const int* knobs5) {
  return guard([&] {
    need(L && knobs5, "null argument");
    pofd::Tune1 t;
    t.own_fft = knobs5[0];
    t.rfill_per = knobs5[1];
    t.rnodes_threads = knobs5[2];
    t.spec_blocks = knobs5[3];
    t.rfill_mode = knobs5[4];
    L->eng->set_tuning(t);
    return POFD_OK;
  });
}

int pofd_like1_set_sigma_prior(pofd_like1* L, int on, double width) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_sigma_prior(on != 0, width);
    return POFD_OK;
  });
}

int pofd_like1_set_cfirb_prior(pofd_like1* L, int on, double mean, double sigma) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_cfirb_prior(on != 0, mean, sigma);
    return POFD_OK;
  });
}

int pofd_like1_set_poisson_prior(pofd_like1* L, int on, double mean, double sigma) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_poisson_prior(on != 0, mean, sigma);
    return POFD_OK;
  });
}

int pofd_like1_set_regularization(pofd_like1* L, double alpha) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_regularization(alpha);
    return POFD_OK;
  });
}

int pofd_like1_bonus(pofd_like1* L, unsigned nprop, const float* theta, unsigned npar,
                     double* out) {
  return guard([&] {
    need(L && theta && out, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->bonus_host(nprop, theta, npar, out);
    return POFD_OK;
  });
}

int pofd_like1_fill_bonus_device(pofd_like1* L, unsigned nprop, float* theta_dev,
                                 unsigned npar, void* stream) {
  return guard([&] {
    need(L && theta_dev, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->fill_bonus(nprop, theta_dev, npar, static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

// ------------------------------------------------------------- 2D beam
int pofd_beam2_create(const double* pix1, const double* pix2, size_t npix,
                      double pixsize, double minval, unsigned nhist,
                      pofd_beam2** out) {
  return guard([&] {
    need(pix1 && pix2 && out, "null argument");
    std::unique_ptr<pofd_beam2> b(new pofd_beam2());
    b->b.build(pix1, pix2, npix, pixsize, minval);
    if (nhist > 0) b->b.histogram(nhist);
    *out = b.release();
    return POFD_OK;
  });
}

int pofd_beam2_destroy(pofd_beam2* b) {
  delete b;
  return POFD_OK;
}

int pofd_beam2_info(const pofd_beam2* bp, double* o) {
  return guard([&] {
    need(bp && o, "null argument");
    const pofd::Beam2& b = bp->b;
    for (int s = 0; s < 4; ++s) {
      o[s] = b.hassign[s];
      o[4 + s] = static_cast<double>(b.pix1[s].size());
      o[8 + s] = b.ishist[s];
      o[12 + s] = static_cast<double>(b.binwt[s].size());
    }
    o[16] = b.pixsize;
    return POFD_OK;
  });
}

// ---------------------------------------------------------- 2D likelihood
int pofd_like2_create(pofd_ctx* ctx, unsigned nknots, const double* knotpos,
                      unsigned nsigma, const double* sigmapos,
                      unsigned noffset, const double* offsetpos,
                      unsigned fftsize, unsigned nedge, int edge_integ,
                      int bin_data, unsigned nbins, pofd_like2** out) {
  return guard([&] {
    need(ctx && knotpos && sigmapos && offsetpos && out, "null argument");
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    std::unique_ptr<pofd_like2> L(new pofd_like2());
    L->ctx = ctx;
    L->eng.reset(new pofd::Engine2(ctx->device, ctx->stream));
    L->eng->configure(nknots, knotpos, nsigma, sigmapos, noffset, offsetpos,
                      fftsize, nedge, edge_integ != 0, bin_data != 0, nbins);
    *out = L.release();
    return POFD_OK;
  });
}

int pofd_like2_destroy(pofd_like2* L) {
  if (L && L->ctx && L->ctx->device >= 0) cudaSetDevice(L->ctx->device);
  delete L;
  return POFD_OK;
}

int pofd_like2_add_beamset(pofd_like2* L, const pofd_beam2* beam,
                           double ec1, double ec2) {
  return guard([&] {
    need(L && beam, "null argument");
    return L->eng->add_beamset(beam->b, ec1, ec2);
  });
}

int pofd_like2_add_dataset(pofd_like2* L, int beamset, const double* d1,
                           const double* d2, size_t nd, int meansub,
                           double sb1, double sb2, double like_norm) {
  return guard([&] {
    need(L && d1 && d2, "null argument");
    L->eng->add_dataset(beamset, d1, d2, nd, meansub != 0, sb1, sb2, like_norm);
    return POFD_OK;
  });
}

int pofd_like2_add_dataset_device(pofd_like2* L, int beamset, double* d1_dev, double* d2_dev,
                                  size_t nd, int meansub, double sb1, double sb2,
                                  double like_norm) {
  return guard([&] {
    need(L && d1_dev && d2_dev, "null argument");
    L->eng->add_dataset_device(beamset, d1_dev, d2_dev, nd, meansub != 0, sb1, sb2, like_norm);
    return POFD_OK;
  });
}

int pofd_like2_set_rranges(pofd_like2* L, const float* theta, unsigned npar) {
  return guard([&] {
    need(L && theta, "null argument");
    L->eng->set_rranges(theta, npar);
    return POFD_OK;
  });
}

int pofd_like2_get_rrange(const pofd_like2* L, int beamset, double* r4) {
  return guard([&] {
    need(L && r4, "null argument");
    L->eng->rrange(beamset, r4);
    return POFD_OK;
  });
}

int pofd_like2_dataset_info(const pofd_like2* L, int beamset, int dataset,
                            double* info10, uint32_t* bins) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->dataset_info(beamset, dataset, info10, bins);
    return POFD_OK;
  });
}

int pofd_like2_reserve(pofd_like2* L, unsigned max_batch) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->reserve(max_batch);
    return POFD_OK;
  });
}

int pofd_like2_loglike(pofd_like2* L, const float* theta, unsigned npar,
                       double* logl, int* pars_invalid) {
  return guard([&] {
    need(L && theta && logl, "null argument");
    int st = 0;
    L->eng->eval_host(1, theta, npar, logl, &st);
    if (pars_invalid) *pars_invalid = (st == POFD_REJECTED) ? 1 : 0;
    if (st < 0) throw pofd::Error(st, "likelihood evaluation failed");
    return st;
  });
}

int pofd_like2_eval_batch(pofd_like2* L, unsigned nprop, const float* theta,
                          unsigned npar, double* logl, int* status) {
  return guard([&] {
    need(L && theta && logl && status, "null argument");
    L->eng->eval_host(nprop, theta, npar, logl, status);
    return POFD_OK;
  });
}

int pofd_like2_eval_batch_device(pofd_like2* L, unsigned nprop,
                                 const float* theta_dev, unsigned npar,
                                 double* logl_dev, int* status_dev,
                                 void* stream) {
  return guard([&] {
    need(L && theta_dev && logl_dev && status_dev, "null argument");
    L->eng->enqueue(nprop, theta_dev, npar, logl_dev, status_dev,
                    static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

int pofd_like2_pd(pofd_like2* L, int beamset, int dataset, const float* theta,
                  unsigned npar, int setlog, double* pd_out, double* info16) {
  return guard([&] {
    need(L && theta && pd_out, "null argument");
    const int st = L->eng->pd_host(beamset, dataset, theta, npar, setlog != 0,
                                   pd_out, info16);
    if (st != 0) throw pofd::Error(st, "P(D) unwrap failed (split point or mean)");
    return POFD_OK;
  });
}

int pofd_like1_get_r(pofd_like1* L, int beamset, const float* theta, unsigned npar,
                     double* out) {
  return guard([&] {
    need(L && theta && out, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->rgrid_host(beamset, theta, npar, out);
    return POFD_OK;
  });
}

int pofd_like2_get_r(pofd_like2* L, int beamset, const float* theta,
                     unsigned npar, double* out) {
  return guard([&] {
    need(L && theta && out, "null argument");
    L->eng->rgrid_host(beamset, theta, npar, out);
    return POFD_OK;
  });
}

int pofd_like2_autotune(pofd_like2* L, unsigned nprop, const float* theta, unsigned npar,
                        int reps, double* out5) {
  return guard([&] {
    need(L && theta, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->autotune(nprop, theta, npar, reps, out5);
    return POFD_OK;
  });
}

int pofd_like2_get_tuning(const pofd_like2* L, int* knobs3) {
  return guard([&] {
    need(L && knobs3, "null argument");
    const pofd::Tune2 t = L->eng->tuning();
    knobs3[0] = t.fft_mode;
    knobs3[1] = t.rgrid_rows;
    knobs3[2] = t.edge_rows;
    return POFD_OK;
  });
}

int pofd_like2_set_tuning(pofd_like2* L, const int* knobs3) {
  return guard([&] {
    need(L && knobs3, "null argument");
    pofd::Tune2 t;
    t.fft_mode = knobs3[0];
    t.rgrid_rows = knobs3[1];
    t.edge_rows = knobs3[2];
    if (L->ctx->device >= 0) cudaSetDevice(L->ctx->device);
    L->eng->set_tuning(t);
    return POFD_OK;
  });
}

int pofd_like2_active_terms(pofd_like2* L, const float* theta, unsigned npar,
                            long long* out2) {
  return guard([&] {
    need(L && theta && out2, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->active_terms(theta, npar, out2);
    return POFD_OK;
  });
}

int pofd_like2_kernels_per_eval(const pofd_like2* L, int* nk) {
  return guard([&] {
    need(L && nk, "null argument");
    *nk = L->eng->kernels_per_eval();
    return POFD_OK;
  });
}

int pofd_like2_set_sigma_prior(pofd_like2* L, int band, int on, double width) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_sigma_prior(band, on != 0, width);
    return POFD_OK;
  });
}

int pofd_like2_set_cfirb_prior(pofd_like2* L, int band, int on, double mean, double sigma) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_cfirb_prior(band, on != 0, mean, sigma);
    return POFD_OK;
  });
}

int pofd_like2_set_poisson_prior(pofd_like2* L, int band, int on, double mean, double sigma) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_poisson_prior(band, on != 0, mean, sigma);
    return POFD_OK;
  });
}

int pofd_like2_set_regularization(pofd_like2* L, double alpha) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_regularization(alpha);
    return POFD_OK;
  });
}

int pofd_like2_bonus(pofd_like2* L, unsigned nprop, const float* theta, unsigned npar,
                     double* out) {
  return guard([&] {
    need(L && theta && out, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->bonus_host(nprop, theta, npar, out);
    return POFD_OK;
  });
}

int pofd_like2_fill_bonus_device(pofd_like2* L, unsigned nprop, float* theta_dev,
                                 unsigned npar, void* stream) {
  return guard([&] {
    need(L && theta_dev, "null argument");
    need(L->ctx->device >= 0, "host-only context has no GPU");
    cudaSetDevice(L->ctx->device);
    L->eng->fill_bonus(nprop, theta_dev, npar, static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

int pofd_like2_profile(pofd_like2* L, unsigned nprop, const float* theta,
                       unsigned npar, int reps, double* stage_ms,
                       int* nstages) {
  return guard([&] {
    need(L && theta && stage_ms && nstages, "null argument");
    need(reps > 0, "reps must be > 0");
    L->eng->profile_stages(nprop, theta, npar, reps, stage_ms);
    *nstages = pofd::Engine2::kNumStages;
    return POFD_OK;
  });
}

const char* pofd_like2_stage_name(int i) { return pofd::Engine2::stage_name(i); }

const char* pofd_like2_stage_name_now(const pofd_like2* L, int i) {
  return (L && L->eng) ? L->eng->stage_name_now(i) : "";
}

int pofd_like2_set_fft(pofd_like2* L, int mode) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_fft_mode(mode);
    return POFD_OK;
  });
}

int pofd_like2_set_reference_sums(pofd_like2* L, int on) {
  return guard([&] {
    need(L != nullptr, "null argument");
    L->eng->set_reference_sums(on != 0);
    return POFD_OK;
  });
}

int pofd_like2_fft_info(const pofd_like2* L, int* fused) {
  return guard([&] {
    need(L && fused, "null argument");
    *fused = L->eng->colspec() ? 1 : 0;
    return POFD_OK;
  });
}

// ------------------------------------------------------------- ensemble
static int like1_batch(void* like, unsigned nprop, const float* theta,
                       unsigned npar, double* logl, int* status, void* stream) {
  return pofd_like1_eval_batch_device(static_cast<pofd_like1*>(like), nprop, theta, npar, logl,
                                      status, stream);
}
static int like1_fill(void* like, unsigned nprop, float* theta, unsigned npar, void* stream) {
  return pofd_like1_fill_bonus_device(static_cast<pofd_like1*>(like), nprop, theta, npar, stream);
}
static int like2_fill(void* like, unsigned nprop, float* theta, unsigned npar, void* stream) {
  return pofd_like2_fill_bonus_device(static_cast<pofd_like2*>(like), nprop, theta, npar, stream);
}
static int like2_batch(void* like, unsigned nprop, const float* theta,
                       unsigned npar, double* logl, int* status, void* stream) {
  return pofd_like2_eval_batch_device(static_cast<pofd_like2*>(like), nprop, theta, npar, logl,
                                      status, stream);
}

int pofd_ensemble_create(pofd_ctx* ctx, unsigned nwalkers, unsigned nparams,
                         double scalefac, unsigned long long seed,
                         pofd_ensemble** out) {
  return guard([&] {
    need(ctx && out, "null argument");
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    std::unique_ptr<pofd_ensemble> e(new pofd_ensemble());
    e->ctx = ctx;
    e->ens.reset(new pofd::Ensemble(ctx->device, ctx->stream, nwalkers, nparams, scalefac, seed));
    *out = e.release();
    return POFD_OK;
  });
}

int pofd_ensemble_destroy(pofd_ensemble* e) {
  if (e && e->ctx && e->ctx->device >= 0) cudaSetDevice(e->ctx->device);
  delete e;
  return POFD_OK;
}

int pofd_ensemble_set_likelihood(pofd_ensemble* e, pofd_batch_loglike_fn fn, void* like) {
  return guard([&] {
    need(e && fn, "null argument");
    e->ens->set_like(fn, like);
    return POFD_OK;
  });
}

int pofd_ensemble_use_like1(pofd_ensemble* e, pofd_like1* like) {
  return guard([&] {
    need(e && like, "null argument");
    e->ens->set_like(like1_batch, like);
    // bonus slots after the knots and the sigma multiplier are filled when
    // the parameter vector has room for them (pofdMCMC.cc:354-360)
    if (e->ens->npar() >= like->eng->nknots() + 3)
      e->ens->set_bonus(like1_fill, like);
    else
      e->ens->set_bonus(nullptr, nullptr);
    return POFD_OK;
  });
}

int pofd_ensemble_set_bonus(pofd_ensemble* e, pofd_batch_bonus_fn fn, void* like) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_bonus(fn, like);
    return POFD_OK;
  });
}

int pofd_ensemble_use_like2(pofd_ensemble* e, pofd_like2* like) {
  return guard([&] {
    need(e && like, "null argument");
    e->ens->set_like(like2_batch, like);
    // bonus slots after the two sigma multipliers (pofdMCMCDouble.cc:408-415)
    if (e->ens->npar() >= like->eng->nparams() + 6)
      e->ens->set_bonus(like2_fill, like);
    else
      e->ens->set_bonus(nullptr, nullptr);
    return POFD_OK;
  });
}

int pofd_ensemble_set_param_state(pofd_ensemble* e, unsigned idx, int state) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_param_state(idx, state);
    return POFD_OK;
  });
}

int pofd_ensemble_set_param_limits(pofd_ensemble* e, unsigned idx, float lo, float hi) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_limits(idx, lo, hi);
    return POFD_OK;
  });
}

int pofd_ensemble_set_temperature(pofd_ensemble* e, double temp) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_temperature(temp);
    return POFD_OK;
  });
}

int pofd_ensemble_init(pofd_ensemble* e, const float* walkers, const double* logl) {
  return guard([&] {
    need(e && walkers, "null argument");
    e->ens->init(walkers, logl);
    return POFD_OK;
  });
}

int pofd_ensemble_reserve_chain(pofd_ensemble* e, unsigned nsteps) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->reserve_chain(nsteps);
    return POFD_OK;
  });
}

int pofd_ensemble_clear_chain(pofd_ensemble* e) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->clear_chain();
    return POFD_OK;
  });
}

int pofd_ensemble_do_steps(pofd_ensemble* e, unsigned nsteps, int record) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->do_steps(nsteps, record != 0);
    return POFD_OK;
  });
}

int pofd_ensemble_nrecorded(pofd_ensemble* e, unsigned* n) {
  return guard([&] {
    need(e && n, "null argument");
    *n = e->ens->nrecorded();
    return POFD_OK;
  });
}

int pofd_ensemble_chain(pofd_ensemble* e, float* theta, double* logl) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->chain(theta, logl);
    return POFD_OK;
  });
}

int pofd_ensemble_last(pofd_ensemble* e, float* theta, double* logl) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->last(theta, logl);
    return POFD_OK;
  });
}

int pofd_ensemble_get_counter(pofd_ensemble* e, unsigned long long* step,
                              unsigned long long* seed) {
  return guard([&] {
    need(e && step && seed, "null argument");
    *step = e->ens->step_counter();
    *seed = e->ens->seed();
    return POFD_OK;
  });
}

int pofd_ensemble_set_counter(pofd_ensemble* e, unsigned long long step) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_step_counter(step);
    return POFD_OK;
  });
}

int pofd_ensemble_set_naccept(pofd_ensemble* e, const unsigned* naccept) {
  return guard([&] {
    need(e && naccept, "null argument");
    e->ens->set_naccept(naccept);
    return POFD_OK;
  });
}

int pofd_ensemble_naccept(pofd_ensemble* e, unsigned* naccept) {
  return guard([&] {
    need(e && naccept, "null argument");
    e->ens->naccept(naccept);
    return POFD_OK;
  });
}

int pofd_ensemble_acor(pofd_ensemble* e, double* tau) {
  return guard([&] {
    need(e && tau, "null argument");
    return e->ens->acor(tau) ? POFD_OK : POFD_REJECTED;
  });
}

int pofd_acor(const float* x, size_t n, double* mean, double* sigma, double* tau) {
  return guard([&] {
    need(x && mean && sigma && tau, "null argument");
    need(n > 0, "empty series");
    std::vector<float> v(x, x + n);
    double m = 0, sg = std::numeric_limits<double>::quiet_NaN(),
           t = std::numeric_limits<double>::quiet_NaN();
    const int rc = pofd::acor_series(m, sg, t, v, static_cast<unsigned>(n));
    *mean = m;
    *sigma = sg;
    *tau = t;
    return rc ? POFD_REJECTED : POFD_OK;
  });
}

// ------------------------------------------------------------ surrogate
int pofd_surrogate_create(pofd_ctx* ctx, unsigned nparams, const int* input_idx,
                          unsigned ninputs, unsigned hidden, unsigned capacity,
                          unsigned long long seed, pofd_surrogate** out) {
  return guard([&] {
    need(ctx && input_idx && out, "null argument");
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    std::unique_ptr<pofd_surrogate> s(new pofd_surrogate());
    s->ctx = ctx;
    s->s.reset(new pofd::Surrogate(ctx->device, ctx->stream, nparams, input_idx, ninputs, hidden,
                                   capacity, seed));
    *out = s.release();
    return POFD_OK;
  });
}

int pofd_surrogate_destroy(pofd_surrogate* s) {
  if (s && s->ctx && s->ctx->device >= 0) cudaSetDevice(s->ctx->device);
  delete s;
  return POFD_OK;
}

int pofd_surrogate_add_pairs(pofd_surrogate* s, unsigned n, const float* theta, unsigned npar,
                             const double* logl, const int* status, void* stream) {
  return guard([&] {
    need(s && theta && logl, "null argument");
    s->s->add_pairs(n, theta, npar, logl, status, static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

int pofd_surrogate_npairs(pofd_surrogate* s, unsigned* n) {
  return guard([&] {
    need(s && n, "null argument");
    *n = s->s->npairs();
    return POFD_OK;
  });
}

int pofd_surrogate_get_pairs(pofd_surrogate* s, unsigned n, float* theta_out,
                             double* logl_out) {
  return guard([&] {
    need(s != nullptr, "null argument");
    s->s->pairs_host(n, theta_out, logl_out);
    return POFD_OK;
  });
}

int pofd_surrogate_train(pofd_surrogate* s, unsigned iters, unsigned batch, float lr,
                         float* last_loss) {
  return guard([&] {
    need(s != nullptr, "null argument");
    s->s->train(iters, batch, lr, last_loss);
    return POFD_OK;
  });
}

int pofd_surrogate_predict_device(void* sv, unsigned nprop, const float* theta, unsigned npar,
                                  double* logl, int* status, void* stream) {
  return guard([&] {
    pofd_surrogate* s = static_cast<pofd_surrogate*>(sv);
    need(s && theta && logl, "null argument");
    s->s->predict(nprop, theta, npar, logl, status, static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

int pofd_surrogate_get_params(pofd_surrogate* s, int t, float* out, size_t* size) {
  return guard([&] {
    need(s != nullptr, "null argument");
    need(t >= 0 && t < pofd::Surrogate::kNumTensors, "tensor index out of range");
    if (size) *size = s->s->tensor_size(t);
    if (out) {
      std::vector<std::vector<float>> h;
      s->s->get_params_host(h);
      std::memcpy(out, h[t].data(), h[t].size() * sizeof(float));
    }
    return POFD_OK;
  });
}

int pofd_surrogate_set_params(pofd_surrogate* s, const float* const* tensors) {
  return guard([&] {
    need(s && tensors, "null argument");
    std::vector<std::vector<float>> h(pofd::Surrogate::kNumTensors);
    for (int t = 0; t < pofd::Surrogate::kNumTensors; ++t) {
      need(tensors[t] != nullptr, "null tensor");
      h[t].assign(tensors[t], tensors[t] + s->s->tensor_size(t));
    }
    s->s->set_params_host(h);
    return POFD_OK;
  });
}

int pofd_surrogate_gradients(pofd_surrogate* s, unsigned n, float* const* grads, float* loss) {
  return guard([&] {
    need(s && grads, "null argument");
    float* dev[pofd::Surrogate::kNumTensors];
    for (int t = 0; t < pofd::Surrogate::kNumTensors; ++t) dev[t] = nullptr;
    struct Free {
      float** d;
      ~Free() {
        for (int t = 0; t < pofd::Surrogate::kNumTensors; ++t)
          if (d[t]) cudaFree(d[t]);
      }
    } fr{dev};
    for (int t = 0; t < pofd::Surrogate::kNumTensors; ++t) {
      need(grads[t] != nullptr, "null gradient buffer");
      if (cudaMalloc(&dev[t], s->s->tensor_size(t) * sizeof(float)) != cudaSuccess)
        throw pofd::Error(POFD_E_NOMEM, "cudaMalloc");
    }
    s->s->gradients(n, dev, loss);
    for (int t = 0; t < pofd::Surrogate::kNumTensors; ++t)
      if (cudaMemcpy(grads[t], dev[t], s->s->tensor_size(t) * sizeof(float),
                     cudaMemcpyDeviceToHost) != cudaSuccess)
        throw pofd::Error(POFD_E_CUDA, "D2H gradients");
    return POFD_OK;
  });
}

int pofd_surrogate_scaling(pofd_surrogate* s, double* out) {
  return guard([&] {
    need(s && out, "null argument");
    s->s->scaling(out);
    return POFD_OK;
  });
}

int pofd_bf16_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C,
                   int ldc, void* stream) {
  return guard([&] {
    need(A && B && C, "null argument");
    int* err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) throw pofd::Error(POFD_E_NOMEM, "cudaMalloc");
    struct Free { int* p; ~Free() { cudaFree(p); } } fr{err};
    cudaMemset(err, 0, sizeof(int));
    pofd::bf16_gemm(M, N, K, A, lda, B, ldb, C, ldc, err, static_cast<cudaStream_t>(stream));
    int e = 0;
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess ||
        cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      throw pofd::Error(POFD_E_CUDA, cudaGetErrorString(cudaGetLastError()));
    if (e) throw pofd::Error(POFD_E_CUDA, "tensor-core wait timed out");
    return POFD_OK;
  });
}

int pofd_ensemble_set_surrogate(pofd_ensemble* e, pofd_batch_loglike_fn sfn, void* sur) {
  return guard([&] {
    need(e && sfn, "null argument");
    e->ens->set_stage1(sfn, sur);
    return POFD_OK;
  });
}

int pofd_ensemble_set_da_scale(pofd_ensemble* e, double a) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_da_scale(a);
    return POFD_OK;
  });
}

int pofd_ensemble_collect_pairs(pofd_ensemble* e, pofd_surrogate* s) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->collect_pairs(s ? s->s.get() : nullptr);
    return POFD_OK;
  });
}

int pofd_ensemble_prepare_da(pofd_ensemble* e) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->prepare_da();
    return POFD_OK;
  });
}

int pofd_ensemble_do_steps_da(pofd_ensemble* e, unsigned nsteps, int record) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->do_steps_da(nsteps, record != 0);
    return POFD_OK;
  });
}

int pofd_ensemble_da_stats(pofd_ensemble* e, unsigned long long* out4) {
  return guard([&] {
    need(e && out4, "null argument");
    e->ens->da_stats(out4);
    return POFD_OK;
  });
}

int pofd_likesum_create(pofd_ctx* ctx, pofd_likesum** out) {
  return guard([&] {
    need(ctx && out, "null argument");
    std::unique_ptr<pofd_likesum> l(new pofd_likesum());
    l->ctx = ctx;
    l->ls.reset(new pofd::LikeSum(ctx->device, ctx->stream));
    *out = l.release();
    return POFD_OK;
  });
}

int pofd_likesum_destroy(pofd_likesum* ls) {
  if (ls && ls->ctx && ls->ctx->device >= 0) cudaSetDevice(ls->ctx->device);
  delete ls;
  return POFD_OK;
}

int pofd_likesum_add(pofd_likesum* ls, pofd_batch_loglike_fn fn, void* like) {
  return guard([&] {
    need(ls && fn, "null argument");
    ls->ls->add(fn, like);
    return POFD_OK;
  });
}

int pofd_likesum_add_like1(pofd_likesum* ls, pofd_like1* like) {
  return guard([&] {
    need(ls && like, "null argument");
    ls->ls->add(like1_batch, like);
    return POFD_OK;
  });
}

int pofd_likesum_add_like2(pofd_likesum* ls, pofd_like2* like) {
  return guard([&] {
    need(ls && like, "null argument");
    ls->ls->add(like2_batch, like);
    return POFD_OK;
  });
}

int pofd_likesum_eval_batch_device(void* lv, unsigned nprop, const float* theta, unsigned npar,
                                   double* logl, int* status, void* stream) {
  return guard([&] {
    pofd_likesum* ls = static_cast<pofd_likesum*>(lv);
    need(ls && theta && logl && status, "null argument");
    ls->ls->enqueue(nprop, theta, npar, logl, status, static_cast<cudaStream_t>(stream));
    return POFD_OK;
  });
}

int pofd_ensemble_set_error_policy(pofd_ensemble* e, int reject_failures) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_error_policy(reject_failures != 0);
    return POFD_OK;
  });
}

int pofd_ensemble_set_limit_policy(pofd_ensemble* e, int reject_outside) {
  return guard([&] {
    need(e != nullptr, "null argument");
    e->ens->set_limit_policy(reject_outside != 0);
    return POFD_OK;
  });
}

int pofd_ensemble_failures(pofd_ensemble* e, unsigned long long* n) {
  return guard([&] {
    need(e && n, "null argument");
    *n = e->ens->failures();
    return POFD_OK;
  });
}

// ------------------------------------------------------ 2D P(D) factory
int pofd_pdfactory2_create(pofd_ctx* ctx, unsigned nedge, pofd_pdfactory2** out) {
  return guard([&] {
    need(ctx && out, "null argument");
    std::unique_ptr<pofd_pdfactory2> f(new pofd_pdfactory2());
    f->ctx = ctx;
    f->nedge = nedge;
    *out = f.release();
    return POFD_OK;
  });
}

int pofd_pdfactory2_destroy(pofd_pdfactory2* f) {
  if (f && f->ctx && f->ctx->device >= 0) cudaSetDevice(f->ctx->device);
  delete f;
  return POFD_OK;
}

// PDFactoryDouble::initPD argument checks (PDFactoryDouble.cc:1145-1170),
// then the engine is configured for one beam set with one noise-only
// dataset and the given ranges.
int pofd_pdfactory2_initpd(pofd_pdfactory2* f, unsigned n, double minflux1, double maxflux1,
                           double minflux2, double maxflux2, unsigned nknots,
                           const double* knotpos, unsigned nsigma, const double* sigmapos,
                           unsigned noffset, const double* offsetpos, const float* params,
                           const pofd_beam2* beam, int setedge) {
  return guard([&] {
    need(f && knotpos && sigmapos && offsetpos && params && beam, "null argument");
    if (n == 0) throw pofd::Error(POFD_E_ARG, "Invalid (zero) n");
    if (maxflux1 <= 0.0) throw pofd::Error(POFD_E_ARG, "Invalid (non-positive) maxflux1");
    if (maxflux2 <= 0.0) throw pofd::Error(POFD_E_ARG, "Invalid (non-positive) maxflux2");
    if (minflux1 == maxflux1) throw pofd::Error(POFD_E_ARG, "Invalid range (0) between min/max flux in band 1");
    if (minflux2 == maxflux2) throw pofd::Error(POFD_E_ARG, "Invalid range (0) between min/max flux in band 2");
    const unsigned np = nknots + nsigma + noffset;
    for (unsigned k = 0; k < np; ++k)
      if (std::isnan(static_cast<double>(params[k])))
        throw pofd::Error(POFD_E_INVALID_MODEL, "Invalid model");
    if (f->ctx->device >= 0) cudaSetDevice(f->ctx->device);
    f->eng.reset(new pofd::Engine2(f->ctx->device, f->ctx->stream));
    f->eng->configure(nknots, knotpos, nsigma, sigmapos, noffset, offsetpos, n, f->nedge,
                      setedge != 0, true, 1);
    const int bs = f->eng->add_beamset(beam->b, 0.0, 0.0);
    f->eng->add_virtual_dataset(bs, 1.0, 1.0);
    f->eng->set_rrange_explicit(bs, minflux1, maxflux1, minflux2, maxflux2);
    f->eng->reserve(1);
    f->theta.assign(params, params + np);
    f->theta.push_back(1.0f);  // sigma multipliers; the noise is the dataset's
    f->theta.push_back(1.0f);
    f->inited = true;
    return POFD_OK;
  });
}

int pofd_pdfactory2_getpd(pofd_pdfactory2* f, double sigma1, double sigma2, int setlog,
                          double* pd_out, double* info4) {
  return guard([&] {
    need(f && pd_out, "null argument");
    if (!f->inited) throw pofd::Error(POFD_E_ARG, "Must call initPD first");
    if (f->ctx->device >= 0) cudaSetDevice(f->ctx->device);
    double info[16];
    f->eng->set_virtual_sigma(0, sigma1, sigma2);
    const int st = f->eng->pd_host(0, 0, f->theta.data(), static_cast<unsigned>(f->theta.size()),
                                   setlog != 0, pd_out, info);
    if (info4) {
      info4[0] = info[10];
      info4[1] = info[0];
      info4[2] = info[11];
      info4[3] = info[1];
    }
    if (st != 0) throw pofd::Error(st, "P(D) unwrap failed (split point or mean)");
    return POFD_OK;
  });
}

int pofd_pdfactory2_get_r(pofd_pdfactory2* f, double* rvals_out) {
  return guard([&] {
    need(f && rvals_out, "null argument");
    if (!f->inited) throw pofd::Error(POFD_E_ARG, "Must call initPD first");
    if (f->ctx->device >= 0) cudaSetDevice(f->ctx->device);
    f->eng->rgrid_host(0, f->theta.data(), static_cast<unsigned>(f->theta.size()), rvals_out);
    return POFD_OK;
  });
}

}  // extern "C"
