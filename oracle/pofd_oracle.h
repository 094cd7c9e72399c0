/*
 * pofd_oracle.h -- C API of the CPU FP64 oracle for the P(D) likelihood path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C++ restatement of the
 * reference algorithm (aconley/pofd_affine 0.5.1) used to check the CUDA
 * path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load it, and only as the checker or the timed CPU baseline.  The product
 * library (pofd_affine_b200) never links, loads or calls it.
 *
 * The reference's third-party numerics are restated from their published
 * algorithms (GSL natural cubic spline / linear interpolation / Brent root
 * finder, FFTW's unnormalised r2c/c2r DFT definitions); no GSL, FFTW or
 * reference source is compiled here.  Each routine in pofd_oracle.cc cites
 * the reference file:line it follows.
 *
 * Conventions: every function returns an int status: 0 ok, <0 error (the
 * reference would have thrown affineExcept).  orc_last_error() returns the
 * message of the most recent error on the calling thread.
 */
#ifndef POFD_ORACLE_H
#define POFD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* orc_last_error(void);

/* ---- numerics building blocks (for self-tests) ---- */
int orc_cspline_eval(int n, const double* x, const double* y, int m,
                     const double* xq, double* out);
/* Transforms of the oracle: 0 (default) radix-2, the parity form; 1 the
 * fast radix-4 real transforms (fastfft.hh) for powers of two >= 8, used by
 * the timed CPU baseline.  Process-wide. */
int orc_set_fast_fft(int on);
int orc_rfft(int n, const double* in, double* out_c /* 2*(n/2+1) */);
int orc_irfft(int n, const double* in_c, double* out);
int orc_rfft2(int n, const double* in, double* out_c /* 2*n*(n/2+1) */);
int orc_irfft2(int n, const double* in_c, double* out);

/* ---- 1D beam (beam.cc) ---- */
void* orc_beam1_new(const double* pix, int64_t npix, double pixsize,
                    double minval, unsigned nhist /* 0 = no histogram */);
void orc_beam1_free(void* b);
/* info: [haspos, hasneg, npos, nneg, poshist, neghist, nposhist, nneghist,
 *        minpos, maxpos, minneg, maxneg, pixsize, totpos, totneg] */
int orc_beam1_info(void* b, double* info15);
/* which: 0 pos weights, 1 pos inverse values, 2 neg weights, 3 neg inverse
 * values (histogrammed arrays), 4 pos inverse raw, 5 neg inverse raw */
int orc_beam1_array(void* b, int which, double* out);

/* ---- 1D counts model (numberCountsKnotsSpline.cc) ---- */
int orc_counts1_eval(int nknots, const double* knotpos, const float* theta,
                     int m, const double* s, double* out);
int orc_counts1_getR(int nknots, const double* knotpos, const float* theta,
                     void* beam, int m, const double* flux, double* out,
                     int scalar_version);
int orc_counts1_rrange(int nknots, const double* knotpos, const float* theta,
                       void* beam, double* range2);
int orc_counts1_integrals(int nknots, const double* knotpos,
                          const float* theta, double* ns_s_s2);

/* ---- 1D likelihood (calcLike.cc + PDFactory.cc + PD.cc) ---- */
void* orc_like1_new(int nknots, const double* knotpos, unsigned fftsize,
                    unsigned ninterp, int bin_data, unsigned nbins);
void orc_like1_free(void* L);
/* Adds a beam set; returns its index (>=0) or <0 on error. */
int orc_like1_add_beamset(void* L, const double* beampix, int64_t nbeampix,
                          double pixsize, double minval, int histogram,
                          unsigned nbeamhist, double exp_conf);
int orc_like1_add_dataset(void* L, int beamset, const double* data,
                          int64_t ndata, int meansub, double sigma_base,
                          double like_norm);
int orc_like1_set_rranges(void* L, const float* theta, int npar);
int orc_like1_get_rrange(void* L, int beamset, double* range2);
/* dataset info: [ndata, nbins, bincent0, bindelta, like_offset, sigma_base,
 *                like_norm, minflux, maxflux] */
int orc_like1_dataset_info(void* L, int beamset, int ds, double* info9);
int orc_like1_dataset_bins(void* L, int beamset, int ds, uint32_t* out);
int orc_like1_eval(void* L, const float* theta, int npar, double* logl);
int orc_like1_eval_batch(void* L, int nprop, const float* theta, int npar,
                         double* logl, int* status, int nthreads);
/* P(D) for one dataset.  dbg (may be NULL) receives
 * [dflux, minflux_R, wrapRidx, mn, var_noi, doshift, shift, splitidx,
 *  sgpos, sgneg, pd_minflux, r0]. rvals_out (may be NULL) gets R*dflux (n). */
int orc_like1_pd(void* L, int beamset, int ds, const float* theta, int npar,
                 int setlog, double* pd_out, double* dbg12,
                 double* rvals_out);
/* R at the interpolation nodes (pos branch): x_out, r_out length ninterp. */
int orc_like1_rinterp(void* L, int beamset, const float* theta, int npar,
                      int neg, double* x_out, double* r_out);

/* ---- 2D beam (doublebeam.cc) ---- */
void* orc_beam2_new(const double* pix1, const double* pix2, int64_t npix,
                    double pixsize, double minval, unsigned nhist);
void orc_beam2_free(void* b);
/* info: [hassign0..3, npix0..3, ishist0..3, nhist0..3, pixsize] (17) */
int orc_beam2_info(void* b, double* info17);
/* component sgn; which: 0 weights, 1 inv1, 2 inv2, 3 logratio (effective
 * arrays used by getR: histogram if histogrammed else raw, weight 1) */
int orc_beam2_array(void* b, int sgn, int which, double* out);
int orc_beam2_minmax(void* b, int sgn, double* mm4);

/* ---- 2D counts model (numberCountsDoubleLogNormal.cc) ---- */
void* orc_counts2_new(int nknots, const double* knotpos, int nsigma,
                      const double* sigmapos, int noffset,
                      const double* offsetpos);
void orc_counts2_free(void* m);
int orc_counts2_set(void* m, const float* theta, int npar);
int orc_counts2_eval(void* m, int n, const double* f1, const double* f2,
                     double* out);
int orc_counts2_getR(void* m, void* beam, int n1, const double* f1, int n2,
                     const double* f2, double* out);
int orc_counts2_getR_scalar(void* m, void* beam, int n, const double* f1,
                            const double* f2, double* out);
int orc_counts2_maxflux(void* m, double* mm2);
/* integral of S1^alpha S2^beta dN/dS1 dS2 (splineInt) */
int orc_counts2_spline_int(void* m, double alpha, double beta, double* out);
int orc_counts2_rrange(void* m, void* beam, double* range4);
int orc_counts2_sigma_offset(void* m, int n, const double* f1, double* sig,
                             double* off);

/* ---- 2D likelihood (calcLikeDouble.cc + PDFactoryDouble.cc + PDDouble.cc) */
void* orc_like2_new(int nknots, const double* knotpos, int nsigma,
                    const double* sigmapos, int noffset,
                    const double* offsetpos, unsigned fftsize, unsigned nedge,
                    int edge_integ, int bin_data, unsigned nbins);
void orc_like2_free(void* L);
int orc_like2_add_beamset(void* L, const double* pix1, const double* pix2,
                          int64_t npix, double pixsize, double minval,
                          int histogram, unsigned nbeamhist, double exp_conf1,
                          double exp_conf2);
int orc_like2_add_dataset(void* L, int beamset, const double* d1,
                          const double* d2, int64_t ndata, int meansub,
                          double sigma_base1, double sigma_base2,
                          double like_norm);
int orc_like2_set_rranges(void* L, const float* theta, int npar);
int orc_like2_get_rrange(void* L, int beamset, double* range4);
/* info: [ndata, nbins, bincent01, bincent02, bindelta1, bindelta2,
 *        like_offset, sigma_base1, sigma_base2, like_norm] */
int orc_like2_dataset_info(void* L, int beamset, int ds, double* info10);
int orc_like2_dataset_bins(void* L, int beamset, int ds, uint32_t* out);
int orc_like2_eval(void* L, const float* theta, int npar, double* logl);
/* priors: p17 = per band b (8 entries at 8b) {has_sigma, width, has_cfirb,
 * mean, sigma, has_poisson, mean, sigma}, then regularization_alpha
 * (calcLikeDouble.h:213-232) */
int orc_like2_set_priors(void* L, const double* p17);
/* bonus parameters <S1>, <S2>, <S1^2>, <S2^2> of the model at theta */
int orc_like2_bonus(void* L, const float* theta, int npar, double* out4);
int orc_like2_eval_batch(void* L, int nprop, const float* theta, int npar,
                         double* logl, int* status, int nthreads);
/* dbg: [dflux1, dflux2, mn1, mn2, var1, var2, shift1, shift2, split1,
 *       split2, pd_minflux1, pd_minflux2, sg1pos, sg1neg, sg2pos, sg2neg] */
/* priors: p9 = {has_sigma_prior, sigma_prior_width, has_cfirb_prior,
 * cfirb_mean, cfirb_sigma, has_poisson_prior, poisson_mean, poisson_sigma,
 * regularization_alpha} (calcLike.h:184-195) */
int orc_like1_set_priors(void* L, const double* p9);
/* bonus parameters <S>, <S^2> of the model at theta */
int orc_like1_bonus(void* L, const float* theta, int npar, double* out2);
int orc_like2_pd(void* L, int beamset, int ds, const float* theta, int npar,
                 int setlog, double* pd_out, double* dbg16,
                 double* rvals_out);

#ifdef __cplusplus
}
#endif
#endif
