/*
 * pofd_b200.h -- C ABI of the B200 P(D) likelihood library (libpofd_b200.so).
 *
 * Drop-in boundary for the likelihood hot path of aconley/pofd_affine 0.5.1:
 * number counts -> R(x) -> FFT -> exp(R~(w) - R~(0)) * noise -> inverse FFT
 * -> unwrap / normalise / log -> binned log-likelihood, computed in FP64 by
 * hand-written sm_100a kernels with batched cuFFT as the only library call.
 *
 * Plain C types only (pointers, sizes, doubles, floats); no CUDA or torch
 * types appear in the signatures -- streams are passed as void*
 * (a cudaStream_t).  Every function returns an int status:
 *     0   POFD_OK
 *     1   POFD_REJECTED    parameters rejected (the reference's
 *                          pars_invalid; it never sets it in 0.5.1)
 *    <0   an error; pofd_last_error() returns the message (thread-local).
 * The negative codes name the exception the reference would have thrown
 * (affineExcept) at the same point.  Model parameters are float, as in the
 * reference's paramSet (include/paramSet.h:20), and are widened to double
 * exactly as numberCountsKnots::setParams does (numberCountsKnots.cc:265).
 *
 * Objects are not thread-safe (like the reference's PDFactory, which keeps
 * mutable buffers, calcLike.h:47-48): use one object per host thread.
 */
#ifndef POFD_B200_H
#define POFD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define POFD_OK 0
#define POFD_REJECTED 1
#define POFD_E_INVALID_MODEL (-1) /* "Invalid model" (PDFactory.cc:1050) */
#define POFD_E_SPLIT_RANGE (-2)   /* "Not enough flux range" (PDFactory.cc:770) */
#define POFD_E_SPLIT_PEAK (-3)    /* "Peak P(D) value was zero" (PDFactory.cc:787) */
#define POFD_E_SPLIT_MIN (-4)     /* "Minimum in pd is too large" (PDFactory.cc:818) */
#define POFD_E_SPLIT_LOGIC (-5)   /* botidx/topidx logic errors (PDFactory.cc:797-802, 873) */
#define POFD_E_SPLIT_TOP (-6)     /* "Topidx is already below jitter" (PDFactory.cc:886) */
#define POFD_E_SPLIT_NONE (-7)    /* "Unable to find split point" (PDFactory.cc:905) */
#define POFD_E_UNSHIFT (-8)       /* "Un-shift amounts not finite" (PDFactory.cc:996) */
#define POFD_E_ARG (-10)          /* invalid argument / state */
#define POFD_E_CUDA (-11)         /* CUDA or cuFFT failure */
#define POFD_E_NOMEM (-12)        /* device allocation failed */

typedef struct pofd_ctx pofd_ctx;
typedef struct pofd_beam1 pofd_beam1;
typedef struct pofd_like1 pofd_like1;
typedef struct pofd_pdfactory1 pofd_pdfactory1;
typedef struct pofd_beam2 pofd_beam2;
typedef struct pofd_like2 pofd_like2;
typedef struct pofd_pdfactory2 pofd_pdfactory2;

/* Message of the last error raised on this thread ("" if none). */
const char* pofd_last_error(void);
/* Library version string. */
const char* pofd_version(void);

/* ---------------------------------------------------------------- context
 * One context per GPU: selects the device and owns a CUDA stream.
 * (Replaces the per-rank process set-up of the reference's MPI farm,
 * pofd_affine_mcmc.cc:42 / pofdMCMC.cc:42.)  device = -1 makes a host-only
 * context: the set-up entry points (beams, datasets, R ranges, dataset
 * info) work on it, anything that needs a GPU returns POFD_E_CUDA. */
int pofd_ctx_create(int device, pofd_ctx** out);
int pofd_ctx_destroy(pofd_ctx* ctx);
/* The context's stream (a cudaStream_t), for callers that enqueue work. */
int pofd_ctx_stream(pofd_ctx* ctx, void** stream_out);
int pofd_ctx_synchronize(pofd_ctx* ctx);

/* ------------------------------------------------------------ FITS input
 * The FITS images the reference's drivers read (no GPU needed).  Both use
 * the two-call pattern: with out == NULL only the sizes are returned.
 *
 * pofd_fits_read_data replaces fitsData::readData(file, ignore_mask,
 * meansub) (fitsData.cc:56-316): the image of an "image"/"IMAGE" extension,
 * else of the primary HDU (a "file.fits[k]" suffix selects HDU k), minus the
 * pixels a "mask"/"MASK" extension marks non-zero, in file order; *n = the
 * pixels kept; errors as the reference ("All data masked", mask extent
 * mismatch, not 2D).  The values feed pofd_like1_add_dataset (meansub = 0
 * there if done here) or, one map per band, pofd_like2_add_dataset.
 *
 * pofd_fits_read_beam replaces beam::readFile (beam.cc:295-395) and each
 * band of doublebeam's: the primary HDU (or HDU k), its PIXSIZE (else
 * PIXSCALE) keyword, nx * ny pixels in file order; the values feed
 * pofd_beam1_create / pofd_beam2_create. */
int pofd_fits_read_data(const char* path, int ignore_mask, int meansub, double* out,
                        size_t cap, size_t* n);
int pofd_fits_read_beam(const char* path, double* out, size_t cap, size_t* nx, size_t* ny,
                        double* pixsize);
/* fitsDataDouble::readData (fitsDataDouble.cc:304-430): the two bands' maps
 * (same pixel count, else an error); with a mask in both files a pixel is
 * dropped where the two mask values share a set bit (mask1 & mask2 != 0),
 * with one mask where it is non-zero; meansub per band. */
int pofd_fits_read_data2(const char* path1, const char* path2, int ignore_mask, int meansub,
                         double* out1, double* out2, size_t cap, size_t* n);

/* ------------------------------------------------------------- 1D beam
 * Replaces beam::beam(filename, histogram, NBINS, MINVAL) (beam.h:69) with
 * an in-memory pixel array: beam::readFile's selection and sorting
 * (beam.cc:295-458) and, if nhist > 0, beam::makeHistogram(nhist)
 * (beam.cc:467-556).  pix holds npix beam values (any order, NaN/inf
 * skipped); pixsize in arcsec. */
int pofd_beam1_create(const double* pix, size_t npix, double pixsize,
                      double minval, unsigned nhist, pofd_beam1** out);
int pofd_beam1_destroy(pofd_beam1* b);
/* info[15] = {haspos, hasneg, npos, nneg, poshist, neghist, nposhist,
 *  nneghist, minpos, maxpos, minneg, maxneg, pixsize, totpos, totneg}
 * (beam.h accessors hasPos..getMinMaxNeg). */
int pofd_beam1_info(const pofd_beam1* b, double* info15);
/* The weight / inverse-beam lists the R sum runs over for one side
 * (numberCountsKnotsSpline.cc:463-477), written to caller arrays of at least
 * *nterms entries (pass NULL arrays to query *nterms). */
int pofd_beam1_terms(const pofd_beam1* b, int negative_side, size_t* nterms,
                     double* weights, double* inv_beam);

/* ------------------------------------------------------- 1D P(D) factory
 * PDFactory (PDFactory.h:136-140).  initPD computes R on the GPU from the
 * knot model (numberCountsKnotsSpline: knots at knotpos[nknots] Jy, log10
 * values knotvals[nknots]), FFTs it and forms exp(R~ - R~0) with the mean
 * shift; getPD applies the noise, inverse-FFTs, unwraps, normalises and
 * (setlog) takes log2, writing n values to pd_out (host) plus the flux of
 * element 0 and the step. */
int pofd_pdfactory1_create(pofd_ctx* ctx, unsigned ninterp,
                           pofd_pdfactory1** out);
int pofd_pdfactory1_destroy(pofd_pdfactory1* f);
int pofd_pdfactory1_initpd(pofd_pdfactory1* f, unsigned n, double minflux,
                           double maxflux, unsigned nknots,
                           const double* knotpos, const float* knotvals,
                           const pofd_beam1* beam);
int pofd_pdfactory1_getpd(pofd_pdfactory1* f, double sigma, int setlog,
                          double* pd_out, double* minflux_out,
                          double* dflux_out);
/* R (times dflux, as the factory holds it) on the n-point wrapped grid. */
int pofd_pdfactory1_get_r(pofd_pdfactory1* f, double* rvals_out);

/* ---------------------------------------------------------- 1D likelihood
 * calcLike (calcLike.h:166-275): datasets grouped into beam sets, one
 * P(D) per beam set and proposal, one noise level per dataset.
 *   create          calcLike(fftsize, ninterp, binned, nbins) + knot
 *                   positions (setKnotPositions)
 *   add_beamset     one beam group (calcLike.cc:741-755); exp_conf is the
 *                   expected confusion noise used by setSigmaBase/setRRange
 *   add_dataset     fitsData read + optional mean subtraction + binning
 *                   (fitsData.cc:393-437) with its sigma_base and like_norm
 *   set_rranges     setRRanges(p) (calcLike.cc:827): freezes the R range
 *   reserve         sizes device work space and cuFFT plans for batches of
 *                   up to max_batch proposals
 *   loglike         getLogLike(p, pars_invalid) for one proposal
 *   eval_batch      getLogLike for nprop proposals theta[nprop][npar]
 *                   (host arrays; synchronous).  status[i] as above.
 *   eval_batch_device  same with device pointers, enqueued on stream
 *                   (void* cudaStream_t, NULL = the context's stream);
 *                   returns after enqueue.
 * The parameter layout is the reference's: nknots log10 knot values, then
 * the sigma multiplier (calcLike.cc:909), then any bonus slots (ignored). */
int pofd_like1_create(pofd_ctx* ctx, unsigned nknots, const double* knotpos,
                      unsigned fftsize, unsigned ninterp, int bin_data,
                      unsigned nbins, pofd_like1** out);
int pofd_like1_destroy(pofd_like1* L);
int pofd_like1_add_beamset(pofd_like1* L, const pofd_beam1* beam,
                           double exp_conf);
int pofd_like1_add_dataset(pofd_like1* L, int beamset, const double* data,
                           size_t ndata, int meansub, double sigma_base,
                           double like_norm);
/* The same for pixels already in device memory (data_dev[ndata], mean-
 * subtracted in place when meansub): the mean subtraction and binning run
 * on the GPU (fitsData::meanSubtract / applyBinning, fitsData.cc:393-437)
 * with the host path's results bit for bit -- the mean is summed in pixel
 * order, every bin index rounded as the host rounds it -- and only the bin
 * counts come back.  An unbinned likelihood copies the pixels back. */
int pofd_like1_add_dataset_device(pofd_like1* L, int beamset, double* data_dev,
                                  size_t ndata, int meansub, double sigma_base,
                                  double like_norm);
/* The GPU ingestion on its own: optional mean subtraction (in place) and
 * binning of ndata device values into nbins counts (bins_dev, device);
 * info3 = {mean (0 without meansub), bincent0, bindelta}.  Synchronises
 * stream (a cudaStream_t; NULL the legacy default stream). */
int pofd_data_bin_device(double* data_dev, size_t ndata, int meansub,
                         unsigned nbins, unsigned* bins_dev, double* info3,
                         void* stream);
int pofd_like1_set_rranges(pofd_like1* L, const float* theta, unsigned npar);
/* range2 = {minRFlux, maxRFlux} of a beam set. */
int pofd_like1_get_rrange(const pofd_like1* L, int beamset, double* range2);
/* The R grid (times dflux) of one beam set for one proposal theta, out[n],
 * as the forward transform sees it (PDFactory::initR, PDFactory.cc:541-620),
 * built by the R fill the tuning selects (materialised forms; the fused
 * form evaluates the same points one exp2 each). */
int pofd_like1_get_r(pofd_like1* L, int beamset, const float* theta,
                     unsigned npar, double* out);
/* info9 = {ndata, nbins, bincent0, bindelta, like_offset, sigma_base,
 *  like_norm, minDataFlux, maxDataFlux}; bins (may be NULL) gets nbins
 *  counts. */
int pofd_like1_dataset_info(const pofd_like1* L, int beamset, int dataset,
                            double* info9, uint32_t* bins);
int pofd_like1_reserve(pofd_like1* L, unsigned max_batch);
int pofd_like1_loglike(pofd_like1* L, const float* theta, unsigned npar,
                       double* logl, int* pars_invalid);
int pofd_like1_eval_batch(pofd_like1* L, unsigned nprop, const float* theta,
                          unsigned npar, double* logl, int* status);
int pofd_like1_eval_batch_device(pofd_like1* L, unsigned nprop,
                                 const float* theta_dev, unsigned npar,
                                 double* logl_dev, int* status_dev,
                                 void* stream);
/* The P(D) of one dataset for one proposal (getPD after initPD), n values
 * to pd_out; info12 (may be NULL) = {dflux, minflux_R, wrapRidx, mean,
 * var_noi, doshift, shift, splitidx, sgpos, sgneg, pd_minflux, 0}. */
int pofd_like1_pd(pofd_like1* L, int beamset, int dataset, const float* theta,
                  unsigned npar, int setlog, double* pd_out, double* info12);
/* R at the ninterp interpolation nodes of a beam set (negative_side 0/1):
 * node fluxes and R (PDFactory.cc:426-527). */
int pofd_like1_rnodes(pofd_like1* L, int beamset, int negative_side,
                      const float* theta, unsigned npar, double* x_out,
                      double* r_out);
/* Number of this library's kernels one eval_batch launches (cuFFT's own
 * kernels not counted). */
int pofd_like1_kernels_per_eval(const pofd_like1* L, int* nkernels);
/* Per-stage device time of one launch sequence over nprop proposals
 * (host theta), averaged over reps runs timed with CUDA events between the
 * stages: stage_ms[i] for i < *nstages (at most 16), names from
 * pofd_like1_stage_name(L, i).  Replaces the reference's -DTIMING clock()
 * accumulators (PDFactory.cc:93-126). */
int pofd_like1_profile(pofd_like1* L, unsigned nprop, const float* theta,
                       unsigned npar, int reps, double* stage_ms,
                       int* nstages);
const char* pofd_like1_stage_name(const pofd_like1* L, int i);
/* Transform used by the likelihood.  By default (no mode set) this
 * library's own FP64 four-step FFT, fused with the R-grid fill and the
 * spectrum, runs when the FFT size is a power of two in [8192, 131072] and
 * cuFFT otherwise (at n = 4096 batched cuFFT is the faster one); mode 0
 * runs the own FFT whenever the size is a power of two in [4096, 131072];
 * mode 1 always uses cuFFT.  pofd_like1_fft_info reports whether the own
 * FFT is in use.  The reference uses FFTW (PDFactory.cc:293-338). */
int pofd_like1_set_fft(pofd_like1* L, int mode);
int pofd_like1_fft_info(pofd_like1* L, int* own);

/* Autotuner of the launch shapes (the project's own; the reference has no
 * GPU and no counterpart): times the whole graph-captured launch sequence on
 * nprop host rows (reps replays per candidate, CUDA events) for each knob in
 * turn -- own FFT vs cuFFT, R-fill points per thread {4, 8, 16}, R-node
 * threads per block {64, 128, 256}, the R grid fill (rfill_mode 0:
 * materialised, one exp2 per grid point; 1: the same inside the forward FFT
 * pass A, the grid never stored; 2: materialised by running products over
 * runs of <= 16 points in one node interval; 3: those runs inside the
 * forward FFT pass A), spectrum blocks per row {2 ... 32} -- and keeps the
 * fastest.  out7 (optional) = {own_fft,
 * rfill_per, rnodes_threads, spec_blocks, rfill_mode, best ms, untuned ms}.
 * get/set_tuning read or impose the five knobs in that order (e.g. a tuning
 * saved from an earlier run).  Results change only by rounding (reduction
 * grouping, FFT implementation, exponential evaluation). */
int pofd_like1_autotune(pofd_like1* L, unsigned nprop, const float* theta,
                        unsigned npar, int reps, double* out7);
int pofd_like1_get_tuning(const pofd_like1* L, int* knobs5);
int pofd_like1_set_tuning(pofd_like1* L, const int* knobs5);

/* Priors added once to the summed log-likelihood, in the reference's order
 * (calcLike.cc:918-952): a Gaussian on the sigma multiplier about 1, on <S>
 * (CFIRB) and on <S^2> (Poisson), then alpha times the log-slope
 * regularisation penalty (numberCountsKnotsSpline.cc:540-559).  on = 0
 * unsets a prior.  Replace calcLike::setSigmaPrior / unsetSigmaPrior,
 * setCFIRBPrior / unsetCFIRBPrior, setPoissonPrior / unsetPoissonPrior and
 * setRegularizationAlpha (calcLike.h:251-269, calcLike.cc:839-877); widths
 * must be positive, means and alpha non-negative. */
int pofd_like1_set_sigma_prior(pofd_like1* L, int on, double width);
int pofd_like1_set_cfirb_prior(pofd_like1* L, int on, double mean, double sigma);
int pofd_like1_set_poisson_prior(pofd_like1* L, int on, double mean, double sigma);
int pofd_like1_set_regularization(pofd_like1* L, double alpha);
/* Bonus parameters <S> and <S^2> of the model of each host row, out
 * [nprop][2]: numberCountsKnotsSpline::getFluxPerArea / getFluxSqPerArea
 * (numberCountsKnotsSpline.cc:300-343), NaN for an invalid model. */
int pofd_like1_bonus(pofd_like1* L, unsigned nprop, const float* theta,
                     unsigned npar, double* out);
/* calcLike::fillBonusParams (calcLike.cc:958-980) on device rows: writes
 * <S>, <S^2> into theta_dev[i][nknots + 1], [nknots + 2]; npar must be at
 * least nknots + 3.  Enqueue only. */
int pofd_like1_fill_bonus_device(pofd_like1* L, unsigned nprop, float* theta_dev,
                                 unsigned npar, void* stream);

/* ------------------------------------------------------------- 2D beam
 * Replaces doublebeam::doublebeam(file1, file2, histogram, NBINS, MINVAL)
 * (doublebeam.h:81) with two in-memory pixel arrays of npix values each:
 * doublebeam::setBeams (doublebeam.cc:331-462) and, if nhist > 0,
 * makeHistogram(nhist) (doublebeam.cc:467-584). */
int pofd_beam2_create(const double* pix1, const double* pix2, size_t npix,
                      double pixsize, double minval, unsigned nhist,
                      pofd_beam2** out);
int pofd_beam2_destroy(pofd_beam2* b);
/* info17 = {hassign[4], npix[4], ishist[4], nhist[4], pixsize} */
int pofd_beam2_info(const pofd_beam2* b, double* info17);

/* ---------------------------------------------------------- 2D likelihood
 * calcLikeDouble (calcLikeDouble.h:192-347) with the log-normal colour
 * model numberCountsDoubleLogNormal: nknots band-1 knots (log10 values),
 * nsigma sigma knots and noffset offset knots (1: constant, 2: linear, >= 3:
 * natural cubic spline, as numberCountsDoubleLogNormal.cc:109-139).  One
 * square fftsize for all beam sets (calcLikeDouble.h:241); edge integration
 * with nedge steps as PDFactoryDouble::initR (PDFactoryDouble.cc:355-585).
 * Parameter layout: knot values, sigma values, offset values, sigma
 * multiplier band 1, band 2 (calcLikeDouble.cc:1217-1218), bonus slots
 * ignored.  bin_data != 0 bins each dataset nbins x nbins
 * (fitsDataDouble.cc:557-608, PDDouble.cc:1103-1222); 0 evaluates the
 * per-pixel likelihood (PDDouble.cc:994-1051). */
int pofd_like2_create(pofd_ctx* ctx, unsigned nknots, const double* knotpos,
                      unsigned nsigma, const double* sigmapos,
                      unsigned noffset, const double* offsetpos,
                      unsigned fftsize, unsigned nedge, int edge_integ,
                      int bin_data, unsigned nbins, pofd_like2** out);
int pofd_like2_destroy(pofd_like2* L);
int pofd_like2_add_beamset(pofd_like2* L, const pofd_beam2* beam,
                           double exp_conf1, double exp_conf2);
int pofd_like2_add_dataset(pofd_like2* L, int beamset, const double* data1,
                           const double* data2, size_t ndata, int meansub,
                           double sigma_base1, double sigma_base2,
                           double like_norm);
/* Two-band pixels in device memory: the GPU mean subtraction and 2D binning
 * (fitsDataDouble.cc:557-608) with the host path's results bit for bit. */
int pofd_like2_add_dataset_device(pofd_like2* L, int beamset, double* d1_dev,
                                  double* d2_dev, size_t ndata, int meansub,
                                  double sigma1, double sigma2,
                                  double like_norm);
/* The two-band ingestion on its own: counts [nbins1][nbins2] (bins_dev);
 * info6 = {mean1, mean2, bincent01, bindelta1, bincent02, bindelta2}. */
int pofd_data2_bin_device(double* d1_dev, double* d2_dev, size_t ndata,
                          int meansub, unsigned nbins1, unsigned nbins2,
                          unsigned* bins_dev, double* info6, void* stream);
/* setRRanges (calcLikeDouble.h:279, calcLikeDouble.cc:496-534). */
int pofd_like2_set_rranges(pofd_like2* L, const float* theta, unsigned npar);
/* range4 = {minRFlux1, maxRFlux1, minRFlux2, maxRFlux2} */
int pofd_like2_get_rrange(const pofd_like2* L, int beamset, double* range4);
/* info10 = {ndata, nbins, bincent01, bincent02, bindelta1, bindelta2,
 *  like_offset, sigma_base1, sigma_base2, like_norm}; bins (may be NULL)
 *  gets nbins*nbins counts. */
int pofd_like2_dataset_info(const pofd_like2* L, int beamset, int dataset,
                            double* info10, uint32_t* bins);
int pofd_like2_reserve(pofd_like2* L, unsigned max_batch);
/* getLogLike(p, pars_invalid) (calcLikeDouble.h:347). */
int pofd_like2_loglike(pofd_like2* L, const float* theta, unsigned npar,
                       double* logl, int* pars_invalid);
int pofd_like2_eval_batch(pofd_like2* L, unsigned nprop, const float* theta,
                          unsigned npar, double* logl, int* status);
int pofd_like2_eval_batch_device(pofd_like2* L, unsigned nprop,
                                 const float* theta_dev, unsigned npar,
                                 double* logl_dev, int* status_dev,
                                 void* stream);
/* PDFactoryDouble::initPD + getPD (PDFactoryDouble.h:142-148) for one
 * dataset: fftsize^2 values (row = band 1); info16 = {dflux1, dflux2, mean1,
 * mean2, var1, var2, shift1, shift2, split1, split2, minflux1, minflux2,
 * sg1pos, sg1neg, sg2pos, sg2neg}. */
int pofd_like2_pd(pofd_like2* L, int beamset, int dataset, const float* theta,
                  unsigned npar, int setlog, double* pd_out, double* info16);
/* R (times dflux1*dflux2, edges filled) on the wrapped fftsize^2 grid. */
int pofd_like2_get_r(pofd_like2* L, int beamset, const float* theta,
                     unsigned npar, double* rvals_out);
int pofd_like2_kernels_per_eval(const pofd_like2* L, int* nkernels);
int pofd_like2_profile(pofd_like2* L, unsigned nprop, const float* theta,
                       unsigned npar, int reps, double* stage_ms,
                       int* nstages);
const char* pofd_like2_stage_name(int i);
/* Stage names of the FFT mode in use (they differ from the above in
 * mode 1). */
const char* pofd_like2_stage_name_now(const pofd_like2* L, int i);

/* FFT of the 2D likelihood (the project's own choice; the reference plans
 * FFTW 2D transforms, PDFactoryDouble.cc:727-768): mode 1 (default) runs
 * batched 1D cuFFT transforms along the rows and this library's kernel that
 * transforms the columns, applies exp/shift/noise per bin and transforms the
 * columns back, where n is a power of two in [512, 4096] (else mode 0);
 * mode 0 runs batched 2D cuFFT transforms with the spectrum kernel between
 * them.  fft_info reports whether the fused column path is in use. */
int pofd_like2_set_fft(pofd_like2* L, int mode);
int pofd_like2_fft_info(const pofd_like2* L, int* fused);

/* Summation order of the 2D normalisation and means (PDDouble::getIntegral,
 * normalize and getMeans, PDDouble.cc:142-208, 355-447).  0 (default): tree
 * sums, exact to ~1e-16 relative.  1: one sequential chain each in the
 * reference's row-major order with every operation rounded separately, so
 * the result carries the reference's own rounding (a few 1e-12 relative at
 * n = 2048, ~1e-5 in a log-likelihood over 2.25 M pixels).  Mode 1 is slow
 * (a 2 n^2-long dependent chain per dataset) and meant for parity checks. */
int pofd_like2_set_reference_sums(pofd_like2* L, int on);
/* Autotuner of the 2D launch shapes (the project's own; no counterpart in
 * the reference): times the whole graph-captured launch sequence on nprop
 * host rows (reps replays per candidate, CUDA events) for each knob in turn
 * -- FFT mode (see pofd_like2_set_fft), R-grid rows per block {2, 4, 8},
 * band-1 edge rows per group {4, 8, 16} -- and keeps the fastest.  out5
 * (optional) = {fft_mode, rgrid_rows, edge_rows, best ms, untuned ms}.
 * get/set_tuning read or impose the three knobs in that order.  Results
 * change only by rounding (reduction grouping, FFT implementation). */
int pofd_like2_autotune(pofd_like2* L, unsigned nprop, const float* theta,
                        unsigned npar, int reps, double* out5);
int pofd_like2_get_tuning(const pofd_like2* L, int* knobs3);
int pofd_like2_set_tuning(pofd_like2* L, const int* knobs3);
/* Work count of the 2D R builders for one proposal theta: out2[0] = the
 * active colour terms (numberCountsDoubleLogNormal.cc:1883-1963, c0 != 0)
 * summed over the main grid rows 1 .. n-1, out2[1] over the edge rows, all
 * beam sets; each term is evaluated once per column.  For roofline
 * accounting; no counterpart in the reference. */
int pofd_like2_active_terms(pofd_like2* L, const float* theta, unsigned npar,
                            long long* out2);

/* Priors per band (band 0 or 1), added once to the summed log-likelihood in
 * the reference's order (calcLikeDouble.cc:1236-1276): Gaussians on the
 * sigma multipliers about 1, on <S_b> and on <S_b^2>, then alpha times the
 * band-1 log-slope penalty.  Replace calcLikeDouble::setSigmaPrior1/2,
 * setCFIRBPrior1/2, setPoissonPrior1/2, their unset forms and
 * setRegularizationAlpha (calcLikeDouble.h:310-341). */
int pofd_like2_set_sigma_prior(pofd_like2* L, int band, int on, double width);
int pofd_like2_set_cfirb_prior(pofd_like2* L, int band, int on, double mean, double sigma);
int pofd_like2_set_poisson_prior(pofd_like2* L, int band, int on, double mean, double sigma);
int pofd_like2_set_regularization(pofd_like2* L, double alpha);
/* <S1>, <S2>, <S1^2>, <S2^2> of each host row, out [nprop][4]
 * (numberCountsDoubleLogNormal::getFluxPerArea / getFluxSqPerArea,
 * numberCountsDoubleLogNormal.cc:1549-1665), NaN for an invalid model. */
int pofd_like2_bonus(pofd_like2* L, unsigned nprop, const float* theta,
                     unsigned npar, double* out);
/* calcLikeDouble::fillBonusParams (calcLikeDouble.cc:1283-1310) on device
 * rows: the four values at theta_dev[i][nmodel + 2 .. nmodel + 5], nmodel =
 * knots + sigma knots + offset knots; npar >= nmodel + 6.  Enqueue only. */
int pofd_like2_fill_bonus_device(pofd_like2* L, unsigned nprop, float* theta_dev,
                                 unsigned npar, void* stream);

/* Allocation-free split / unwrap / normalise / binned log-likelihood of
 * one wrapped 1D P(D) (the inverse-FFT output), for callers that cannot
 * allocate GPU memory when they evaluate: a program whose device memory is
 * already reserved by another allocator, or a latency-sensitive caller that
 * cannot take the synchronisation cudaMalloc/cudaFree imply.  No counterpart
 * in the reference.  All pointers are device pointers owned by the caller:
 * pofd_dev[n] (n <= 262144, larger n returns POFD_E_ARG), the non-zero bins
 * (nzidx_dev[nnz] bin indices, nzcnt_dev[nnz] counts) of data binned at
 * bincent0 + i*bindelta; out_dev[3] receives {(logL - like_offset) /
 * like_norm, split index, flux of the first unwrapped element} and
 * *status_dev the POFD_* status of the split/unwrap.  The grid (dflux,
 * minflux_R, wrapRidx), the variance of R without noise (var_noi) and the
 * noise sigma are those of PDFactory.  Work is enqueued on stream (a
 * cudaStream_t; NULL = the legacy default stream) of the current device; the
 * call returns after enqueueing.  Its scratch is a fixed static device array
 * shared by all calls (one per GPU, held until exit): calls that overlap on
 * the GPU race, so serialise them.  Each call made outside stream capture
 * looks the array's device address up with cudaGetSymbolAddress (so a
 * device reset, which moves the array, is harmless); a call made while its
 * stream is capturing uses the address of the last uncaptured call on that
 * device, so make one call before any stream capture, and none across a
 * device reset inside a capture. */
int pofd_pd1_loglike_noalloc(const double* pofd_dev, unsigned n, double dflux,
                             double minflux_R, unsigned wrapRidx,
                             double var_noi, double sigma,
                             const int* nzidx_dev, const double* nzcnt_dev,
                             unsigned nnz, double bincent0, double bindelta,
                             double like_offset, double like_norm,
                             double* out_dev, int* status_dev, void* stream);

/* ------------------------------------------------------- 2D P(D) factory
 * PDFactoryDouble (PDFactoryDouble.h:142-148): initPD(n, minflux1,
 * maxflux1, minflux2, maxflux2, model, beam, setEdge) with the log-normal
 * colour model given as knot positions plus params (knot log10 values, sigma
 * values, offset values); getPD(sigma1, sigma2, setLog) writes the n x n
 * unwrapped, normalised P(D) (row-major, band 1 major) and info4 =
 * {minflux1, dflux1, minflux2, dflux2}; get_r the R grid (x dflux1 dflux2)
 * the transform sees.  nedge: edge-integral steps (PDFactoryDouble.h:62). */
int pofd_pdfactory2_create(pofd_ctx* ctx, unsigned nedge, pofd_pdfactory2** out);
int pofd_pdfactory2_destroy(pofd_pdfactory2* f);
int pofd_pdfactory2_initpd(pofd_pdfactory2* f, unsigned n, double minflux1,
                           double maxflux1, double minflux2, double maxflux2,
                           unsigned nknots, const double* knotpos,
                           unsigned nsigma, const double* sigmapos,
                           unsigned noffset, const double* offsetpos,
                           const float* params, const pofd_beam2* beam,
                           int setedge);
int pofd_pdfactory2_getpd(pofd_pdfactory2* f, double sigma1, double sigma2,
                          int setlog, double* pd_out, double* info4);
int pofd_pdfactory2_get_r(pofd_pdfactory2* f, double* rvals_out);

/* ------------------------------------------------------------------ MCMC
 * Batched affine-invariant stretch-move ensemble: replaces affineEnsemble
 * (affineEnsemble.h:60-200) and its MPI master/worker farm with one process
 * that evaluates each half of the ensemble in one batched likelihood launch.
 * Parameter states are the reference's mcmc_affine flags
 * (global_settings.h:57). */
#define POFD_PARAM_FIXED 1    /* mcmc_affine::FIXED */
#define POFD_PARAM_ACIGNORE 2 /* mcmc_affine::ACIGNORE */
#define POFD_PARAM_BONUS 4    /* mcmc_affine::BONUS */

/* A batched likelihood: evaluates nprop proposals theta_dev[nprop][npar]
 * (device) into logl_dev[nprop] and status_dev[nprop] (POFD_OK,
 * POFD_REJECTED or an error), enqueued on stream; graph-capturable once it
 * has run once at that batch size.  pofd_like1_eval_batch_device and
 * pofd_like2_eval_batch_device have this signature; it replaces the
 * per-proposal virtual affineEnsemble::getLogLike (affineEnsemble.h:175). */
typedef int (*pofd_batch_loglike_fn)(void* like, unsigned nprop,
                                     const float* theta_dev, unsigned npar,
                                     double* logl_dev, int* status_dev,
                                     void* stream);
/* ------------------------------------------------------ several GPUs
 * The batched likelihood split over the ranks (one process per GPU) of one
 * node; replaces the reference's MPI master/worker farm
 * (affineEnsemble.cc:1233-1521) for one ensemble.  Every rank runs the same
 * ensemble (same seed) with a shard as its likelihood: rank r evaluates
 * rows [P r / W, P (r + 1) / W) of each batch of P proposals with its own
 * replica inner/inner_like (any pofd_batch_loglike_fn), then one NCCL
 * all-gather on the caller's stream assembles the whole batch's logL and
 * status on every rank, so the chains stay identical on every rank and to
 * a single-GPU run's.  pofd_nccl_unique_id (on one rank, shared with the
 * others by the caller) and pofd_shard_create (on every rank, concurrently)
 * set up the communicator; pofd_shard_eval_batch_device has the
 * pofd_batch_loglike_fn signature (a NULL stream is the context's stream,
 * as for the likelihoods).  Batch sizes must first be seen outside a stream
 * capture (buffers are sized then).  NCCL is opened at run time
 * (libnccl.so.2).  pofd_shard_rows gives rank's rows [lo, hi) of a batch. */
typedef struct pofd_shard pofd_shard;
int pofd_shard_rows(unsigned nprop, int world, int rank, unsigned* lo,
                    unsigned* hi);
int pofd_nccl_unique_id(unsigned char* id_out /* 128 bytes */);
int pofd_shard_create(pofd_ctx* ctx, const unsigned char* id, int rank,
                      int world, pofd_batch_loglike_fn inner, void* inner_like,
                      pofd_shard** out);
int pofd_shard_destroy(pofd_shard* s);
int pofd_shard_eval_batch_device(void* s, unsigned nprop,
                                 const float* theta_dev, unsigned npar,
                                 double* logl_dev, int* status_dev,
                                 void* stream);

/* Bonus-parameter hook: fills the bonus slots of nprop device rows that were
 * just evaluated (the slave's fillBonusParams after getLogLike,
 * affineEnsemble.cc:1490-1493).  Enqueue only, on stream. */
typedef int (*pofd_batch_bonus_fn)(void* like, unsigned nprop, float* theta_dev,
                                   unsigned npar, void* stream);

typedef struct pofd_ensemble pofd_ensemble;

/* affineEnsemble(nwalkers, nparams, ..., scalefac) (affineEnsemble.h:100);
 * seed keys the counter-based generator (the reference seeds ran from the
 * clock). */
int pofd_ensemble_create(pofd_ctx* ctx, unsigned nwalkers, unsigned nparams,
                         double scalefac, unsigned long long seed,
                         pofd_ensemble** out);
int pofd_ensemble_destroy(pofd_ensemble* e);
int pofd_ensemble_set_likelihood(pofd_ensemble* e, pofd_batch_loglike_fn fn,
                                 void* like);
/* Convenience: the 1D / 2D likelihoods of this library.  With nparams >=
 * nknots + 3 (1D) or the 2D model's count + 6, the bonus slots after the
 * sigma multipliers are filled on every evaluation, as pofdMCMC /
 * pofdMCMCDouble::fillBonusParams do. */
int pofd_ensemble_use_like1(pofd_ensemble* e, pofd_like1* like);
int pofd_ensemble_use_like2(pofd_ensemble* e, pofd_like2* like);
/* Bonus hook for a caller's likelihood (fn NULL: none; bonus slots stay NaN). */
int pofd_ensemble_set_bonus(pofd_ensemble* e, pofd_batch_bonus_fn fn, void* like);
/* setParamFixed / setParamIgnoreAcor / setParamBonus
 * (affineEnsemble.h:131-140): state is an OR of POFD_PARAM_*. */
int pofd_ensemble_set_param_state(pofd_ensemble* e, unsigned idx, int state);
/* areParamsValid (affineEnsemble.h:183): a proposal is valid when every
 * non-fixed, non-bonus parameter lies in [lo, hi] (pofdMCMC uses the
 * initialisation file's limits and sigma multiplier > 0). */
int pofd_ensemble_set_param_limits(pofd_ensemble* e, unsigned idx, float lo,
                                   float hi);
int pofd_ensemble_set_temperature(pofd_ensemble* e, double temp);
/* Initial walker positions walkers[nwalkers][nparams] (host) and their
 * log-likelihoods (NULL = -infinity, so the first step is always taken, as
 * pofdMCMC::generateInitialPosition does, pofdMCMC.cc:242-290). */
int pofd_ensemble_init(pofd_ensemble* e, const float* walkers,
                       const double* logl);
int pofd_ensemble_reserve_chain(pofd_ensemble* e, unsigned nsteps);
int pofd_ensemble_clear_chain(pofd_ensemble* e);
/* doSteps (affineEnsemble.cc:529-620, doMasterStep 1233-1284): nsteps full
 * steps, recorded into the chain when record != 0 (burn-in passes 0). */
int pofd_ensemble_do_steps(pofd_ensemble* e, unsigned nsteps, int record);
int pofd_ensemble_nrecorded(pofd_ensemble* e, unsigned* n);
/* Recorded chain: theta[nrec][nwalkers][nparams], logl[nrec][nwalkers]
 * (either may be NULL). */
int pofd_ensemble_chain(pofd_ensemble* e, float* theta, double* logl);
int pofd_ensemble_last(pofd_ensemble* e, float* theta, double* logl);
/* Accepted steps per walker (getAcceptanceFrac numerator,
 * affineEnsemble.h:157). */
int pofd_ensemble_naccept(pofd_ensemble* e, unsigned* naccept);
/* Checkpoint / resume (no counterpart: the reference writes its chain once
 * at the end and cannot restart, pofd_affine_mcmc.cc:313-316).  Every
 * random draw is keyed by (seed; step, walker, draw), so the generator's
 * position is one step counter.  A run re-created with the same seed,
 * initialised from pofd_ensemble_last's walkers and log-likelihoods and
 * given the saved counter (and acceptance counts) continues the random
 * stream of the uninterrupted run: the plain stretch-move chains are
 * identical.  (Delayed acceptance also needs its first-stage model
 * restored by the caller.) */
int pofd_ensemble_get_counter(pofd_ensemble* e, unsigned long long* step,
                              unsigned long long* seed);
int pofd_ensemble_set_counter(pofd_ensemble* e, unsigned long long step);
int pofd_ensemble_set_naccept(pofd_ensemble* e, const unsigned* naccept);
/* getAcor (affineEnsemble.h:155, affineChainSet.cc:824-1030): tau[nparams]
 * over the recorded chain, NaN for ACIGNORE parameters; returns POFD_OK, or
 * POFD_REJECTED when some parameter's series was too short (< 50). */
int pofd_ensemble_acor(pofd_ensemble* e, double* tau);

/* ------------------------------------------------------------- surrogate
 * An MLP surrogate of the log-likelihood (inputs: the listed parameters,
 * standardised; 3 hidden layers of `hidden` SiLU units; output logL - max),
 * trained online with Adam on exact (theta, logL) pairs by hand-written
 * BF16 tensor-core (tcgen05, FP32 accumulate) forward and backward kernels.
 * It is the first stage of the delayed-acceptance stretch move.  No
 * counterpart in the reference. */
typedef struct pofd_surrogate pofd_surrogate;
int pofd_surrogate_create(pofd_ctx* ctx, unsigned nparams,
                          const int* input_idx, unsigned ninputs,
                          unsigned hidden, unsigned capacity,
                          unsigned long long seed, pofd_surrogate** out);
int pofd_surrogate_destroy(pofd_surrogate* s);
/* Appends the POFD_OK, finite pairs of device arrays theta_dev[n][npar],
 * logl_dev[n] (status_dev may be NULL) to the ring buffer of capacity
 * pairs; enqueued on stream. */
int pofd_surrogate_add_pairs(pofd_surrogate* s, unsigned n,
                             const float* theta_dev, unsigned npar,
                             const double* logl_dev, const int* status_dev,
                             void* stream);
int pofd_surrogate_npairs(pofd_surrogate* s, unsigned* n);
/* The first n training pairs held, in buffer order, into host arrays
 * theta_out [n][nparams] and logl_out [n] (either may be NULL). */
int pofd_surrogate_get_pairs(pofd_surrogate* s, unsigned n, float* theta_out,
                             double* logl_out);
/* iters Adam steps (lr, beta 0.9/0.999) on minibatches of batch pairs drawn
 * with replacement; the scaling is refreshed from the pairs first. */
int pofd_surrogate_train(pofd_surrogate* s, unsigned iters, unsigned batch,
                         float lr, float* last_loss);
/* Predicted logL, with the pofd_batch_loglike_fn signature. */
int pofd_surrogate_predict_device(void* s, unsigned nprop,
                                  const float* theta_dev, unsigned npar,
                                  double* logl_dev, int* status_dev,
                                  void* stream);
/* Parameters (FP32 masters) by tensor t = 0..7: W1 [hidden][16], b1, W2
 * [hidden][hidden], b2, W3, b3, w4 [hidden], b4 [1]; *size receives the
 * element count.  set_params takes all eight and resets Adam. */
int pofd_surrogate_get_params(pofd_surrogate* s, int t, float* out,
                              size_t* size);
int pofd_surrogate_set_params(pofd_surrogate* s, const float* const* tensors);
/* Mean-square-loss gradients over the first n pairs held, without an
 * update: grads[8] host buffers of the tensor sizes. */
int pofd_surrogate_gradients(pofd_surrogate* s, unsigned n,
                             float* const* grads, float* loss);
/* The input transform and target scaling fixed at the last training:
 * mean[16], W[16][16] (row-major; network inputs x = W (theta_free - mean),
 * W the inverse Cholesky factor of the inputs' covariance, or diagonal 1/sd
 * when that covariance is singular), the target offset (max logL), scale
 * and floor (targets are max(logL - max, -floor) / scale), and 1 when W is
 * the full whitening (276 values). */
int pofd_surrogate_scaling(pofd_surrogate* s, double* out276);
/* The tensor-core main loop on its own, on device pointers of the current
 * device: C[M][N] (fp32, ldc) = A[M][K] * B[N][K]^T, A and B bf16 with
 * leading dimensions multiple of 8, N in [16, 512] and K >= 16 multiples of
 * 16. */
int pofd_bf16_gemm(int M, int N, int K, const void* A, int lda, const void* B,
                   int ldb, float* C, int ldc, void* stream);

/* Delayed acceptance (Christen & Fox 2005) with the stretch move: stage one
 * accepts with min(1, z^(nparams-nfixed-1) e^{(S'-S)/T}) on the surrogate S;
 * only stage-one survivors get the exact likelihood L, accepted with
 * min(1, e^{((L'-L) - (S'-S))/T}), so the chain targets the exact
 * posterior.  sfn/sur evaluate the first stage (pofd_surrogate_predict_device
 * for the surrogate above). */
int pofd_ensemble_set_surrogate(pofd_ensemble* e, pofd_batch_loglike_fn sfn,
                                void* sur);
/* Stretch parameter a (> 1) of the delayed-acceptance steps; 0 (default)
 * uses the plain steps' scalefac.  A rejected first-stage proposal costs a
 * surrogate evaluation only, so a wider stretch than the plain optimum
 * (a = 2) gives more effective samples per exact evaluation; the target
 * stays exact for any a.  No counterpart in the reference. */
int pofd_ensemble_set_da_scale(pofd_ensemble* e, double a);
/* Every exact evaluation of the ensemble is also appended to this
 * surrogate's training pairs (NULL stops collecting). */
int pofd_ensemble_collect_pairs(pofd_ensemble* e, pofd_surrogate* s);
/* Set-up before delayed-acceptance steps: one exact evaluation of every
 * survivor batch size on the buffers the steps use, so that plans and
 * captured graphs are made outside the sampling loop (no counterpart). */
int pofd_ensemble_prepare_da(pofd_ensemble* e);
int pofd_ensemble_do_steps_da(pofd_ensemble* e, unsigned nsteps, int record);
/* Failed likelihood evaluations (a P(D) split or unwrap error, a
 * non-finite logL): reject_failures == 0 (default) stops the run with the
 * error, as the reference's master does ("Problem encountered in slave",
 * affineEnsemble.cc:1346-1352); != 0 rejects the step and counts it
 * (pofd_ensemble_failures). */
int pofd_ensemble_set_error_policy(pofd_ensemble* e, int reject_failures);
/* Steps outside the parameter limits: reject_outside == 0 (default) redraws
 * z up to 40 more times, as the reference's generateNewStep does
 * (affineEnsemble.cc:1144-1228); != 0 rejects such a step at once, the
 * limits acting as a prior that is zero outside them.  Redrawing makes the
 * proposal depend on a walker's distance to a limit and biases the chain
 * where the posterior reaches one; rejecting keeps the stretch move (plain
 * and delayed acceptance alike) exact for the truncated posterior. */
int pofd_ensemble_set_limit_policy(pofd_ensemble* e, int reject_outside);
int pofd_ensemble_failures(pofd_ensemble* e, unsigned long long* n);
/* Counters since init: [0] proposals, [1] stage-one passes, [2] exact
 * evaluations (padding included), [3] accepted moves. */
int pofd_ensemble_da_stats(pofd_ensemble* e, unsigned long long* out4);

/* Sum of batched likelihoods over the same proposals: fields fitted jointly
 * with different FFT sizes (the reference's calcLikeDouble takes one
 * fftsize for all beam sets, calcLikeDouble.h:241), evaluated concurrently
 * on forked streams and summed; statuses combine as the first failure.
 * pofd_likesum_eval_batch_device has the pofd_batch_loglike_fn signature.
 * No counterpart in the reference. */
typedef struct pofd_likesum pofd_likesum;
int pofd_likesum_create(pofd_ctx* ctx, pofd_likesum** out);
int pofd_likesum_destroy(pofd_likesum* ls);
int pofd_likesum_add(pofd_likesum* ls, pofd_batch_loglike_fn fn, void* like);
int pofd_likesum_add_like1(pofd_likesum* ls, pofd_like1* like);
int pofd_likesum_add_like2(pofd_likesum* ls, pofd_like2* like);
int pofd_likesum_eval_batch_device(void* ls, unsigned nprop,
                                   const float* theta_dev, unsigned npar,
                                   double* logl_dev, int* status_dev,
                                   void* stream);

/* Goodman's acor on one series x[n] (affineChainSet.cc:884-951); returns
 * POFD_REJECTED when n < 50 (mean only). */
int pofd_acor(const float* x, size_t n, double* mean, double* sigma,
              double* tau);


#ifdef __cplusplus
}
#endif
#endif
