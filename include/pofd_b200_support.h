/*
 * pofd_b200_support.h -- measurement and test helpers of the B200 P(D)
 * likelihood library, in their own library (libpofd_b200_support.so) so
 * that the likelihood's C ABI (pofd_b200.h) carries only the drop-in
 * interface.  None of these has a counterpart in the reference, which has
 * no GPU code.  Status codes are those of pofd_b200.h.
 */
#ifndef POFD_B200_SUPPORT_H
#define POFD_B200_SUPPORT_H

#include "pofd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Measured FP64 FMA throughput of a device (TFLOP/s, 2 flops per FMA): the
 * denominator of the FP64-bound kernels' roofline. */
int pofd_fp64_peak(int device, double* tflops);

/* Self-check of the table-driven exp2 the R builders use (2^x = 2^k T[j]
 * 2^r, T[j] = 2^(j/256), Taylor series for 2^r): the largest relative
 * difference from the CUDA library exp2 over n arguments in [lo, hi), hi <
 * 1023 (below -1022 the table function returns 0; the check then reports
 * its absolute value). */
int pofd_exp2_check(int device, int n, double lo, double hi, double* max_rel);

/* The tensor-core kernels' failure path, exercised without a fault: a kernel
 * waits with their bounded mbarrier wait (limit try_wait rounds, 1..2^20) on
 * a barrier of arrival count 1, on which nothing arrives (arrive = 0) or one
 * thread arrives before the wait (arrive = 1).  *timed_out = 1 when the wait
 * ran out and the kernel returned that status normally, 0 when it
 * completed. */
int pofd_wait_check(int device, unsigned limit, int arrive, int* timed_out);

/* A multivariate Gaussian test likelihood, log N(theta[0:k]; mean, icov^-1)
 * up to a constant (k <= 64), batched on the device with the
 * pofd_batch_loglike_fn signature (pofd_gauss_eval_batch_device; the work
 * goes on the stream passed): a target with a known posterior for checking
 * the sampler and the surrogate. */
typedef struct pofd_gauss pofd_gauss;
int pofd_gauss_create(int device, unsigned k, const double* mean,
                      const double* icov, pofd_gauss** out);
int pofd_gauss_destroy(pofd_gauss* g);
int pofd_gauss_eval_batch_device(void* g, unsigned nprop,
                                 const float* theta_dev, unsigned npar,
                                 double* logl_dev, int* status_dev,
                                 void* stream);

#ifdef __cplusplus
}
#endif
#endif
